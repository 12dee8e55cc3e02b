// Kernel argument blocks and launcher declarations shared by the dedup translation units.
#pragma once
#include "common.cuh"
#include "map.cuh"

namespace b2d {

constexpr uint32_t TMA_CONSUMER_WARPS = 8;   // 256 chunks per TMA tile
constexpr uint32_t FOREST_BAND_LEVELS = 12;  // levels fused per forest band launch (4096-leaf subtrees)
constexpr uint32_t SCAN_GRID = 296;          // fixed grid of the reduce-then-scan passes (2 x 148 SMs)
constexpr uint32_t MAX_BUCKETS = 8192;       // source-checkpoint buckets handled per shift partition

struct LeafArgs {
  const uint8_t* data;
  uint64_t len;
  uint32_t cs;
  uint32_t n;       // chunks
  int kind;
  int baseline;
  uint32_t cur;
  Digest* tree;
  uint8_t* lab;
  MapView map;
  DevStatus* st;
};

struct ForestArgs {
  Digest* tree;
  uint8_t* lab;
  uint8_t* push;
  MapView map;
  DevStatus* st;
  const int* zero_exists;   // baseline: does the all-zero digest exist in the map
  uint32_t n, N, D;         // chunks, nodes, deepest level
  uint32_t cur;
  int kind;
  int baseline;
};

// Per-checkpoint sizes, computed on the device so no host round trip is needed mid-checkpoint.
struct DevMeta {
  uint32_t F;            // first-occurrence regions
  uint32_t S;            // shifted-duplicate regions
  uint32_t P;            // prior checkpoints referenced (repeat table rows)
  uint32_t delta;        // pad in front of the diff so its data section is 16-byte aligned
  unsigned long long T;  // chunks in the data section
  unsigned long long diff_len;      // bytes of the diff (header included)
  unsigned long long first_off, count_off, shift_off, data_off;  // byte offsets in the device diff buffer
  unsigned long long map_size;      // occupied map slots after this checkpoint
};

struct DiffArgs {
  const uint8_t* data;   // checkpointed buffer
  uint64_t len;
  uint32_t cs, n, N, D, cur, baseline_id;
  Digest* tree;
  const uint8_t* push;
  MapView map;
  DevStatus* st;
  DevMeta* meta;
  uint32_t* first_list;   // F node ids, canonical order
  uint32_t* shift_list;   // S node ids, canonical order
  uint32_t* region_off;   // F exclusive chunk offsets, then T
  uint32_t* sprev;        // S source node ids
  uint32_t* skey;         // S source checkpoint ids
  uint32_t* hist;         // cur+1 per-checkpoint counts
  uint32_t* bucket_start; // cur+1 exclusive offsets
  uint32_t* partial;      // SCAN_GRID * max(2, cur+1) scratch
  uint32_t* partial2;     // SCAN_GRID * 2 scratch
  uint8_t* diff;          // device diff buffer
};

int launch_leaves(const LeafArgs& a, int sm_count, bool allow_tma, cudaStream_t stream);
cudaError_t launch_forest(const ForestArgs& a, int phase, cudaStream_t stream);
cudaError_t launch_zero_exists(const MapView& m, int* flag, cudaStream_t stream);
cudaError_t launch_collect_diff(const DiffArgs& a, int sm_count, cudaStream_t stream);

}  // namespace b2d

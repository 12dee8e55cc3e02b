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
  uint8_t* leaflab;   // per chunk: label of leaf n-1+c
  uint8_t* dupflag;   // per chunk: leaf shares a new digest with another leaf (see leaf.cu)
  MapView map;
  DevStatus* st;
};

struct ForestArgs {
  Digest* tree;
  uint8_t* lab;             // per node: labels handed from one band to the next
  uint8_t* leaflab;         // per chunk: leaf labels (relabelled in place by phase 1)
  uint8_t* push;
  MapView map;
  DevStatus* st;
  const int* zero_exists;   // baseline: does the all-zero digest exist in the map
  uint8_t* dupflag;         // per chunk, set by the leaf stage, cleared by phase 1
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
  uint8_t* push;          // cleared by the compaction
  MapView map;
  DevStatus* st;
  DevMeta* meta;
  uint32_t* first_list;   // F node ids, canonical order
  uint32_t* shift_list;   // S node ids, canonical order
  uint32_t* tmp_first;    // F node ids, node order
  uint32_t* tmp_shift;    // S node ids, node order
  uint32_t* levels;       // 2 x 34 level-run starts of the node-order lists
  uint32_t* region_off;   // F exclusive chunk offsets, then T
  uint32_t* sprev;        // S source node ids
  uint32_t* skey;         // S source checkpoint ids
  uint32_t* hist;         // cur+1 per-checkpoint counts
  uint32_t* bucket_start; // cur+1 exclusive offsets
  uint32_t* partial;      // SCAN_GRID * max(2, cur+1) scratch
  uint32_t* partial2;     // SCAN_GRID * 2 scratch
  uint8_t* diff;          // device diff buffer
};

// Tunables of the staged leaf kernel (0 = default).  Chosen per workload by the autotuner.
struct LeafTuning {
  int allow_tma = 1;
  int stages = 0;        // TMA ring depth per CTA (default: a 64 KB ring)
  int ctas_per_sm = 0;   // resident CTAs per SM (default 3)
};
int launch_leaves(const LeafArgs& a, int sm_count, const LeafTuning& tune, cudaStream_t stream);
cudaError_t launch_forest(const ForestArgs& a, int phase, cudaStream_t stream);
int forest_launch_count(uint32_t D);
cudaError_t launch_zero_exists(const MapView& m, int* flag, cudaStream_t stream);
cudaError_t launch_baseline_inserts(const ForestArgs& a, int sm_count, cudaStream_t stream);
cudaError_t launch_collect_diff(const DiffArgs& a, int sm_count, cudaStream_t stream);

}  // namespace b2d

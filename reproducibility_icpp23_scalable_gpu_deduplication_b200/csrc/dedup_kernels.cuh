// Kernel argument blocks and launcher declarations shared by the dedup translation units.
#pragma once
#include <cuda.h>

#include <vector>

#include "common.cuh"
#include "map.cuh"

namespace b2d {

constexpr uint32_t TMA_CONSUMER_WARPS = 8;   // 256 chunks per TMA tile
constexpr uint32_t FOREST_BAND_LEVELS = 12;  // levels fused per forest band launch (4096-leaf subtrees)
constexpr uint32_t SCAN_GRID = 296;          // fixed grid of the reduce-then-scan passes (2 x 148 SMs)
// largest grid of the diff assembly's region-flag compaction and region passes (their partial
// counts are scanned by one CTA of 1024 threads)
#ifndef B2D_COMPACT_GRID
#define B2D_COMPACT_GRID 592
#endif
constexpr uint32_t COMPACT_GRID = B2D_COMPACT_GRID;
static_assert(COMPACT_GRID <= 1024, "one scan CTA");
constexpr uint32_t MAX_BUCKETS = 8192;       // source-checkpoint buckets handled per shift partition

// Values that change from one checkpoint to the next.  Kernels read them from device memory
// (not from launch parameters), so one captured launch sequence -- a CUDA graph -- serves every
// checkpoint of a buffer.
struct RoundState {
  uint32_t cur;          // current_id
  uint32_t baseline_id;  // ref_id written into the header
  uint32_t baseline;     // 1: baseline checkpoint
  uint32_t buckets;      // cur + 1: source-checkpoint buckets of the shift entries
  MapView map;           // the digest map (moves when it grows; graphs read it here)
};

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
  const RoundState* rs;
  uint32_t wait_polls;   // 0: the barrier waits' normal bound; else give up after this many
                         // non-blocking polls (a test of the give-up path)
  uint32_t one;          // 1: the MD5 rounds' multiply-add factor (md5_pre_add)
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
  const RoundState* rs;
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
  uint32_t* partial2;     // COMPACT_GRID * 2 scratch
  uint8_t* diff;          // device diff buffer
  const RoundState* rs;
  uint32_t id_bias;       // subtracted from every node id written into the diff (list approach:
                          // n - 1, so leaf heap indices become chunk indices; tree: 0)
};

// Programmatic dependent launch (sm_90 and later).  The forest and diff-assembly kernels of one
// checkpoint are launched with launch_dependent(): each may be scheduled while the kernel before
// it on the stream is still finishing, because every such kernel first lets its own successor
// launch and then waits (griddepcontrol.wait) until its predecessor has completed and its memory
// is visible, before it reads anything.  Launched the ordinary way, both are no-ops.
__device__ __forceinline__ void griddep_enter() {
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
  asm volatile("griddepcontrol.wait;" ::: "memory");
}
template <typename... KArgs, typename... Args>
cudaError_t launch_dependent(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t stream,
                             Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kernel, static_cast<KArgs>(args)...);
}

// launch parameters carry the buffer geometry; the per-checkpoint values come from *rs
__device__ __forceinline__ LeafArgs with_round(const LeafArgs& p) {
  LeafArgs a = p;
  a.cur = p.rs->cur;
  a.baseline = (int)p.rs->baseline;
  a.map = p.rs->map;
  return a;
}
__device__ __forceinline__ ForestArgs with_round(const ForestArgs& p) {
  ForestArgs a = p;
  a.cur = p.rs->cur;
  a.baseline = (int)p.rs->baseline;
  a.map = p.rs->map;
  return a;
}
__device__ __forceinline__ DiffArgs with_round(const DiffArgs& p) {
  DiffArgs a = p;
  a.cur = p.rs->cur;
  a.baseline_id = p.rs->baseline_id;
  a.map = p.rs->map;
  return a;
}

// Tunables of the staged leaf kernel (0 = default).  Chosen per workload by the autotuner.
struct LeafTuning {
  int allow_tma = 1;
  int stages = 0;        // TMA ring depth per CTA (default: a 64 KB ring)
  int ctas_per_sm = 0;   // resident CTAs per SM (default 3)
  int unit = 0;          // staged segment width in bytes (0: the largest of 128/64/32/16 dividing the chunk)
  int wait_polls = 0;    // see LeafArgs::wait_polls
};
int launch_leaves(const LeafArgs& a, int sm_count, const LeafTuning& tune, cudaStream_t stream);

// one buffer of a batched hashing launch (the tensor map must stay 64-byte aligned)
constexpr uint32_t BATCH_MAX_ITEMS = 1024;
struct __align__(64) BatchLeafItem {
  CUtensorMap map;
  LeafArgs args;
  uint32_t nfull;        // whole chunks (TMA rows)
  uint32_t S;            // segments per chunk
  uint32_t tile_begin;   // first global tile of this buffer
  uint32_t ntiles;
};
// Fills `item` for one buffer; returns the segment width U (0: the buffer cannot be staged).
int batch_leaf_item(const LeafArgs& a, BatchLeafItem& item);
// One persistent launch over all items (same U and hash kind).  `queue` is a zeroed counter.
cudaError_t launch_leaves_batch(const BatchLeafItem* d_items, uint32_t nitems, uint32_t total_tiles, int U, int kind,
                                unsigned int* queue, DevStatus* st, int sm_count, const LeafTuning& tune,
                                uint32_t tiles_per_pop, cudaStream_t stream);
// Which forest phases start with a warp band (7 levels per task in phase 1, 9 in phase 2)
// instead of a CTA band (10 and 12 levels): bit 0 phase 1, bit 1 phase 2.  The default of the
// handle parameter "warp_bands" and of the batch tuner's fused-levels knob.
#ifndef B2D_WARP_BANDS
#define B2D_WARP_BANDS 3
#endif
// sm_count > 0: the first band runs on a resident grid (see forest.cu); warp_mask as above
cudaError_t launch_forest(const ForestArgs& a, int phase, cudaStream_t stream, int sm_count = 0,
                          int warp_mask = B2D_WARP_BANDS);

// CTA b of a segmented launch belongs to the handle h with beg[h] <= b < beg[h+1]
__device__ __forceinline__ uint32_t seg_find(const uint32_t* beg, uint32_t n, uint32_t& bid, uint32_t& nb) {
  uint32_t lo = 0, hi = n;
  while (hi - lo > 1) {
    const uint32_t mid = (lo + hi) >> 1;
    if (beg[mid] <= blockIdx.x) lo = mid; else hi = mid;
  }
  bid = blockIdx.x - beg[lo];
  nb = beg[lo + 1] - beg[lo];
  return lo;
}
// one launch of a forest phase of a tree: kind 0 = a full band with input level p0, kind 1 = a
// general band of levels p0 (top) .. p1 (bottom), kind 2 = a warp band over the leaves; `ctas`
// CTAs
struct ForestStep {
  uint8_t kind;
  uint32_t p0, p1, ctas;
};
void forest_steps(uint32_t D, uint64_t N, int phase, std::vector<ForestStep>& out);
// the steps of the batched form: a warp band first where the tree allows one (kind 2: p0 = D,
// one warp per task of 128 (phase 1) or 512 (phase 2) leaves, 8 tasks per CTA), then the bands
// above it
void forest_steps_batch(uint32_t n, uint32_t D, uint64_t N, int phase, std::vector<ForestStep>& out,
                        int warp_mask = B2D_WARP_BANDS);
// the same step of many handles' trees in one launch (batched form); handles without this
// step have no CTAs
struct ForestSeg {
  const ForestArgs* args;
  const uint32_t* beg;   // n + 1
  const uint32_t* p0;    // per handle
  const uint32_t* p1;
  uint32_t n;
};
cudaError_t launch_forest_seg(const ForestSeg& s, int phase, int kind, uint32_t ctas, cudaStream_t stream);
cudaError_t launch_zero_exists_seg(const ForestArgs* args, uint32_t n, cudaStream_t stream);
int forest_launch_count(uint32_t n, uint32_t D, int phase, int warp_mask = B2D_WARP_BANDS);
cudaError_t launch_zero_exists(int* flag, const RoundState* rs, cudaStream_t stream);
// bcap: bucket capacity the scratch was sized for (>= rs->buckets of every checkpoint run).
// node_order: the region lists stay in node order (the list approach's order, whose regions
// are single leaves) instead of the tree's level-descending order.
cudaError_t launch_collect_diff(const DiffArgs& a, uint32_t bcap, int sm_count, cudaStream_t stream,
                                bool node_order = false);
// the list approach's labels: the lowest-index owner of a digest shared by several changed
// chunks stays the first occurrence, the others become shifted duplicates; region flags are
// set for both (src/list_approach.cpp:41-71)
cudaError_t launch_list_label(const ForestArgs& a, int sm_count, cudaStream_t stream);

// Diff assembly of many handles in one launch per step (batched form).  A segmented launch
// gives handle h the CTAs beg[h] .. beg[h+1]-1 and runs its kernels as if launched alone on
// that many CTAs.
struct SegGrid {
  const DiffArgs* args;   // per handle
  const uint32_t* beg;    // n + 1 CTA offsets of the launch
  const uint32_t* g;      // per handle: CTAs of its compaction and region launches
  const uint32_t* gs;     // per handle: CTAs of its shift-entry launches
  const uint32_t* bcap;   // per handle: bucket capacity of its scratch
  uint32_t n;
};
// grid sizes of one handle's diff assembly; variant = data-gather kernel (0: 16-byte
// copies, 1: byte copies)
struct DiffGrids {
  uint32_t g, gs, gl, gp, gg;
  int variant;
};
constexpr int GATHER_VARIANTS = 2;
DiffGrids diff_grids(const DiffArgs& a, int sm_count);
struct DiffBatch {
  SegGrid base;                     // beg unused
  const uint32_t* beg_one;          // one CTA per handle that takes part (prefix table)
  const uint32_t* beg_g;
  const uint32_t* beg_gl;
  const uint32_t* beg_gp;
  const uint32_t* beg_gs;
  const uint32_t* beg_gather[GATHER_VARIANTS];
  uint32_t tot_one;                 // handles with one CTA in the scan and layout launches
  uint32_t tot_g, tot_gl, tot_gp, tot_gs, tot_gather[GATHER_VARIANTS];
  uint32_t max_bcap;
};
// launches (count returned in *launches); the handles' hist arrays are cleared here
cudaError_t launch_collect_diff_batch(const DiffBatch& b, cudaStream_t stream, uint32_t* launches);

}  // namespace b2d

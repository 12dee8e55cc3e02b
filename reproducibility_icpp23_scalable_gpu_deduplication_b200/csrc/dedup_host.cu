// Host side of the tree deduplicator: state, checkpoint / restart orchestration, logs, and
// the C ABI declared in include/b200dedup.h.
//
// Mirrors TreeDeduplicator (src/tree_approach.cpp of the reference): checkpoint() sets up the
// tree and map (:1594-1623), runs the baseline or incremental dedup (:1644-1653), assembles
// the diff (:1668) and copies it to the host (:1683-1684); restart() rebuilds a checkpoint
// from the chain of diffs (:712-1128).  Differences in mechanics, not in output:
//   * no host synchronisation inside a checkpoint: every size is computed on the device,
//     the host reads one small record (DevMeta + DevStatus) at the end;
//   * errors are status codes; device kernels record failures instead of trapping.
#include <cuda_runtime.h>

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <algorithm>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include "../../include/b200dedup.h"
#include "dedup_kernels.cuh"
#include "hash.cuh"
#include "map.cuh"
#include "restart.cuh"

namespace b2d {

static int cuda_status(cudaError_t e) {
  if (e == cudaSuccess) return B2D_OK;
  if (e == cudaErrorMemoryAllocation) return B2D_ERR_NOMEM;
  return B2D_ERR_CUDA;
}
#define B2D_CU(expr)                          \
  do {                                        \
    cudaError_t _e = (expr);                  \
    if (_e != cudaSuccess) return cuda_status(_e); \
  } while (0)

template <class T>
struct DevBuf {
  T* p = nullptr;
  size_t n = 0;
  ~DevBuf() { release(); }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
  cudaError_t reserve(size_t count) {
    if (count <= n && p) return cudaSuccess;
    release();
    if (count == 0) count = 1;
    cudaError_t e = cudaMalloc(&p, count * sizeof(T));
    if (e == cudaSuccess) n = count;
    else p = nullptr;
    return e;
  }
};

template <class T>
struct PinnedBuf {
  T* p = nullptr;
  size_t n = 0;
  ~PinnedBuf() { release(); }
  void release() {
    if (p) cudaFreeHost(p);
    p = nullptr;
    n = 0;
  }
  cudaError_t reserve(size_t count) {
    if (count <= n && p) return cudaSuccess;
    release();
    if (count == 0) count = 1;
    cudaError_t e = cudaMallocHost(&p, count * sizeof(T));
    if (e == cudaSuccess) n = count;
    else p = nullptr;
    return e;
  }
  // for buffers whose size drifts from call to call (diffs): grow by a quarter plus slack, so a
  // diff a few bytes longer than the last one does not free and re-pin tens of megabytes
  cudaError_t grow(size_t count) {
    if (count <= n && p) return cudaSuccess;
    const size_t unit = (1u << 20) / sizeof(T) + 1;
    return reserve((count + count / 4 + unit - 1) / unit * unit);
  }
};

// move every occupied slot of `from` into the (empty) table `to`
__global__ void map_rehash_kernel(MapView from, MapView to, DevStatus* st) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i <= from.cap;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const unsigned long long v = *map_val(from, i);
    if (i == from.cap) {   // the extra slot (the all-ones digest), present when its value is set
      if (v != MAP_EMPTY) *map_val(to, to.cap) = v;
      continue;
    }
    const Key128 k = *map_key(from, i);
    if (k.lo == MAP_EMPTY && k.hi == MAP_EMPTY) continue;
    Digest d;
    d.w[0] = (uint32_t)k.lo; d.w[1] = (uint32_t)(k.lo >> 32);
    d.w[2] = (uint32_t)k.hi; d.w[3] = (uint32_t)(k.hi >> 32);
    const MapRef r = map_insert_packed(to, d, v, st);
    if (r.found) *map_val(to, r.slot) = v;
  }
}

__global__ void hash_chunks_kernel(int kind, const uint8_t* data, uint64_t len, uint32_t cs, uint64_t n, Digest* out) {
  for (uint64_t c = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; c < n; c += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t off = c * cs;
    const uint64_t nb = (c == n - 1) ? len - off : cs;
    out[c] = hash_bytes(kind, data + off, nb);
  }
}

struct DevState {
  DevStatus status;
  int zero_exists;
  unsigned int pad;
  DevMeta meta;
  StraddleInfo straddle;
  RoundState round;
};

}  // namespace b2d

using namespace b2d;

// default size of a baseline's digest map over its minimum, and the factor a growing map
// takes over its new minimum.  A baseline's minimum is its own N entries plus the next
// checkpoint's N at the load limit: 2N / 0.75; times 1.5 that is 4N slots (32 B each, 128 B per
// node: 2 bytes per byte of a 4 GiB buffer at 128-byte chunks), at load 0.25 after the
// baseline, and the table grows only once its entries pass 2N (after about a hundred
// checkpoints that each change 1% of the chunks).
constexpr double MAP_HEADROOM = 1.5;
constexpr double MAP_GROWTH = 2.0;

struct b2d_dedup {
  // BaseDeduplicator state (include/deduplicator_interface.hpp:16-23)
  uint32_t chunk_size = 0;
  uint32_t current_id = 0;
  uint32_t baseline_id = 0;
  uint64_t data_len = 0;
  uint64_t datasizes[2] = {0, 0};
  double timers[4] = {0, 0, 0, 0};
  double restart_timers[2] = {0, 0};
  int kind = HASH_MURMUR3;
  int list = 0;   // 1: ListDeduplicator (src/list_approach.cpp), 0: TreeDeduplicator

  uint32_t n = 0, N = 0, D = 0;
  uint64_t F = 0, S = 0;
  uint32_t launches = 0;
  double phase[3] = {0, 0, 0};   // device time of leaves, forest, diff assembly (last checkpoint)
  bool leaf_tma = false;
  bool have_tree = false;
  LeafTuning tune;
  double map_max_load = 0.75;
  // replay each checkpoint's launches as one CUDA graph (off by default: on the 4 GiB series
  // the graph launch measured 0.15-0.2 ms slower per checkpoint than the 22 stream launches)
  bool use_graph = false;
  bool graph_timing = true;       // phase timing events inside the graph
  double map_headroom = MAP_HEADROOM;   // baseline table size over its minimum (entries + N at max load)
  bool map_retune = false;              // resize an existing table to map_headroom at the next checkpoint
  int warp_bands = B2D_WARP_BANDS;      // forest phases that start with a warp band (bit 0: 1, bit 1: 2)

  cudaStream_t own_stream = nullptr;
  cudaStream_t cap_stream = nullptr;   // graph capture only
  cudaStream_t stream = nullptr;
  int device = 0;
  int sm_count = 148;
  cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};

  DevBuf<Digest> tree;
  DevBuf<uint8_t> lab, leaflab, push, dupflag;
  void* map_mem = nullptr;        // map_cap + 1 keys, then their values (map_at), from the library's map pool
  uint64_t map_cap = 0;
  double map_grow_s = 0;          // host seconds spent growing the map (all checkpoints)
  double map_alloc_s = 0;         // host seconds in the map allocation calls (all tables)
  uint32_t map_grows = 0;
  uint64_t map_size_host = 0;     // occupied slots after the last checkpoint
  DevBuf<unsigned long long> map_size;
  DevBuf<uint32_t> tmp_first, tmp_shift, levels;
  DevBuf<uint32_t> first_list, shift_list, region_off, sprev, skey, hist, bucket_start, partial, partial2;
  DevBuf<uint8_t> diff;
  DevBuf<DevState> state;
  PinnedBuf<DevState> state_h;
  PinnedBuf<RoundState> round_h;   // this checkpoint's RoundState, uploaded by the graph
  const void* data = nullptr;      // buffer of the current checkpoint
  uint32_t bcap = 0;               // source-checkpoint bucket capacity of the scratch
  cudaGraphExec_t graph_exec = nullptr;
  std::vector<uint64_t> graph_key;
  PinnedBuf<uint8_t> diff_h;
  uint64_t diff_len = 0;
  uint32_t diff_delta = 0;
  bool diff_valid = false;

  // restart scratch
  DevBuf<uint2> r_node_list, r_rep;      // restart: NodeIDs of the main diff's chunks; slots' rep
  DevBuf<uint32_t> r_dist;                 // slots' data offsets
  DevBuf<uint8_t> r_mflag, r_flag;
  DevBuf<uint32_t> r_offs, r_partial;      // r_offs: offsets, region starts, source starts, trees
  DevBuf<unsigned long long> r_cum, r_total;
  DevBuf<uint8_t> r_diff;
  PinnedBuf<uint8_t> r_stage;

  ~b2d_dedup();
};

namespace {

// Device memory pool for digest maps (one per device).  Maps are the largest allocations and
// the only ones that grow during a series: the pool keeps freed maps' memory for the next
// growth instead of returning it to the driver, and its frees are stream-ordered, so growing
// a map neither waits for the whole device nor maps fresh pages each time.  Unused memory
// goes back to the driver when a handle is destroyed.
std::mutex g_pool_mu;
std::vector<uint64_t> g_pool_keep;   // bytes each device's pool keeps mapped (b2d_pool_reserve)

cudaMemPool_t map_pool(int device) {
  static std::mutex mu;
  static std::vector<cudaMemPool_t> pools;
  std::lock_guard<std::mutex> lock(mu);
  if ((int)pools.size() <= device) pools.resize(device + 1, nullptr);
  if (!pools[device]) {
    cudaMemPoolProps props;
    std::memset(&props, 0, sizeof(props));
    props.allocType = cudaMemAllocationTypePinned;
    props.handleTypes = cudaMemHandleTypeNone;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = device;
    cudaMemPool_t p = nullptr;
    if (cudaMemPoolCreate(&p, &props) != cudaSuccess) return nullptr;
    uint64_t keep = ~0ull;
    cudaMemPoolSetAttribute(p, cudaMemPoolAttrReleaseThreshold, &keep);
    pools[device] = p;
  }
  return pools[device];
}

}  // namespace

b2d_dedup::~b2d_dedup() {
  {
    if (map_mem) {
      cudaStream_t s = own_stream ? own_stream : stream;
      cudaFreeAsync(map_mem, s);
      cudaStreamSynchronize(s);
      if (cudaMemPool_t p = map_pool(device)) {
        std::lock_guard<std::mutex> lock(g_pool_mu);
        cudaMemPoolTrimTo(p, device < (int)g_pool_keep.size() ? g_pool_keep[device] : 0);
      }
    }
    if (graph_exec) cudaGraphExecDestroy(graph_exec);
    for (auto& e : ev)
      if (e) cudaEventDestroy(e);
    if (own_stream) cudaStreamDestroy(own_stream);
    if (cap_stream) cudaStreamDestroy(cap_stream);
  }
}

namespace {

// A timing event inside a stream capture must be an external record node (a plain record only
// joins streams there); outside a capture it is an ordinary record.
cudaError_t record_timing(cudaEvent_t ev, cudaStream_t s) {
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  cudaError_t e = cudaStreamIsCapturing(s, &cs);
  if (e != cudaSuccess) return e;
  return cs == cudaStreamCaptureStatusActive ? cudaEventRecordWithFlags(ev, s, cudaEventRecordExternal)
                                             : cudaEventRecord(ev, s);
}

// events that were never recorded (a failed launch) read as 0 and leave no error behind for
// the next call's launch checks
float elapsed_ms(cudaEvent_t a, cudaEvent_t b) {
  float ms = 0.f;
  if (cudaEventElapsedTime(&ms, a, b) != cudaSuccess) {
    (void)cudaGetLastError();
    ms = 0.f;
  }
  return ms;
}

double secs(std::chrono::high_resolution_clock::time_point a, std::chrono::high_resolution_clock::time_point b) {
  return std::chrono::duration<double>(b - a).count();
}

template <class T>
uint64_t buf_bytes(const DevBuf<T>& b) {
  return b.p ? (uint64_t)b.n * sizeof(T) : 0;
}

// device bytes a handle holds (everything it allocated with cudaMalloc)
uint64_t handle_bytes(const b2d_dedup* d) {
  return buf_bytes(d->tree) + buf_bytes(d->lab) + buf_bytes(d->leaflab) + buf_bytes(d->push) +
         buf_bytes(d->dupflag) + (d->map_mem ? (d->map_cap + 1) * MAP_SLOT_BYTES : 0) +
         buf_bytes(d->map_size) + buf_bytes(d->tmp_first) +
         buf_bytes(d->tmp_shift) + buf_bytes(d->levels) + buf_bytes(d->first_list) + buf_bytes(d->shift_list) +
         buf_bytes(d->region_off) + buf_bytes(d->sprev) + buf_bytes(d->skey) + buf_bytes(d->hist) +
         buf_bytes(d->bucket_start) + buf_bytes(d->partial) + buf_bytes(d->partial2) + buf_bytes(d->diff) +
         buf_bytes(d->state) + buf_bytes(d->r_node_list) + buf_bytes(d->r_rep) + buf_bytes(d->r_dist) +
         buf_bytes(d->r_mflag) + buf_bytes(d->r_flag) +
         buf_bytes(d->r_offs) + buf_bytes(d->r_partial) + buf_bytes(d->r_cum) + buf_bytes(d->r_total) +
         buf_bytes(d->r_diff);
}

int map_view(b2d_dedup* d, MapView& m) {
  m = map_at(d->map_mem, d->map_cap, d->map_size.p);
  return B2D_OK;
}

// a fresh map of `cap` slots (+ the special slot) on the handle's stream
int map_alloc(b2d_dedup* d, uint64_t cap, void** out) {
  cudaMemPool_t pool = map_pool(d->device);
  if (!pool) return B2D_ERR_CUDA;
  const auto t0 = std::chrono::high_resolution_clock::now();
  B2D_CU(cudaMallocFromPoolAsync(out, MAP_SLOT_BYTES * (cap + 1), pool, d->stream));
  d->map_alloc_s += secs(t0, std::chrono::high_resolution_clock::now());
  // all keys EMPTY, all values all-ones (the extra slot: absent)
  B2D_CU(cudaMemsetAsync(*out, 0xff, MAP_SLOT_BYTES * (cap + 1), d->stream));
  return B2D_OK;
}

int map_reset(b2d_dedup* d, uint64_t cap) {
  if (!d->map_mem || d->map_cap != cap) {
    void* fresh = nullptr;
    int rc = map_alloc(d, cap, &fresh);
    if (rc) return rc;
    if (d->map_mem) cudaFreeAsync(d->map_mem, d->stream);
    d->map_mem = fresh;
    d->map_cap = cap;
  } else {
    B2D_CU(cudaMemsetAsync(d->map_mem, 0xff, MAP_SLOT_BYTES * (cap + 1), d->stream));
  }
  B2D_CU(d->map_size.reserve(1));
  B2D_CU(cudaMemsetAsync(d->map_size.p, 0, sizeof(unsigned long long), d->stream));
  d->map_size_host = 0;
  return B2D_OK;
}

// Capacity policy.  The reference rehashes when capacity < size + num_nodes
// (src/tree_approach.cpp:1622-1623): room for every node of the next checkpoint to be new.
// Here that room must fit under the load limit map_max_load (default 0.75), so no checkpoint
// can push the table past it: a new table holds its entries plus N at that load, times
// map_headroom (default 1.5) at a baseline and MAP_GROWTH when it grows.  Growing allocates and
// rehashes (allocation dominates: tens of ms per GB), so a series whose digests keep changing
// grows less often with more headroom.  Capacities are multiples of 1024, not powers of two.
uint64_t map_capacity(uint64_t need, double max_load, double headroom) {
  const uint64_t c = (uint64_t)((double)need * headroom / max_load) + 1;
  return (c + 1023) / 1024 * 1024;
}

int map_ensure(b2d_dedup* d) {
  const uint64_t need = d->map_size_host + d->N;
  // a retune (the batch tuner's load-factor knob) resizes the table to map_headroom over its
  // minimum, unless it is already within 10 % of that
  uint64_t cap = 0;
  if (d->map_retune && d->map_mem && d->map_size_host > 0) {
    const uint64_t want = map_capacity(need, d->map_max_load, d->map_headroom);
    if (want * 10 < d->map_cap * 9 || want * 9 > d->map_cap * 10) cap = want;
  }
  d->map_retune = false;
  const bool grow = cap == 0;
  if (grow) {
    if (d->map_mem && (double)need <= d->map_max_load * (double)d->map_cap) return B2D_OK;
    cap = map_capacity(need, d->map_max_load, MAP_GROWTH);
  }
  if (!d->map_mem || d->map_size_host == 0) return map_reset(d, cap);
  const auto t0 = std::chrono::high_resolution_clock::now();
  void* fresh = nullptr;
  int rc = map_alloc(d, cap, &fresh);
  if (rc) return rc;
  DevBuf<unsigned long long> cnt;
  B2D_CU(cnt.reserve(1));
  B2D_CU(cudaMemsetAsync(cnt.p, 0, sizeof(unsigned long long), d->stream));
  MapView from, to;
  map_view(d, from);
  to = map_at(fresh, cap, cnt.p);
  map_rehash_kernel<<<(unsigned)d->sm_count * 8u, 256, 0, d->stream>>>(from, to, &d->state.p->status);
  const cudaError_t ke = cudaGetLastError();
  if (ke != cudaSuccess) {
    cudaFreeAsync(fresh, d->stream);
    return cuda_status(ke);
  }
  cudaFreeAsync(d->map_mem, d->stream);
  B2D_CU(cudaStreamSynchronize(d->stream));
  d->map_mem = fresh;
  std::swap(d->map_size.p, cnt.p);
  std::swap(d->map_size.n, cnt.n);
  d->map_cap = cap;
  d->map_grow_s += secs(t0, std::chrono::high_resolution_clock::now());
  if (grow) d->map_grows += 1;
  return B2D_OK;
}

int status_code(const DevStatus& st) {
  switch (st.error) {
    case DERR_NONE: return B2D_OK;
    case DERR_MAP_FULL: return B2D_ERR_MAP_FULL;
    case DERR_WAIT_TIMEOUT: return B2D_ERR_TIMEOUT;
    case DERR_RESTART_RANGE: return B2D_ERR_RESTART_RANGE;
    default: return B2D_ERR_INTERNAL;
  }
}


LeafArgs leaf_args(const b2d_dedup* d, const RoundState* rs_dev) {
  const MapView m = map_at(d->map_mem, d->map_cap, d->map_size.p);
  return LeafArgs{static_cast<const uint8_t*>(d->data), d->data_len, d->chunk_size, d->n, d->kind, 0, 0,
                  d->tree.p, d->leaflab.p, d->dupflag.p, m, &d->state.p->status, rs_dev,
                  (uint32_t)d->tune.wait_polls, 1u};
}

// ------------------------------------------------------------------------------------------
// One checkpoint = prepare (host: sizes, allocations, map reset/growth, per-checkpoint values)
// + enqueue (device work, identical launch parameters for every checkpoint of a buffer, so it
// is captured once into a CUDA graph and replayed) + finish (host: status and sizes).
// ------------------------------------------------------------------------------------------
// The argument checks of one checkpoint; they change nothing, so a batch runs them for every
// handle before it prepares any.
int check_checkpoint(const b2d_dedup* d, const void* d_data, uint64_t len, bool make_baseline) {
  if (!d_data || len == 0) return B2D_ERR_ARG;
  const uint64_t nc = (len + d->chunk_size - 1) / d->chunk_size;
  if (nc > 0x7fffffffull) return B2D_ERR_ARG;
  const bool baseline = (d->current_id == 0) || make_baseline;
  if (!baseline && (!d->have_tree || nc != d->n)) return B2D_ERR_LEN_CHANGED;
  // source-checkpoint buckets, and the map's checkpoint field (MAP_TREE_PENDING is reserved)
  if (d->current_id + 1u > MAX_BUCKETS || d->current_id >= MAP_TREE_PENDING) return B2D_ERR_UNSUPPORTED;
  return B2D_OK;
}

int prepare_checkpoint(b2d_dedup* d, const void* d_data, uint64_t len, bool make_baseline) {
  const int vrc = check_checkpoint(d, d_data, len, make_baseline);
  if (vrc) return vrc;
  const uint64_t nc = (len + d->chunk_size - 1) / d->chunk_size;
  const bool baseline = (d->current_id == 0) || make_baseline;
  // a baseline replaces the tree and the map: until it completes the handle holds neither the
  // old checkpoint's state nor the new one's, and only another baseline may follow
  if (baseline) d->have_tree = false;
  d->diff_valid = false;
  d->data = d_data;
  d->data_len = len;
  d->n = (uint32_t)nc;
  d->N = 2u * d->n - 1u;
  d->D = node_level(d->N - 1u);
  // setup (:1594-1623): tree, labels, map, scratch
  B2D_CU(d->tree.reserve(d->N));
  B2D_CU(d->lab.reserve(d->N));
  B2D_CU(d->leaflab.reserve((uint64_t)d->n + 16u));
  if (d->dupflag.n < d->n || !d->dupflag.p) {
    // duplicate flags stay all-zero between checkpoints (phase 1 clears what it reads)
    B2D_CU(d->dupflag.reserve(d->n));
    B2D_CU(cudaMemsetAsync(d->dupflag.p, 0, d->dupflag.n, d->stream));
  }
  const uint64_t push_bytes = ((uint64_t)d->N + 63ull) / 64ull * 16ull + 16ull;   // 2 bits per node
  if (d->push.n < push_bytes || !d->push.p) {
    // flags stay all-zero between checkpoints (the compaction clears what it reads)
    B2D_CU(d->push.reserve(push_bytes));
    B2D_CU(cudaMemsetAsync(d->push.p, 0, d->push.n, d->stream));
  }
  if (baseline) {
    int rc = map_reset(d, map_capacity(2ull * d->N, d->map_max_load, d->map_headroom));
    if (rc) return rc;
    d->baseline_id = d->current_id;
    // the list approach starts a baseline from an all-zero digest list (src/list_approach.cpp:865-869)
    if (d->list) B2D_CU(cudaMemsetAsync(d->tree.p + (d->n - 1u), 0, sizeof(Digest) * (size_t)d->n, d->stream));
  } else {
    int rc = map_ensure(d);
    if (rc) return rc;
  }
  // bucket capacity grows in powers of two so a buffer's graph survives many checkpoints
  uint32_t bcap = d->bcap ? d->bcap : 64u;
  while (bcap < d->current_id + 1u) bcap <<= 1;
  if (bcap > MAX_BUCKETS) bcap = MAX_BUCKETS;
  d->bcap = bcap;
  B2D_CU(d->first_list.reserve(d->n));
  B2D_CU(d->shift_list.reserve(d->n));
  B2D_CU(d->tmp_first.reserve(d->n));
  B2D_CU(d->tmp_shift.reserve(d->n));
  B2D_CU(d->levels.reserve(68));
  B2D_CU(d->region_off.reserve(d->n));
  B2D_CU(d->sprev.reserve(d->n));
  B2D_CU(d->skey.reserve(d->n));
  B2D_CU(d->hist.reserve(bcap));
  B2D_CU(d->bucket_start.reserve(bcap));
  B2D_CU(d->partial.reserve((size_t)1184 * bcap));
  B2D_CU(d->partial2.reserve(2 * COMPACT_GRID));
  B2D_CU(d->diff.reserve(64 + 16ull * d->n + (uint64_t)d->n * d->chunk_size));
  B2D_CU(d->state.reserve(1));
  B2D_CU(d->state_h.reserve(1));
  B2D_CU(d->round_h.reserve(1));
  RoundState* r = d->round_h.p;
  r->cur = d->current_id;
  r->baseline_id = d->baseline_id;
  // the list approach applies one per-chunk rule to every checkpoint (src/list_approach.cpp:41-71):
  // the incremental leaf rule against a list that a baseline has zeroed
  r->baseline = (baseline && !d->list) ? 1u : 0u;
  r->buckets = d->current_id + 1u;
  map_view(d, r->map);
  return B2D_OK;
}

// everything a checkpoint's launches depend on; a different key means a different graph (the
// digest map is not in it: kernels read its location from the RoundState)
void graph_key(const b2d_dedup* d, const RoundState* rs_dev, std::vector<uint64_t>& k) {
  k.assign({(uint64_t)d->data, d->data_len, d->chunk_size, (uint64_t)d->kind, (uint64_t)d->tree.p,
            (uint64_t)d->lab.p, (uint64_t)d->leaflab.p, (uint64_t)d->push.p, (uint64_t)d->dupflag.p,
            (uint64_t)d->first_list.p,
            (uint64_t)d->shift_list.p, (uint64_t)d->tmp_first.p, (uint64_t)d->tmp_shift.p, (uint64_t)d->levels.p,
            (uint64_t)d->region_off.p, (uint64_t)d->sprev.p, (uint64_t)d->skey.p, (uint64_t)d->hist.p,
            (uint64_t)d->bucket_start.p, (uint64_t)d->partial.p, (uint64_t)d->partial2.p, (uint64_t)d->diff.p,
            (uint64_t)d->state.p, (uint64_t)d->state_h.p, (uint64_t)d->round_h.p, (uint64_t)rs_dev, d->bcap,
            (uint64_t)d->tune.allow_tma, (uint64_t)d->tune.stages, (uint64_t)d->tune.ctas_per_sm, (uint64_t)d->graph_timing,
            (uint64_t)d->tune.unit, (uint64_t)d->tune.wait_polls,
            (uint64_t)d->sm_count, (uint64_t)d->list, (uint64_t)d->warp_bands});
}

// Device work of one checkpoint on `s`.  `rs_dev` is where the kernels read this checkpoint's
// RoundState; with `upload` the host copy (pinned) is copied there first.  `managed`: a batch
// clears the DevState, writes the RoundState and reads the DevState back for all its handles
// at once (and may have hashed the leaves already: `skip_leaves`).
DiffArgs diff_args(b2d_dedup* d, const RoundState* rs_dev) {
  MapView m;
  map_view(d, m);
  DevState* ds = d->state.p;
  return DiffArgs{static_cast<const uint8_t*>(d->data), d->data_len, d->chunk_size, d->n, d->N, d->D, 0, 0,
                  d->tree.p, d->push.p, m, &ds->status, &ds->meta, d->first_list.p, d->shift_list.p, d->tmp_first.p,
                  d->tmp_shift.p, d->levels.p, d->region_off.p, d->sprev.p, d->skey.p, d->hist.p, d->bucket_start.p,
                  d->partial.p, d->partial2.p, d->diff.p, rs_dev, 0u};
}

ForestArgs forest_args(b2d_dedup* d, const RoundState* rs_dev) {
  MapView m;
  map_view(d, m);
  DevState* ds = d->state.p;
  return ForestArgs{d->tree.p, d->lab.p, d->leaflab.p, d->push.p, m, &ds->status, &ds->zero_exists, d->dupflag.p,
                    d->n, d->N, d->D, 0, d->kind, 0, rs_dev};
}

int enqueue_checkpoint(b2d_dedup* d, cudaStream_t s, RoundState* rs_dev, bool upload, bool timing, bool skip_leaves,
                       bool managed = false, bool skip_diff = false, bool skip_forest = false) {
  DevState* ds = d->state.p;
  bool zero_probe_skipped = false;
  if (!managed) {
    B2D_CU(cudaMemsetAsync(ds, 0, sizeof(DevState), s));
    if (upload) B2D_CU(cudaMemcpyAsync(rs_dev, d->round_h.p, sizeof(RoundState), cudaMemcpyHostToDevice, s));
  }
  if (timing) B2D_CU(record_timing(d->ev[0], s));
  // dedup_data_baseline (:13-259) / dedup_data (:261-509)
  if (!skip_leaves) {
    const LeafArgs la = leaf_args(d, rs_dev);
    const int leaf_path = launch_leaves(la, d->sm_count, d->tune, s);
    if (leaf_path < 0) return B2D_ERR_CUDA;
    d->leaf_tma = leaf_path == 1;
  }
  if (timing) B2D_CU(record_timing(d->ev[3], s));
  if (d->list) {
    // list approach: no tree; per-chunk labels and region flags (src/list_approach.cpp:41-71)
    B2D_CU(launch_list_label(forest_args(d, rs_dev), d->sm_count, s));
  } else if (!skip_forest) {
    const ForestArgs fa = forest_args(d, rs_dev);
    B2D_CU(launch_forest(fa, 1, s, d->sm_count, d->warp_bands));
    // the zero-digest probe matters to baselines only; launches issued one by one for a single
    // handle skip it otherwise (a captured graph or a batch keeps it: it serves both kinds)
    if (managed || d->use_graph || d->round_h.p->baseline) B2D_CU(launch_zero_exists(&ds->zero_exists, rs_dev, s));
    else zero_probe_skipped = true;
    B2D_CU(launch_forest(fa, 2, s, d->sm_count, d->warp_bands));
  }
  if (timing) B2D_CU(record_timing(d->ev[1], s));
  // collect_diff (:511-710; list approach src/list_approach.cpp:79-257, single-chunk regions in
  // chunk order, chunk indices in the diff); a batch may assemble all its handles' diffs in
  // shared launches
  if (!skip_diff) {
    DiffArgs da = diff_args(d, rs_dev);
    if (d->list) da.id_bias = d->n - 1u;
    B2D_CU(launch_collect_diff(da, d->bcap, d->sm_count, s, d->list != 0));
  }
  if (timing) B2D_CU(record_timing(d->ev[2], s));
  if (!managed) B2D_CU(cudaMemcpyAsync(d->state_h.p, d->state.p, sizeof(DevState), cudaMemcpyDeviceToHost, s));
  // kernels only (memsets and copies are not counted): the diff assembly is 12 kernels, 10 in
  // node order (no level reordering)
  if (d->list)
    d->launches = (skip_leaves ? 0 : 1) + 1 + (skip_diff ? 0 : 10);
  else
    d->launches = (skip_leaves ? 0 : 1) +
                  (skip_forest ? 0 : forest_launch_count(d->n, d->D, 1, d->warp_bands) +
                                         forest_launch_count(d->n, d->D, 2, d->warp_bands) +
                                         (zero_probe_skipped ? 0 : 1)) +
                  (skip_diff ? 0 : 12);
  return B2D_OK;
}

int finish_checkpoint(b2d_dedup* d, bool advance, bool timing) {
  const DevState& st = *d->state_h.p;
  if (timing) {
    const float ms_dedup = elapsed_ms(d->ev[0], d->ev[1]);
    const float ms_gather = elapsed_ms(d->ev[1], d->ev[2]);
    const float ms_leaf = elapsed_ms(d->ev[0], d->ev[3]);
    d->phase[0] = ms_leaf * 1e-3;
    d->phase[1] = (ms_dedup - ms_leaf) * 1e-3;
    d->phase[2] = ms_gather * 1e-3;
    d->timers[1] = ms_dedup * 1e-3;
    d->timers[2] = ms_gather * 1e-3;
  }
  d->timers[3] = 0;
  int rc = status_code(st.status);
  d->map_size_host = st.meta.map_size;
  if (rc) {
    // the tree and the map may be part-way updated: the next checkpoint must be a baseline
    d->have_tree = false;
    // a failed checkpoint may leave region flags behind; they must be zero for the next one
    cudaMemsetAsync(d->push.p, 0, d->push.n, d->stream);
    cudaMemsetAsync(d->dupflag.p, 0, d->dupflag.n, d->stream);
    cudaStreamSynchronize(d->stream);
    return rc;
  }
  d->F = st.meta.F;
  d->S = st.meta.S;
  d->diff_len = st.meta.diff_len;
  d->diff_delta = st.meta.delta;
  const uint64_t meta_bytes = 4ull * st.meta.F + 8ull * st.meta.P + 8ull * st.meta.S;
  d->datasizes[0] = d->diff_len - meta_bytes;
  d->datasizes[1] = meta_bytes;
  d->diff_valid = true;
  d->have_tree = true;
  if (advance) d->current_id += 1;
  return B2D_OK;
}

int do_checkpoint(b2d_dedup* d, const void* d_data, uint64_t len, bool make_baseline, bool advance) {
  using clk = std::chrono::high_resolution_clock;
  const auto t0 = clk::now();
  int rc = prepare_checkpoint(d, d_data, len, make_baseline);
  if (rc) return rc;
  RoundState* rs_dev = &d->state.p->round;
  if (!d->use_graph) {
    d->timers[0] = secs(t0, clk::now());
    rc = enqueue_checkpoint(d, d->stream, rs_dev, true, true, false);
    if (rc) return rc;
    B2D_CU(cudaStreamSynchronize(d->stream));
    return finish_checkpoint(d, advance, true);
  }
  // the round state lives in DevState, which the enqueue clears first: upload after the clear
  std::vector<uint64_t> key;
  graph_key(d, rs_dev, key);
  if (!d->graph_exec || key != d->graph_key) {
    if (d->graph_exec) {
      cudaGraphExecDestroy(d->graph_exec);
      d->graph_exec = nullptr;
    }
    // captured on a private stream (the caller's may be the legacy default stream, which
    // cannot be captured) and launched on the caller's
    cudaGraph_t g = nullptr;
    B2D_CU(cudaStreamBeginCapture(d->cap_stream, cudaStreamCaptureModeThreadLocal));
    rc = enqueue_checkpoint(d, d->cap_stream, rs_dev, true, d->graph_timing, false);
    const cudaError_t ce = cudaStreamEndCapture(d->cap_stream, &g);
    if (rc) {
      if (g) cudaGraphDestroy(g);
      return rc;
    }
    B2D_CU(ce);
    const cudaError_t ie = cudaGraphInstantiate(&d->graph_exec, g, 0);
    cudaGraphDestroy(g);
    B2D_CU(ie);
    d->graph_key = key;
  }
  d->timers[0] = secs(t0, clk::now());
  B2D_CU(cudaGraphLaunch(d->graph_exec, d->stream));
  B2D_CU(cudaStreamSynchronize(d->stream));
  return finish_checkpoint(d, advance, d->graph_timing);
}

int copy_diff(b2d_dedup* d, void* dst, uint64_t cap) {
  if (!d->diff_valid) return B2D_ERR_ARG;
  if (cap < d->diff_len) return B2D_ERR_ARG;
  const auto t0 = std::chrono::high_resolution_clock::now();
  B2D_CU(cudaMemcpyAsync(dst, d->diff.p + d->diff_delta, d->diff_len, cudaMemcpyDeviceToHost, d->stream));
  B2D_CU(cudaStreamSynchronize(d->stream));
  d->timers[3] = secs(t0, std::chrono::high_resolution_clock::now());
  return B2D_OK;
}

int checkpoint_to_pinned(b2d_dedup* d, const void* d_data, uint64_t len, bool make_baseline, bool advance,
                         const uint8_t** diff, uint64_t* diff_len) {
  int rc = do_checkpoint(d, d_data, len, make_baseline, advance);
  if (rc) return rc;
  B2D_CU(d->diff_h.grow(d->diff_len));
  rc = copy_diff(d, d->diff_h.p, d->diff_h.n);
  if (rc) return rc;
  if (diff) *diff = d->diff_h.p;
  if (diff_len) *diff_len = d->diff_len;
  return B2D_OK;
}

// write_chkpt_log (:1853-1896) with write_metadata_breakdown (src/utils.cpp:38-124); the
// checkpoint id written is the one just taken (logs are written before current_id += 1)
// `diff` holds at least the 32-byte header; `ctab` the repeat table ((ckpt, count) rows)
int write_chkpt_log(b2d_dedup* d, const uint8_t* diff, const uint8_t* ctab, const std::string& logname, uint32_t id) {
  const std::string base = logname + ".chunk_size." + std::to_string(d->chunk_size);
  FILE* result = fopen((base + ".csv").c_str(), "a");
  FILE* size = fopen((base + ".size.csv").c_str(), "a");
  FILE* timing = fopen((base + ".timing.csv").c_str(), "a");
  if (!result || !size || !timing) {
    if (result) fclose(result);
    if (size) fclose(size);
    if (timing) fclose(timing);
    return B2D_ERR_IO;
  }
  if (ftell(result) == 0)
    fprintf(result,
            "Approach,Chkpt ID,Chunk Size,Uncompressed Size,Compressed Size,Data Size,Metadata Size,Setup Time,"
            "Comparison Time,Gather Time,Write Time\n");
  auto g = [](double v) {
    char b[64];
    snprintf(b, sizeof b, "%g", v);
    return std::string(b);
  };
  const char* approach = d->list ? "List" : "Tree";
  fprintf(result, "%s,%u,%u,%llu,%llu,%llu,%llu,%s,%s,%s,%s\n", approach, id, d->chunk_size,
          (unsigned long long)d->data_len, (unsigned long long)(d->datasizes[0] + d->datasizes[1]),
          (unsigned long long)d->datasizes[0], (unsigned long long)d->datasizes[1], g(d->timers[0]).c_str(),
          g(d->timers[1]).c_str(), g(d->timers[2]).c_str(), g(d->timers[3]).c_str());
  fprintf(timing, "%s,%u,%u,%s,%s,%s\n", approach, id, d->chunk_size, g(d->timers[1]).c_str(), g(d->timers[2]).c_str(),
          g(d->timers[3]).c_str());
  fprintf(size, "%s,%u,%u,%llu,%llu,", approach, id, d->chunk_size, (unsigned long long)d->datasizes[0],
          (unsigned long long)d->datasizes[1]);
  // write_metadata_breakdown (src/utils.cpp:38-124)
  uint32_t h[8];
  memcpy(h, diff, 32);
  uint64_t datalen;
  memcpy(&datalen, diff + 8, 8);
  const uint32_t ref_id = h[0], chkpt_id = h[1], cs = h[4], nf = h[5], np = h[6], ns = h[7];
  fprintf(size, "%zu,%llu,", (size_t)32, (unsigned long long)nf * 4ull);
  if (ref_id != chkpt_id) {
    fprintf(size, "%llu", 8ull * np);
    for (uint32_t i = 0; i < id; i++) {
      if (i < np) {
        uint32_t num = 0;
        memcpy(&num, ctab + 8ull * i + 4, 4);
        fprintf(size, ",%llu", 8ull * num);
      } else {
        fprintf(size, ",0");
      }
    }
    fprintf(size, "\n");
  } else {
    fprintf(size, "0,%llu", 8ull * ns);
    for (uint32_t i = 1; i < id; i++) fprintf(size, ",0");
    fprintf(size, "\n");
  }
  (void)cs;
  (void)datalen;
  fclose(result);
  fclose(size);
  fclose(timing);
  return B2D_OK;
}

// write_restart_log (:1904-1915)
int write_restart_log(b2d_dedup* d, uint32_t id, const std::string& logname) {
  FILE* f = fopen(logname.c_str(), "a");
  if (!f) return B2D_OK;   // the reference ignores an unopenable restart log ("/dev/null/")
  fprintf(f, "%s,%u,%u,%g,%g\n", d->list ? "List" : "Tree", id, d->chunk_size, d->restart_timers[0],
          d->restart_timers[1]);
  fclose(f);
  return B2D_OK;
}

struct HostHdr {
  uint32_t ref_id, chkpt_id;
  uint64_t datalen;
  uint32_t cs, F, P, S;
  uint64_t first_off, count_off, shift_off, data_off;
};

bool parse_hdr(const uint8_t* b, uint64_t size, HostHdr& h) {
  if (!b || size < 32) return false;
  memcpy(&h.ref_id, b, 4);
  memcpy(&h.chkpt_id, b + 4, 4);
  memcpy(&h.datalen, b + 8, 8);
  memcpy(&h.cs, b + 16, 4);
  memcpy(&h.F, b + 20, 4);
  memcpy(&h.P, b + 24, 4);
  memcpy(&h.S, b + 28, 4);
  h.first_off = 32;
  h.count_off = h.first_off + 4ull * h.F;
  h.shift_off = h.count_off + 8ull * h.P;
  h.data_off = h.shift_off + 8ull * h.S;
  return h.data_off <= size && h.cs > 0 && h.datalen > 0;
}

int do_restart(b2d_dedup* d, void* d_out, uint64_t len, const uint8_t* const* diffs, const uint64_t* sizes,
               uint32_t count, uint32_t id, const void* const* ddiffs = nullptr) {
  using clk = std::chrono::high_resolution_clock;
  const auto t0 = clk::now();
  if (!d_out || (!diffs && !ddiffs) || !sizes || id >= count) return B2D_ERR_ARG;
  // device-resident diffs: the host reads only their headers and repeat tables (small copies)
  std::vector<std::vector<uint8_t>> hmeta;
  std::vector<const uint8_t*> hptr;
  if (ddiffs) {
    hmeta.resize(count);
    hptr.assign(count, nullptr);
    // the same chain walk as below: from `id` down while the index is not below the last ref_id
    for (int idx = (int)id; idx >= 0; idx--) {
      if (!ddiffs[idx] || sizes[idx] < 32) return B2D_ERR_FORMAT;
      uint8_t hdr[32];
      B2D_CU(cudaMemcpy(hdr, ddiffs[idx], 32, cudaMemcpyDeviceToHost));
      HostHdr hh;
      if (!parse_hdr(hdr, sizes[idx], hh)) return B2D_ERR_FORMAT;
      // header, then the repeat table right behind it (not at its offset in the diff: the
      // first-occurrence list in between can be tens of megabytes)
      auto& m = hmeta[idx];
      m.resize(32 + 8ull * hh.P);
      std::memcpy(m.data(), hdr, 32);
      if (hh.P) B2D_CU(cudaMemcpy(m.data() + 32, static_cast<const uint8_t*>(ddiffs[idx]) + hh.count_off,
                                  8ull * hh.P, cudaMemcpyDeviceToHost));
      hptr[idx] = m.data();
      if (idx - 1 < (int)hh.ref_id) break;
    }
    diffs = hptr.data();
  }
  HostHdr h;
  if (!parse_hdr(diffs[id], sizes[id], h)) return B2D_ERR_FORMAT;
  // every diff the checkpoint path writes has ref_id <= chkpt_id == its position in the list;
  // a list that breaks this names no chain to walk, so it is rejected before any device work
  if (h.ref_id > h.chkpt_id || h.chkpt_id != id) return B2D_ERR_FORMAT;
  if (len < h.datalen) return B2D_ERR_ARG;
  uint64_t nc = (h.datalen + h.cs - 1) / h.cs;
  if (nc > 0x7fffffffull) return B2D_ERR_FORMAT;
  const uint32_t n = (uint32_t)nc, N = 2u * n - 1u;
  // the chain, newest first: from `id` down while the index is not below the last ref_id
  std::vector<int> chain;
  std::vector<HostHdr> hdrs;
  uint64_t max_size = 0, max_list = 0, max_ids = 0;
  {
    uint32_t ref = h.ref_id;
    for (int idx = (int)id; idx >= 0 && idx >= (int)ref; idx--) {
      HostHdr hh;
      if (!parse_hdr(diffs[idx], sizes[idx], hh)) return B2D_ERR_FORMAT;
      if (idx != (int)id) ref = hh.ref_id;
      chain.push_back(idx);
      hdrs.push_back(hh);
      max_size = std::max<uint64_t>(max_size, sizes[idx]);
      max_list = std::max<uint64_t>(max_list, std::max<uint64_t>(hh.F, hh.S));
      max_ids = std::max<uint64_t>(max_ids, (uint64_t)hh.chkpt_id + 1);
    }
  }
  // window slots: older diffs resolved per walk.  Device diffs are read where they lie, so a
  // window holds several (bounded by the slots' memory); host diffs pass one at a time through
  // one device copy.
  const uint64_t older = chain.size() - 1;
  uint32_t W = 1;
  if (ddiffs && older > 1) {
    const uint64_t per_slot = 13ull * n;   // dist u32 + rep uint2 + a flag byte per chunk
    W = (uint32_t)std::min<uint64_t>(std::min<uint64_t>(older, RESTART_WINDOW),
                                     std::max<uint64_t>(1, RESTART_SLOT_BYTES / per_slot));
  }
  B2D_CU(d->r_node_list.reserve(n));
  B2D_CU(d->r_mflag.reserve(n));
  B2D_CU(d->r_dist.reserve((uint64_t)n * W));
  B2D_CU(d->r_rep.reserve((uint64_t)n * W));
  B2D_CU(d->r_flag.reserve((uint64_t)n * W));
  B2D_CU(d->r_offs.reserve(4 * std::max<uint64_t>(max_list, 1)));
  B2D_CU(d->r_partial.reserve(SCAN_GRID));
  B2D_CU(d->r_cum.reserve(max_ids));
  B2D_CU(d->r_total.reserve(1));
  if (!ddiffs) B2D_CU(d->r_diff.reserve(max_size + 16));   // device diffs are read where they lie
  B2D_CU(d->state.reserve(1));
  B2D_CU(d->state_h.reserve(1));
  if (!ddiffs) B2D_CU(d->r_stage.grow(max_size + 16 + 8 * max_ids));
  B2D_CU(cudaMemsetAsync(d->state.p, 0, sizeof(DevState), d->stream));
  d->launches = 0;
  double copy_time = 0;
  auto slot = [&](uint32_t k) {
    RestartSlot sl;
    sl.dist = d->r_dist.p + (uint64_t)n * k;
    sl.rep = d->r_rep.p + (uint64_t)n * k;
    sl.flag = d->r_flag.p + (uint64_t)n * k;
    return sl;
  };

  RestartArgs a{};
  a.n = n;
  a.N = N;
  a.out = static_cast<uint8_t*>(d_out);
  a.out_len = h.datalen;
  a.node_list = d->r_node_list.p;
  a.mflag = d->r_mflag.p;
  const uint64_t lcap = std::max<uint64_t>(max_list, 1);
  a.offs = d->r_offs.p;
  a.rstart = d->r_offs.p + lcap;
  a.pstart = d->r_offs.p + 2 * lcap;
  a.rtree = d->r_offs.p + 3 * lcap;
  a.partial = d->r_partial.p;
  a.total = d->r_total.p;
  a.st = &d->state.p->status;
  // list diffs name chunks; the restart kernels work on leaf heap indices (leaf of chunk c = n-1+c)
  a.id_bias = d->list ? n - 1u : 0u;
  RestartWalk w{};
  w.main_cur = h.chkpt_id;
  w.n = n;
  w.N = N;
  w.out = a.out;
  w.out_len = h.datalen;
  w.node_list = a.node_list;
  w.mflag = a.mflag;
  w.st = a.st;
  uint32_t wcount = 0;
  auto flush = [&](bool last) -> cudaError_t {
    if (wcount == 0) return cudaSuccess;
    w.count = wcount;
    w.last = last;
    cudaError_t e = launch_restart_walk(w, d->sm_count, d->stream);
    d->launches += 1;
    w.dense = 1;   // a walk that is not the last wrote every chunk's NodeID
    wcount = 0;
    return e;
  };

  for (size_t k = 0; k < chain.size(); k++) {
    const int idx = chain[k];
    const HostHdr& hh = hdrs[k];
    const bool is_main = k == 0;
    // host diffs: one copy into the device scratch, placed so the data section is 16-byte
    // aligned; pinned (page-locked) host diffs are copied straight from where they are, others
    // go through the handle's pinned staging buffer.  The repeat table's running counts are
    // uploaded beside them.
    const uint32_t delta = (uint32_t)((16u - (hh.data_off & 15u)) & 15u);
    const uint64_t ncum = (uint64_t)hh.chkpt_id + 1;
    bool pinned = ddiffs != nullptr;
    if (!ddiffs) {
      cudaPointerAttributes pa;
      pinned = cudaPointerGetAttributes(&pa, diffs[idx]) == cudaSuccess && pa.type == cudaMemoryTypeHost;
      if (!pinned) (void)cudaGetLastError();
    }
    if (!pinned) B2D_CU(cudaStreamSynchronize(d->stream));
    const auto c0 = clk::now();
    const uint8_t* src = ddiffs ? static_cast<const uint8_t*>(ddiffs[idx]) : diffs[idx];
    if (!pinned) {
      memcpy(d->r_stage.p + delta, diffs[idx], sizes[idx]);
      src = d->r_stage.p + delta;
    }
    std::vector<unsigned long long> cum(ncum, 0ull);
    bool bad_row = false;
    const uint8_t* ctab = ddiffs ? diffs[idx] + 32 : diffs[idx] + hh.count_off;   // repeat table on the host
    for (uint32_t i = 0; i < hh.P; i++) {
      uint32_t ck, cnt;
      memcpy(&ck, ctab + 8ull * i, 4);
      memcpy(&cnt, ctab + 8ull * i + 4, 4);
      if (ck < ncum) cum[ck] = cnt; else bad_row = true;
    }
    for (uint64_t t = 1; t < ncum; t++) cum[t] += cum[t - 1];
    if (!ddiffs)
      B2D_CU(cudaMemcpyAsync(d->r_diff.p + delta, src, sizes[idx], cudaMemcpyHostToDevice, d->stream));
    B2D_CU(cudaMemcpyAsync(d->r_cum.p, cum.data(), sizeof(unsigned long long) * ncum, cudaMemcpyHostToDevice,
                           d->stream));
    if (is_main && !ddiffs) {
      B2D_CU(cudaStreamSynchronize(d->stream));
      copy_time = secs(c0, clk::now());
    }
    a.diff = ddiffs ? src : d->r_diff.p + delta;
    a.diff_size = sizes[idx];
    a.first_off = hh.first_off;
    a.count_off = hh.count_off;
    a.shift_off = hh.shift_off;
    a.data_off = hh.data_off;
    a.F = hh.F;
    a.P = hh.P;
    a.S = hh.S;
    a.cur_id = hh.chkpt_id;
    a.datalen = hh.datalen;
    a.cs = hh.cs;
    a.is_main = is_main;
    a.cum = d->r_cum.p;
    a.ncum = (uint32_t)ncum;
    a.slot = slot(is_main ? 0 : wcount);
    B2D_CU(launch_restart_diff(a, &d->state.p->straddle, d->sm_count, d->stream));
    d->launches += restart_diff_launches(n, d->list != 0);
    if (!is_main) {
      // the window's walk copies from every diff in it, which share one chunk size
      if (wcount == 0) w.cs = hh.cs;
      w.data[wcount] = a.diff + hh.data_off;
      w.data_len[wcount] = sizes[idx] - hh.data_off;
      w.datalen[wcount] = hh.datalen;
      w.cur[wcount] = hh.chkpt_id;
      w.slot[wcount] = a.slot;
      wcount++;
      const bool end = k + 1 == chain.size();
      if (bad_row || end || wcount == W || hdrs[k + 1].cs != hh.cs) B2D_CU(flush(bad_row || end));
    }
    if (bad_row) {
      B2D_CU(cudaStreamSynchronize(d->stream));
      d->restart_timers[0] = copy_time;
      d->restart_timers[1] = secs(t0, clk::now());
      return B2D_ERR_RESTART_RANGE;
    }
  }
  B2D_CU(cudaMemcpyAsync(d->state_h.p, d->state.p, sizeof(DevState), cudaMemcpyDeviceToHost, d->stream));
  B2D_CU(cudaStreamSynchronize(d->stream));
  d->restart_timers[0] = copy_time;
  d->restart_timers[1] = secs(t0, clk::now());
  return status_code(d->state_h.p->status);
}

int read_file(const std::string& path, std::vector<uint8_t>& out) {
  FILE* f = fopen(path.c_str(), "rb");
  if (!f) return B2D_ERR_IO;
  if (fseek(f, 0, SEEK_END) != 0) { fclose(f); return B2D_ERR_IO; }
  long sz = ftell(f);
  if (sz < 0) { fclose(f); return B2D_ERR_IO; }
  fseek(f, 0, SEEK_SET);
  out.resize((size_t)sz);
  size_t got = sz ? fread(out.data(), 1, (size_t)sz, f) : 0;
  fclose(f);
  return got == (size_t)sz ? B2D_OK : B2D_ERR_IO;
}

// ------------------------------------------------------------------------------------------
// Batched checkpoints: one checkpoint of each of many handles (buffers of any sizes, each
// with its own device-resident tree and map) as ONE CUDA graph:
//   upload (one copy: leaf work items, round states, state pointers)
//   -> batch_init_kernel (clears every handle's DevState, writes its RoundState)
//   -> one persistent leaf kernel per (unit, hash kind) group, fed by a tile work queue
//   -> per handle: forest + diff assembly, spread over parallel graph branches
//   -> batch_collect_kernel + one read-back of every handle's DevState.
// Each handle's output is what its own b2d_checkpoint_device would produce.
// ------------------------------------------------------------------------------------------
static_assert(sizeof(DevState) % 4 == 0, "DevState is cleared word by word");

__global__ void batch_init_kernel(DevState* const* states, const RoundState* rounds, uint32_t count,
                                  unsigned int* queues, uint32_t ngroups, DevStatus* bst) {
  const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
  for (uint32_t i = tid; i < count; i += gridDim.x * blockDim.x) {
    uint32_t* w = reinterpret_cast<uint32_t*>(states[i]);
    for (uint32_t j = 0; j < sizeof(DevState) / 4; j++) w[j] = 0u;
    states[i]->round = rounds[i];
  }
  if (tid < ngroups) queues[tid] = 0u;
  if (tid == 0) {
    bst->error = 0u;
    bst->detail = 0u;
  }
}

__global__ void batch_collect_kernel(DevState* const* states, uint32_t count, DevState* out) {
  const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
  for (uint32_t i = tid; i < count; i += gridDim.x * blockDim.x) out[i] = *states[i];
}

struct BatchCand {
  int stages, ctas, tiles_per_pop, streams, shared;
  int warp;       // forest phases starting with a warp band (B2D_WARP_BANDS mask): fused levels
  int headroom;   // digest-map size over its minimum, percent: the load factor
};

// Online coordinate-descent tuner.  Each incremental batch (same bytes every time) measures one
// setting by its graph's device time: first the current setting, then, one knob at a time,
// each other value of that knob, keeping a value when it is at least 1 % faster (batches
// differ in content, so smaller gains are not trusted).  Knobs:
//   shared      segmented forest/diff launches for all handles, or per-handle launches on 32
//               graph branches;
//   tiles/pop   chunk ranges (tiles of 256 chunks) a hashing CTA takes per work-queue pop: 4, 1, 16;
//   staging     ring depth x CTAs per SM of the hashing kernel;
//   fused       levels fused in the first forest band: warp bands (7 + 9) or CTA bands (10 + 12);
//   load        digest-map headroom 1.5 or 1.25 (load 0.25 or 0.3 after a baseline; both leave
//               room for dozens of checkpoints before a growth); a change resizes every
//               handle's table before the next batch (outside the timed graph).
// 1 + 1 + 2 + 1 + 1 + 1 = 7 measured batches.
struct BatchTuner {
  static constexpr int KNOBS = 5;
  BatchCand base{0, 3, 4, 32, 1, B2D_WARP_BANDS, 150};
  double base_score = 0;
  bool have_base = false, done = false;
  int knob = 0;
  size_t idx = 0;
  BatchCand pending = base;

  static size_t nvalues(int k) { return k == 1 ? 3 : 2; }
  static BatchCand with_value(BatchCand c, int k, size_t i) {
    static const int tpp[3] = {4, 1, 16};
    static const int stages[2] = {0, 3}, ctas[2] = {3, 2};
    static const int warp[2] = {B2D_WARP_BANDS, 0}, headroom[2] = {150, 125};
    if (k == 0) c.shared = i == 0 ? 1 : 0;
    else if (k == 1) c.tiles_per_pop = tpp[i];
    else if (k == 2) {
      c.stages = stages[i];
      c.ctas = ctas[i];
    } else if (k == 3) c.warp = warp[i];
    else c.headroom = headroom[i];
    return c;
  }
  static bool same(const BatchCand& a, const BatchCand& b) {
    return a.stages == b.stages && a.ctas == b.ctas && a.tiles_per_pop == b.tiles_per_pop &&
           a.streams == b.streams && a.shared == b.shared && a.warp == b.warp && a.headroom == b.headroom;
  }
  void reset(const BatchCand& start) {
    *this = BatchTuner();
    base = pending = start;
  }
  BatchCand next() {
    if (!have_base || done) return pending = base;
    while (knob < KNOBS) {
      while (idx < nvalues(knob)) {
        const BatchCand c = with_value(base, knob, idx);
        if (!same(c, base)) return pending = c;
        idx++;
      }
      knob++;
      idx = 0;
    }
    done = true;
    return pending = base;
  }
  void report(double score) {
    if (done) return;
    if (!have_base) {
      have_base = true;
      base_score = score;
      return;
    }
    if (score > 1.01 * base_score) {
      base = pending;
      base_score = score;
    }
    idx++;
    next();   // settles `done` once the last knob is exhausted
  }
};

struct BatchLayout {
  size_t items = 0, rounds = 0, states = 0, queues = 0, bstatus = 0, dargs = 0, dtab = 0, fargs = 0, ftab = 0,
         total = 0;
};
// u32 tables of the shared diff assembly, each n (+1) long, in this order in the blob
enum DiffTable { DT_G, DT_GS, DT_BCAP, DT_ONE, DT_BEG_G, DT_BEG_GL, DT_BEG_GP, DT_BEG_GS, DT_BEG_GATHER, DT_COUNT };
constexpr int DIFF_TABLES = DT_BEG_GATHER + GATHER_VARIANTS;

}  // namespace

struct b2d_batch {
  int device = 0;
  int sm_count = 148;
  cudaStream_t own_stream = nullptr, stream = nullptr, cap = nullptr;
  std::vector<cudaStream_t> side;
  std::vector<cudaEvent_t> side_ev;
  cudaEvent_t fork_ev = nullptr;
  cudaEvent_t ev[2] = {nullptr, nullptr};
  DevBuf<uint8_t> blob;
  PinnedBuf<uint8_t> blob_h;
  DevBuf<DevState> coll;
  PinnedBuf<DevState> coll_h;
  BatchLayout lay;
  // instantiated graphs by batch composition, least recently used evicted beyond graph_cap
  struct GraphEntry {
    std::vector<uint64_t> key;
    uint64_t hash = 0;
    cudaGraphExec_t exec = nullptr;
    uint32_t launches = 0;
    uint64_t last_use = 0;
  };
  std::vector<GraphEntry> graphs;
  size_t graph_cap = 16;
  int graph_mode = 2;                // 0 direct launches, 1 always a graph, 2 graph from the 2nd sighting
  bool batch_diff = true;            // all handles' diff assembly in shared segmented launches
  bool batch_forest = true;          // and their forest phases (needs batch_diff)
  std::vector<uint64_t> seen;        // compositions launched directly once
  uint64_t use_clock = 0;
  // the batch in flight (launched, not yet finished)
  bool inflight = false;
  std::vector<b2d_dedup*> fl_handles;
  uint64_t fl_bytes = 0;
  bool fl_scoring = false, fl_any_baseline = false;
  std::chrono::high_resolution_clock::time_point fl_t0;
  // tuning: current values, and the online tuner
  BatchCand cur{0, 3, 4, 32, 1, B2D_WARP_BANDS, 150};
  bool autotune = false;
  BatchTuner tuner;
  // last batch
  double dev_s = 0, host_s = 0;
  uint32_t launches = 0;
  uint32_t leaf_groups = 0;

  ~b2d_batch() {
    for (auto& g : graphs)
      if (g.exec) cudaGraphExecDestroy(g.exec);
    for (auto e : side_ev)
      if (e) cudaEventDestroy(e);
    for (auto s : side)
      if (s) cudaStreamDestroy(s);
    if (fork_ev) cudaEventDestroy(fork_ev);
    for (auto e : ev)
      if (e) cudaEventDestroy(e);
    if (own_stream) cudaStreamDestroy(own_stream);
    if (cap) cudaStreamDestroy(cap);
  }
};

namespace {

int ensure_side_streams(b2d_batch* b, int n) {
  while ((int)b->side.size() < n) {
    cudaStream_t s = nullptr;
    cudaEvent_t e = nullptr;
    B2D_CU(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    b->side.push_back(s);
    B2D_CU(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    b->side_ev.push_back(e);
  }
  return B2D_OK;
}

size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

uint64_t key_hash(const std::vector<uint64_t>& k) {
  uint64_t h = 0x9E3779B97F4A7C15ull ^ k.size();
  for (uint64_t v : k) {
    h ^= v + 0x9E3779B97F4A7C15ull + (h << 6) + (h >> 2);
  }
  return h;
}

// Host preparation, graph lookup or capture, and launch of one batch; the device work is left
// running and batch_finish collects it.
int batch_launch(b2d_batch* b, b2d_dedup* const* hs, const void* const* data, const uint64_t* lens,
                 const int* make_baseline, uint32_t count, int* rcs) {
  using clk = std::chrono::high_resolution_clock;
  const auto t0 = clk::now();
  if (b->inflight) return B2D_ERR_ARG;   // one batch in flight per batch object
  if (count == 0) return B2D_OK;
  for (uint32_t i = 0; i < count; i++) {
    if (!hs[i]) return B2D_ERR_ARG;
    for (uint32_t j = 0; j < i; j++)
      if (hs[j] == hs[i]) return B2D_ERR_ARG;   // one checkpoint per handle per batch
  }
  // every handle's arguments before any handle is prepared: a rejected batch changes no handle
  for (uint32_t i = 0; i < count; i++) {
    const int vrc = check_checkpoint(hs[i], data[i], lens[i], make_baseline && make_baseline[i]);
    if (vrc) {
      if (rcs) rcs[i] = vrc;
      return vrc;
    }
  }
  // tuning for this batch
  const bool scoring = b->autotune && !b->tuner.done;
  const BatchCand cand = scoring ? b->tuner.next() : b->cur;
  int rc = ensure_side_streams(b, cand.streams);
  if (rc) return rc;

  // host preparation of every handle, with its stream work on the batch stream
  bool any_baseline = false;
  uint64_t bytes = 0;
  for (uint32_t i = 0; i < count; i++) {
    b2d_dedup* d = hs[i];
    // the batch's fused levels and map headroom apply to every handle it checkpoints
    d->warp_bands = cand.warp;
    if (d->map_headroom != cand.headroom / 100.0) {
      d->map_headroom = cand.headroom / 100.0;
      d->map_retune = true;
    }
    cudaStream_t keep = d->stream;
    d->stream = b->stream;
    const bool mb = make_baseline && make_baseline[i];
    any_baseline = any_baseline || mb || d->current_id == 0;
    rc = prepare_checkpoint(d, data[i], lens[i], mb);
    d->stream = keep;
    if (rc) {
      if (rcs) rcs[i] = rc;
      return rc;
    }
    bytes += lens[i];
  }

  // leaf work items: handles whose leaves the persistent kernel can hash, grouped by
  // (staging unit, hash kind); the rest hash their own leaves in their branch
  struct Group {
    int U, kind;
    uint32_t beg, end, tiles;
  };
  std::vector<Group> groups;
  std::vector<int> item_of(count, -1);
  std::vector<std::vector<BatchLeafItem>> by_group;
  for (uint32_t i = 0; i < count; i++) {
    b2d_dedup* d = hs[i];
    if (!d->tune.allow_tma) continue;
    BatchLeafItem it;
    std::memset(&it, 0, sizeof(it));
    const int U = batch_leaf_item(leaf_args(d, &d->state.p->round), it);
    if (U == 0) continue;
    size_t g = 0;
    while (g < groups.size() && !(groups[g].U == U && groups[g].kind == d->kind)) g++;
    if (g == groups.size()) {
      groups.push_back(Group{U, d->kind, 0, 0, 0});
      by_group.emplace_back();
    }
    if (by_group[g].size() >= BATCH_MAX_ITEMS) continue;
    it.tile_begin = groups[g].tiles;
    groups[g].tiles += it.ntiles;
    item_of[i] = (int)g;
    by_group[g].push_back(it);
  }
  std::vector<BatchLeafItem> items;
  for (size_t g = 0; g < groups.size(); g++) {
    groups[g].beg = (uint32_t)items.size();
    items.insert(items.end(), by_group[g].begin(), by_group[g].end());
    groups[g].end = (uint32_t)items.size();
  }

  // blob layout and contents
  BatchLayout L;
  L.items = 0;
  L.rounds = align_up(sizeof(BatchLeafItem) * items.size(), 64);
  L.states = align_up(L.rounds + sizeof(RoundState) * count, 64);
  L.queues = align_up(L.states + sizeof(DevState*) * count, 64);
  L.bstatus = align_up(L.queues + sizeof(unsigned int) * (groups.size() + 1), 64);
  L.dargs = align_up(L.bstatus + sizeof(DevStatus), 64);
  // list handles label and assemble their diffs in their own branches; the shared segmented
  // forest and diff launches take the tree handles (none: no shared launches)
  uint32_t trees = 0;
  for (uint32_t i = 0; i < count; i++) trees += hs[i]->list ? 0u : 1u;
  const bool seg_diff = b->batch_diff && cand.shared && trees > 0;
  L.dtab = align_up(L.dargs + (seg_diff ? sizeof(DiffArgs) * count : 0), 64);
  const size_t tab_len = (size_t)count + 1;   // entries per table
  // shared forest phases: every handle's launch steps, one segmented launch per (phase, step,
  // kind) with three tables (CTA offsets, p0, p1)
  const bool seg_forest = b->batch_forest && seg_diff;
  std::vector<std::vector<ForestStep>> fsteps[2];
  struct FLaunch {
    int phase, kind;
    uint32_t k, ctas;
    size_t off;
  };
  std::vector<FLaunch> flaunch;
  if (seg_forest) {
    for (int ph = 0; ph < 2; ph++) {
      fsteps[ph].resize(count);
      uint32_t K = 0;
      for (uint32_t i = 0; i < count; i++) {
        if (!hs[i]->list) forest_steps_batch(hs[i]->n, hs[i]->D, hs[i]->N, ph + 1, fsteps[ph][i], hs[i]->warp_bands);
        K = std::max<uint32_t>(K, (uint32_t)fsteps[ph][i].size());
      }
      for (uint32_t k = 0; k < K; k++)
        for (int kind = 0; kind < 3; kind++) {
          uint32_t ctas = 0;
          for (uint32_t i = 0; i < count; i++)
            if (k < fsteps[ph][i].size() && fsteps[ph][i][k].kind == kind) ctas += fsteps[ph][i][k].ctas;
          if (ctas) flaunch.push_back(FLaunch{ph + 1, kind, k, ctas, 0});
        }
    }
  }
  L.fargs = align_up(L.dtab + (seg_diff ? sizeof(uint32_t) * tab_len * DIFF_TABLES : 0), 64);
  L.ftab = align_up(L.fargs + (seg_forest ? sizeof(ForestArgs) * count : 0), 64);
  for (size_t q = 0; q < flaunch.size(); q++) flaunch[q].off = L.ftab + sizeof(uint32_t) * 3 * tab_len * q;
  L.total = align_up(L.ftab + sizeof(uint32_t) * 3 * tab_len * flaunch.size(), 256);
  B2D_CU(b->blob.reserve(L.total));
  B2D_CU(b->blob_h.reserve(L.total));
  B2D_CU(b->coll.reserve(count));
  B2D_CU(b->coll_h.reserve(count));
  uint8_t* H = b->blob_h.p;
  if (!items.empty()) std::memcpy(H + L.items, items.data(), sizeof(BatchLeafItem) * items.size());
  for (uint32_t i = 0; i < count; i++) {
    std::memcpy(H + L.rounds + sizeof(RoundState) * i, hs[i]->round_h.p, sizeof(RoundState));
    DevState* p = hs[i]->state.p;
    std::memcpy(H + L.states + sizeof(DevState*) * i, &p, sizeof(p));
  }
  uint8_t* B = b->blob.p;
  // shared diff assembly: every handle's DiffArgs, grid sizes and the CTA offset tables
  DiffBatch dplan{};
  if (seg_diff) {
    auto tab = [&](int t) { return reinterpret_cast<uint32_t*>(H + L.dtab) + (size_t)t * tab_len; };
    auto dtab = [&](int t) { return reinterpret_cast<const uint32_t*>(B + L.dtab) + (size_t)t * tab_len; };
    uint32_t tot_g = 0, tot_gl = 0, tot_gp = 0, tot_gs = 0, tot_one = 0, tot_v[GATHER_VARIANTS] = {0};
    uint32_t max_bcap = 1;
    for (uint32_t i = 0; i < count; i++) {
      b2d_dedup* d = hs[i];
      const DiffArgs da = diff_args(d, &d->state.p->round);
      std::memcpy(H + L.dargs + sizeof(DiffArgs) * i, &da, sizeof(da));
      DiffGrids dg = diff_grids(da, b->sm_count);
      if (d->list) dg.g = dg.gl = dg.gp = dg.gs = dg.gg = 0;   // its own branch assembles its diff
      tab(DT_G)[i] = dg.g;
      tab(DT_GS)[i] = dg.gs;
      tab(DT_BCAP)[i] = d->bcap;
      max_bcap = std::max(max_bcap, d->bcap);
      tab(DT_ONE)[i] = tot_one;
      tot_one += d->list ? 0u : 1u;
      tab(DT_BEG_G)[i] = tot_g;
      tot_g += dg.g;
      tab(DT_BEG_GL)[i] = tot_gl;
      tot_gl += dg.gl;
      tab(DT_BEG_GP)[i] = tot_gp;
      tot_gp += dg.gp;
      tab(DT_BEG_GS)[i] = tot_gs;
      tot_gs += dg.gs;
      for (int v = 0; v < GATHER_VARIANTS; v++) {
        tab(DT_BEG_GATHER + v)[i] = tot_v[v];
        if (v == dg.variant) tot_v[v] += dg.gg;
      }
    }
    tab(DT_ONE)[count] = tot_one;
    tab(DT_BEG_G)[count] = tot_g;
    tab(DT_BEG_GL)[count] = tot_gl;
    tab(DT_BEG_GP)[count] = tot_gp;
    tab(DT_BEG_GS)[count] = tot_gs;
    for (int v = 0; v < GATHER_VARIANTS; v++) tab(DT_BEG_GATHER + v)[count] = tot_v[v];
    dplan.base = SegGrid{reinterpret_cast<const DiffArgs*>(B + L.dargs), nullptr, dtab(DT_G), dtab(DT_GS),
                         dtab(DT_BCAP), count};
    dplan.beg_one = dtab(DT_ONE);
    dplan.beg_g = dtab(DT_BEG_G);
    dplan.beg_gl = dtab(DT_BEG_GL);
    dplan.beg_gp = dtab(DT_BEG_GP);
    dplan.beg_gs = dtab(DT_BEG_GS);
    for (int v = 0; v < GATHER_VARIANTS; v++) {
      dplan.beg_gather[v] = dtab(DT_BEG_GATHER + v);
      dplan.tot_gather[v] = tot_v[v];
    }
    dplan.tot_one = tot_one;
    dplan.tot_g = tot_g;
    dplan.tot_gl = tot_gl;
    dplan.tot_gp = tot_gp;
    dplan.tot_gs = tot_gs;
    dplan.max_bcap = max_bcap;
  }
  // shared forest phases: ForestArgs and per-launch tables
  std::vector<ForestSeg> fseg(flaunch.size());
  if (seg_forest) {
    for (uint32_t i = 0; i < count; i++) {
      const ForestArgs fa = forest_args(hs[i], &hs[i]->state.p->round);
      std::memcpy(H + L.fargs + sizeof(ForestArgs) * i, &fa, sizeof(fa));
    }
    for (size_t q = 0; q < flaunch.size(); q++) {
      const FLaunch& f = flaunch[q];
      uint32_t* beg = reinterpret_cast<uint32_t*>(H + f.off);
      uint32_t* p0 = beg + tab_len;
      uint32_t* p1 = p0 + tab_len;
      uint32_t acc = 0;
      for (uint32_t i = 0; i < count; i++) {
        beg[i] = acc;
        p0[i] = p1[i] = 0;
        const auto& st = fsteps[f.phase - 1][i];
        if (f.k < st.size() && st[f.k].kind == f.kind) {
          acc += st[f.k].ctas;
          p0[i] = st[f.k].p0;
          p1[i] = st[f.k].p1;
        }
      }
      beg[count] = acc;
      const uint32_t* dbeg = reinterpret_cast<const uint32_t*>(B + f.off);
      fseg[q] = ForestSeg{reinterpret_cast<const ForestArgs*>(B + L.fargs), dbeg, dbeg + tab_len,
                          dbeg + 2 * tab_len, count};
    }
  }
  auto* d_items = reinterpret_cast<BatchLeafItem*>(B + L.items);
  auto* d_rounds = reinterpret_cast<RoundState*>(B + L.rounds);
  auto* d_states = reinterpret_cast<DevState* const*>(B + L.states);
  auto* d_queues = reinterpret_cast<unsigned int*>(B + L.queues);
  auto* d_bst = reinterpret_cast<DevStatus*>(B + L.bstatus);

  // graph key: every handle's launch parameters, the grouping and the tuning
  std::vector<uint64_t> key, k1;
  for (uint32_t i = 0; i < count; i++) {
    graph_key(hs[i], &hs[i]->state.p->round, k1);
    key.insert(key.end(), k1.begin(), k1.end());
    key.push_back((uint64_t)(int64_t)item_of[i]);
  }
  for (auto& g : groups) key.insert(key.end(), {(uint64_t)g.U, (uint64_t)g.kind, g.beg, g.end, g.tiles});
  key.insert(key.end(), {(uint64_t)B, (uint64_t)H, L.total, (uint64_t)seg_diff, (uint64_t)seg_forest,
                         (uint64_t)b->coll.p,
                         (uint64_t)b->coll_h.p, (uint64_t)cand.stages,
                         (uint64_t)cand.ctas, (uint64_t)cand.tiles_per_pop, (uint64_t)cand.streams,
                         (uint64_t)cand.shared, (uint64_t)cand.warp});

  const uint64_t kh = key_hash(key);
  b2d_batch::GraphEntry* ge = nullptr;
  for (auto& g : b->graphs)
    if (g.hash == kh && g.key == key) ge = &g;

  // Everything the batch does, enqueued on `main` (the capture stream or the batch stream) and
  // the side streams: blob upload, init, hashing launches, per-handle branches, collection.
  auto enqueue_batch = [&](cudaStream_t main, uint32_t& launches) -> int {
    // branch assignment: largest handles first, each to the least loaded branch
    std::vector<uint32_t> order(count);
    for (uint32_t i = 0; i < count; i++) order[i] = i;
    std::sort(order.begin(), order.end(), [&](uint32_t x, uint32_t y) { return lens[x] > lens[y]; });
    const int nb = std::min<int>(cand.streams, (int)count);
    std::vector<uint64_t> load(nb, 0);
    std::vector<std::vector<uint32_t>> branch(nb);
    for (uint32_t i : order) {
      int best = 0;
      for (int j = 1; j < nb; j++)
        if (load[j] < load[best]) best = j;
      load[best] += lens[i] + (1ull << 20);   // fixed per-checkpoint cost ~ 1 MiB of data
      branch[best].push_back(i);
    }
    int erc = B2D_OK;
    auto cap_err = [&](cudaError_t e) {
      if (e != cudaSuccess && erc == B2D_OK) erc = cuda_status(e);
    };
    cap_err(cudaMemcpyAsync(B, H, L.total, cudaMemcpyHostToDevice, main));
    batch_init_kernel<<<(count + 255) / 256, 256, 0, main>>>(d_states, d_rounds, count, d_queues,
                                                             (uint32_t)groups.size(), d_bst);
    cap_err(cudaGetLastError());
    launches = 1;
    LeafTuning lt;
    lt.allow_tma = 1;
    lt.stages = cand.stages;
    lt.ctas_per_sm = cand.ctas;
    for (size_t gi = 0; gi < groups.size() && erc == B2D_OK; gi++) {
      const Group& gr = groups[gi];
      cap_err(launch_leaves_batch(d_items + gr.beg, gr.end - gr.beg, gr.tiles, gr.U, gr.kind, d_queues + gi, d_bst,
                                  b->sm_count, lt, (uint32_t)cand.tiles_per_pop, main));
      launches++;
    }
    cap_err(cudaEventRecord(b->fork_ev, main));
    for (int j = 0; j < nb && erc == B2D_OK; j++) {
      cudaStream_t s = b->side[j];
      cap_err(cudaStreamWaitEvent(s, b->fork_ev, 0));
      for (uint32_t i : branch[j]) {
        if (erc != B2D_OK) break;
        b2d_dedup* d = hs[i];
        const bool skip_leaves = item_of[i] >= 0;
        // nothing of a tree handle runs in a branch when its leaves, forest and diff are all
        // shared; a list handle labels and assembles its diff here
        if (seg_forest && skip_leaves && !d->list) continue;
        const int r = enqueue_checkpoint(d, s, &d->state.p->round, false, false, skip_leaves, true,
                                         seg_diff && !d->list, seg_forest);
        if (r != B2D_OK) erc = r;
        launches += d->launches;
      }
      cap_err(cudaEventRecord(b->side_ev[j], s));
      cap_err(cudaStreamWaitEvent(main, b->side_ev[j], 0));
    }
    if (seg_forest && erc == B2D_OK) {
      // phase 1 steps, the zero-digest probe, phase 2 steps: each over every handle at once
      for (size_t q = 0; q < flaunch.size() && erc == B2D_OK; q++) {
        if (flaunch[q].phase != 1) continue;
        cap_err(launch_forest_seg(fseg[q], 1, flaunch[q].kind, flaunch[q].ctas, main));
        launches++;
      }
      cap_err(launch_zero_exists_seg(reinterpret_cast<const ForestArgs*>(B + L.fargs), count, main));
      launches++;
      for (size_t q = 0; q < flaunch.size() && erc == B2D_OK; q++) {
        if (flaunch[q].phase != 2) continue;
        cap_err(launch_forest_seg(fseg[q], 2, flaunch[q].kind, flaunch[q].ctas, main));
        launches++;
      }
    }
    if (seg_diff && erc == B2D_OK) {
      uint32_t dl = 0;
      cap_err(launch_collect_diff_batch(dplan, main, &dl));
      launches += dl;
    }
    batch_collect_kernel<<<(count + 127) / 128, 128, 0, main>>>(d_states, count, b->coll.p);
    cap_err(cudaGetLastError());
    cap_err(cudaMemcpyAsync(b->coll_h.p, b->coll.p, sizeof(DevState) * count, cudaMemcpyDeviceToHost, main));
    cap_err(cudaMemcpyAsync(H + L.bstatus, d_bst, sizeof(DevStatus), cudaMemcpyDeviceToHost, main));
    launches += 1;
    return erc;
  };

  // graph_mode 1: always replay a graph; 2: capture one the second time a composition comes
  // (a stream of ever-new compositions, like a request loop's, would pay a capture each time)
  // (the tuner compares graph replays: a direct launch's device time includes host enqueueing)
  bool use_graph = ge != nullptr || b->graph_mode == 1 || (scoring && b->graph_mode != 0);
  if (!use_graph && b->graph_mode == 2) {
    if (std::find(b->seen.begin(), b->seen.end(), kh) != b->seen.end()) {
      use_graph = true;
    } else {
      if (b->seen.size() >= 4 * b->graph_cap) b->seen.erase(b->seen.begin());
      b->seen.push_back(kh);
    }
  }
  b->leaf_groups = (uint32_t)groups.size();
  b->lay = L;
  if (!use_graph) {
    uint32_t launches = 0;
    B2D_CU(cudaEventRecord(b->ev[0], b->stream));
    const int erc = enqueue_batch(b->stream, launches);
    if (erc != B2D_OK) {
      cudaStreamSynchronize(b->stream);
      return erc;
    }
    B2D_CU(cudaEventRecord(b->ev[1], b->stream));
    b->launches = launches;
  } else {
    if (!ge) {
      if (b->graphs.size() >= b->graph_cap) {
        size_t lru = 0;
        for (size_t i = 1; i < b->graphs.size(); i++)
          if (b->graphs[i].last_use < b->graphs[lru].last_use) lru = i;
        cudaGraphExecDestroy(b->graphs[lru].exec);
        b->graphs.erase(b->graphs.begin() + (long)lru);
      }
      cudaGraph_t g = nullptr;
      uint32_t launches = 0;
      B2D_CU(cudaStreamBeginCapture(b->cap, cudaStreamCaptureModeThreadLocal));
      const int erc = enqueue_batch(b->cap, launches);
      const cudaError_t ce = cudaStreamEndCapture(b->cap, &g);
      if (erc != B2D_OK) {
        if (g) cudaGraphDestroy(g);
        return erc;
      }
      B2D_CU(ce);
      cudaGraphExec_t exec = nullptr;
      const cudaError_t ie = cudaGraphInstantiate(&exec, g, 0);
      cudaGraphDestroy(g);
      B2D_CU(ie);
      const cudaError_t ue = cudaGraphUpload(exec, b->stream);
      if (ue != cudaSuccess) {
        cudaGraphExecDestroy(exec);
        return cuda_status(ue);
      }
      b->graphs.emplace_back();
      ge = &b->graphs.back();
      ge->key = key;
      ge->hash = kh;
      ge->exec = exec;
      ge->launches = launches;
    }
    ge->last_use = ++b->use_clock;
    b->launches = ge->launches;
    B2D_CU(cudaEventRecord(b->ev[0], b->stream));
    B2D_CU(cudaGraphLaunch(ge->exec, b->stream));
    B2D_CU(cudaEventRecord(b->ev[1], b->stream));
  }
  b->inflight = true;
  b->fl_handles.assign(hs, hs + count);
  b->fl_bytes = bytes;
  b->fl_scoring = scoring;
  b->fl_any_baseline = any_baseline;
  b->fl_t0 = t0;
  return B2D_OK;
}

// Waits for the batch in flight and completes every handle's checkpoint.
int batch_finish(b2d_batch* b, int* rcs) {
  using clk = std::chrono::high_resolution_clock;
  if (!b->inflight) return B2D_ERR_ARG;
  b->inflight = false;
  B2D_CU(cudaEventSynchronize(b->ev[1]));
  b->dev_s = elapsed_ms(b->ev[0], b->ev[1]) * 1e-3;
  const uint32_t count = (uint32_t)b->fl_handles.size();
  b2d_dedup* const* hs = b->fl_handles.data();

  // the persistent leaf kernel's own status (a wait that ran out) fails every handle
  DevStatus bst;
  std::memcpy(&bst, b->blob_h.p + b->lay.bstatus, sizeof(bst));
  int first_rc = status_code(bst);
  for (uint32_t i = 0; i < count; i++) {
    b2d_dedup* d = hs[i];
    *d->state_h.p = b->coll_h.p[i];
    cudaStream_t keep = d->stream;
    d->stream = b->stream;
    int r = finish_checkpoint(d, true, false);
    d->stream = keep;
    if (r == B2D_OK && first_rc != B2D_OK) {
      r = first_rc;
      d->diff_valid = false;
      d->have_tree = false;   // its leaves may not have been hashed
    }
    d->phase[0] = d->phase[1] = d->phase[2] = 0;
    if (rcs) rcs[i] = r;
    if (r != B2D_OK && first_rc == B2D_OK) first_rc = r;
  }
  b->host_s = secs(b->fl_t0, clk::now());
  // baselines cost more than incremental checkpoints: only incremental batches are compared
  if (b->fl_scoring && !b->fl_any_baseline && first_rc == B2D_OK) {
    b->tuner.report(b->dev_s > 0 ? (double)b->fl_bytes / b->dev_s : 0.0);
    if (b->tuner.done) b->cur = b->tuner.base;
  }
  b->fl_handles.clear();
  return first_rc;
}

}  // namespace

#define B2D_GUARD(body)                    \
  try {                                    \
    body                                   \
  } catch (const std::bad_alloc&) {        \
    return B2D_ERR_NOMEM;                  \
  } catch (...) {                          \
    return B2D_ERR_INTERNAL;               \
  }

extern "C" {

int b2d_create_list(uint32_t chunk_size, int hash_kind, b2d_dedup** out) {
  const int rc = b2d_create(chunk_size, hash_kind, out);
  if (rc == B2D_OK) (*out)->list = 1;
  return rc;
}

int b2d_create(uint32_t chunk_size, int hash_kind, b2d_dedup** out) {
  B2D_GUARD({
    if (!out || chunk_size == 0 || (hash_kind != B2D_HASH_MURMUR3 && hash_kind != B2D_HASH_MD5)) return B2D_ERR_ARG;
    *out = nullptr;
    b2d_dedup* d = new b2d_dedup();
    d->chunk_size = chunk_size;
    d->kind = hash_kind;
    cudaError_t e = cudaGetDevice(&d->device);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&d->sm_count, cudaDevAttrMultiProcessorCount, d->device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&d->own_stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&d->cap_stream, cudaStreamNonBlocking);
    for (auto& ev : d->ev)
      if (e == cudaSuccess) e = cudaEventCreate(&ev);
    if (e != cudaSuccess) {
      delete d;
      return cuda_status(e);
    }
    d->stream = d->own_stream;
    *out = d;
    return B2D_OK;
  })
}

int b2d_destroy(b2d_dedup* d) {
  if (!d) return B2D_ERR_ARG;
  if (d->stream) cudaStreamSynchronize(d->stream);
  delete d;
  return B2D_OK;
}

int b2d_set_stream(b2d_dedup* d, void* s) {
  if (!d) return B2D_ERR_ARG;
  d->stream = s ? static_cast<cudaStream_t>(s) : d->own_stream;
  return B2D_OK;
}

int b2d_checkpoint_device(b2d_dedup* d, const void* d_data, uint64_t len, int make_baseline, int advance_id,
                          uint64_t* diff_len) {
  B2D_GUARD({
    if (!d) return B2D_ERR_ARG;
    int rc = do_checkpoint(d, d_data, len, make_baseline != 0, advance_id != 0);
    if (rc == B2D_OK && diff_len) *diff_len = d->diff_len;
    return rc;
  })
}

int b2d_diff_device(b2d_dedup* d, const void** d_diff, uint64_t* diff_len) {
  if (!d || !d->diff_valid) return B2D_ERR_ARG;
  if (d_diff) *d_diff = d->diff.p + d->diff_delta;
  if (diff_len) *diff_len = d->diff_len;
  return B2D_OK;
}

int b2d_copy_diff(b2d_dedup* d, void* dst, uint64_t cap) {
  B2D_GUARD({
    if (!d || !dst) return B2D_ERR_ARG;
    return copy_diff(d, dst, cap);
  })
}

int b2d_copy_diff_async(b2d_dedup* d, void* dst, uint64_t cap, void* stream) {
  if (!d || !dst || !d->diff_valid || cap < d->diff_len) return B2D_ERR_ARG;
  cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : d->stream;
  B2D_CU(cudaMemcpyAsync(dst, d->diff.p + d->diff_delta, d->diff_len, cudaMemcpyDeviceToHost, s));
  return B2D_OK;
}

int b2d_write_chkpt_log(b2d_dedup* d, const char* logname) {
  B2D_GUARD({
    if (!d || !logname || !d->diff_valid) return B2D_ERR_ARG;
    // header and repeat table of the device diff (the first-occurrence list between them stays)
    const uint8_t* dd = d->diff.p + d->diff_delta;
    uint8_t hdr[32];
    B2D_CU(cudaMemcpyAsync(hdr, dd, 32, cudaMemcpyDeviceToHost, d->stream));
    B2D_CU(cudaStreamSynchronize(d->stream));
    uint32_t nf = 0;
    uint32_t np = 0;
    memcpy(&nf, hdr + 20, 4);
    memcpy(&np, hdr + 24, 4);
    std::vector<uint8_t> ctab(8ull * np + 8);
    if (np) {
      B2D_CU(cudaMemcpyAsync(ctab.data(), dd + 32 + 4ull * nf, 8ull * np, cudaMemcpyDeviceToHost, d->stream));
      B2D_CU(cudaStreamSynchronize(d->stream));
    }
    uint32_t id = 0;
    memcpy(&id, hdr + 4, 4);   // chkpt_id of the diff
    return write_chkpt_log(d, hdr, ctab.data(), logname, id);
  })
}

int b2d_write_chkpt_log_host(b2d_dedup* d, const void* header, const uint8_t* diff, uint64_t diff_len,
                             const char* logname) {
  B2D_GUARD({
    if (!d || !header || !diff || !logname) return B2D_ERR_ARG;
    const uint8_t* h = static_cast<const uint8_t*>(header);
    uint32_t nf = 0;
    uint32_t np = 0;
    memcpy(&nf, h + 20, 4);
    memcpy(&np, h + 24, 4);
    if (diff_len < 32ull + 4ull * nf + 8ull * np) return B2D_ERR_FORMAT;
    return write_chkpt_log(d, h, diff + 32 + 4ull * nf, logname, d->current_id);
  })
}

int b2d_write_restart_log(b2d_dedup* d, uint32_t select_chkpt, const char* logname) {
  B2D_GUARD({
    if (!d || !logname) return B2D_ERR_ARG;
    return write_restart_log(d, select_chkpt, logname);
  })
}

int b2d_checkpoint(b2d_dedup* d, const void* d_data, uint64_t len, int make_baseline, const uint8_t** diff,
                   uint64_t* diff_len) {
  B2D_GUARD({
    if (!d) return B2D_ERR_ARG;
    return checkpoint_to_pinned(d, d_data, len, make_baseline != 0, true, diff, diff_len);
  })
}

int b2d_checkpoint_log(b2d_dedup* d, const void* d_data, uint64_t len, const char* logname, int make_baseline,
                       const uint8_t** diff, uint64_t* diff_len) {
  B2D_GUARD({
    if (!d || !logname) return B2D_ERR_ARG;
    const uint8_t* p = nullptr;
    uint64_t n = 0;
    int rc = checkpoint_to_pinned(d, d_data, len, make_baseline != 0, false, &p, &n);
    if (rc) return rc;
    if (n < 32) return B2D_ERR_FORMAT;
    rc = write_chkpt_log(d, p, p + 32 + 4ull * d->F, logname, d->current_id);
    d->current_id += 1;
    if (diff) *diff = p;
    if (diff_len) *diff_len = n;
    return rc;
  })
}

int b2d_checkpoint_file(b2d_dedup* d, const void* d_data, uint64_t len, const char* filename, const char* logname,
                        int make_baseline) {
  B2D_GUARD({
    if (!d || !filename || !logname) return B2D_ERR_ARG;
    const uint8_t* p = nullptr;
    uint64_t n = 0;
    int rc = checkpoint_to_pinned(d, d_data, len, make_baseline != 0, false, &p, &n);
    if (rc) return rc;
    // the tree and map now hold this checkpoint; if its file is not written, no later diff may
    // reference it, so the handle then accepts only a baseline (with the same checkpoint id)
    if (n < 32) rc = B2D_ERR_FORMAT;
    if (!rc) rc = write_chkpt_log(d, p, p + 32 + 4ull * d->F, logname, d->current_id);
    if (!rc) {
      FILE* f = fopen(filename, "wb");
      if (!f) {
        rc = B2D_ERR_IO;
      } else {
        const size_t w = fwrite(p, 1, n, f);
        const int cl = fclose(f);
        if (w != n || cl != 0) rc = B2D_ERR_IO;
      }
    }
    if (rc) {
      d->have_tree = false;
      return rc;
    }
    d->current_id += 1;
    return B2D_OK;
  })
}

int b2d_restart(b2d_dedup* d, void* d_out, uint64_t len, const uint8_t* const* diffs, const uint64_t* sizes,
                uint32_t num_diffs, uint32_t chkpt_id, const char* logname) {
  B2D_GUARD({
    if (!d) return B2D_ERR_ARG;
    int rc = do_restart(d, d_out, len, diffs, sizes, num_diffs, chkpt_id);
    if (logname) {
      const std::string ln = std::string(logname) + ".chunk_size." + std::to_string(d->chunk_size) +
                             ".restart_timing.csv";
      write_restart_log(d, chkpt_id, ln);
    }
    return rc;
  })
}

int b2d_restart_device(b2d_dedup* d, void* d_out, uint64_t len, const void* const* d_diffs, const uint64_t* sizes,
                       uint32_t num_diffs, uint32_t chkpt_id) {
  B2D_GUARD({
    if (!d || !d_diffs) return B2D_ERR_ARG;
    return do_restart(d, d_out, len, nullptr, sizes, num_diffs, chkpt_id, d_diffs);
  })
}

int b2d_restart_files(b2d_dedup* d, void* d_out, uint64_t len, const char* const* names, uint32_t num_files,
                      uint32_t chkpt_id, const char* logname) {
  B2D_GUARD({
    if (!d || !names || chkpt_id >= num_files) return B2D_ERR_ARG;
    std::vector<std::vector<uint8_t>> bufs(num_files);
    std::vector<const uint8_t*> ptrs(num_files, nullptr);
    std::vector<uint64_t> sizes(num_files, 0);
    for (uint32_t i = 0; i < num_files; i++) {
      if (!names[i]) return B2D_ERR_ARG;
      if (i > chkpt_id) continue;
      int rc = read_file(std::string(names[i]) + ".hashtree.incr_chkpt", bufs[i]);
      if (rc) return rc;
      ptrs[i] = bufs[i].data();
      sizes[i] = bufs[i].size();
    }
    int rc = do_restart(d, d_out, len, ptrs.data(), sizes.data(), num_files, chkpt_id);
    if (logname) write_restart_log(d, chkpt_id, logname);
    return rc;
  })
}

int b2d_set_param(b2d_dedup* d, const char* name, int64_t value) {
  if (!d || !name) return B2D_ERR_ARG;
  const std::string k(name);
  if (k == "leaf_tma") d->tune.allow_tma = value != 0;
  else if (k == "leaf_stages" && value >= 0 && value <= 16) d->tune.stages = (int)value;
  else if (k == "leaf_ctas_per_sm" && value >= 0 && value <= 8) d->tune.ctas_per_sm = (int)value;
  else if (k == "leaf_unit" && (value == 0 || value == 16 || value == 32 || value == 64 || value == 128))
    d->tune.unit = (int)value;
  else if (k == "leaf_wait_polls" && value >= 0 && value <= (1 << 20)) d->tune.wait_polls = (int)value;
  else if (k == "map_max_load_pct" && value >= 10 && value <= 90) d->map_max_load = value / 100.0;
  else if (k == "map_headroom_pct" && value >= 100 && value <= 1000) d->map_headroom = value / 100.0;
  else if (k == "warp_bands" && value >= 0 && value <= 3) d->warp_bands = (int)value;
  else if (k == "graph" && value >= 0 && value <= 2) {
    d->use_graph = value != 0;
    d->graph_timing = value != 2;
  }
  else return B2D_ERR_ARG;
  return B2D_OK;
}

int b2d_num_first_ocur(b2d_dedup* d, uint64_t* out) {
  if (!d || !out) return B2D_ERR_ARG;
  *out = d->F;
  return B2D_OK;
}
int b2d_num_shift_dupl(b2d_dedup* d, uint64_t* out) {
  if (!d || !out) return B2D_ERR_ARG;
  *out = d->S;
  return B2D_OK;
}
int b2d_current_id(b2d_dedup* d, uint32_t* out) {
  if (!d || !out) return B2D_ERR_ARG;
  *out = d->current_id;
  return B2D_OK;
}
int b2d_baseline_id(b2d_dedup* d, uint32_t* out) {
  if (!d || !out) return B2D_ERR_ARG;
  *out = d->baseline_id;
  return B2D_OK;
}
int b2d_timers(b2d_dedup* d, double out[4]) {
  if (!d || !out) return B2D_ERR_ARG;
  for (int i = 0; i < 4; i++) out[i] = d->timers[i];
  return B2D_OK;
}
int b2d_restart_timers(b2d_dedup* d, double out[2]) {
  if (!d || !out) return B2D_ERR_ARG;
  out[0] = d->restart_timers[0];
  out[1] = d->restart_timers[1];
  return B2D_OK;
}
int b2d_datasizes(b2d_dedup* d, uint64_t out[2]) {
  if (!d || !out) return B2D_ERR_ARG;
  out[0] = d->datasizes[0];
  out[1] = d->datasizes[1];
  return B2D_OK;
}
int b2d_phase_times(b2d_dedup* d, double out[3], int* leaf_path) {
  if (!d || !out) return B2D_ERR_ARG;
  for (int i = 0; i < 3; i++) out[i] = d->phase[i];
  if (leaf_path) *leaf_path = d->leaf_tma ? 1 : 0;
  return B2D_OK;
}
int b2d_last_launch_count(b2d_dedup* d, uint32_t* out) {
  if (!d || !out) return B2D_ERR_ARG;
  *out = d->launches;
  return B2D_OK;
}
int b2d_debug_tree(b2d_dedup* d, void* dst, uint64_t nodes) {
  if (!d || !dst || nodes > d->N || !d->tree.p) return B2D_ERR_ARG;
  B2D_CU(cudaMemcpyAsync(dst, d->tree.p, 16ull * nodes, cudaMemcpyDeviceToHost, d->stream));
  B2D_CU(cudaStreamSynchronize(d->stream));
  return B2D_OK;
}
int b2d_debug_labels(b2d_dedup* d, void* dst, uint64_t leaves) {
  if (!d || !dst || leaves > d->n || !d->leaflab.p) return B2D_ERR_ARG;
  B2D_CU(cudaMemcpyAsync(dst, d->leaflab.p, leaves, cudaMemcpyDeviceToHost, d->stream));
  B2D_CU(cudaStreamSynchronize(d->stream));
  return B2D_OK;
}
int b2d_hash_host(int kind, const void* data, uint64_t len, void* out16) {
  if ((!data && len) || !out16 || (kind != HASH_MURMUR3 && kind != HASH_MD5)) return B2D_ERR_ARG;
  const Digest dg = hash_bytes(kind, static_cast<const uint8_t*>(data), len);
  std::memcpy(out16, dg.w, 16);
  return B2D_OK;
}

int b2d_hash_chunks(int kind, const void* d_data, uint64_t len, uint32_t cs, void* d_out, void* stream) {
  if (!d_data || !d_out || cs == 0 || len == 0) return B2D_ERR_ARG;
  const uint64_t n = (len + cs - 1) / cs;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  uint64_t blocks = (n + 255) / 256;
  if (blocks > 65535) blocks = 65535;
  hash_chunks_kernel<<<(unsigned)blocks, 256, 0, s>>>(kind, static_cast<const uint8_t*>(d_data), len, cs, n,
                                                      static_cast<Digest*>(d_out));
  B2D_CU(cudaGetLastError());
  B2D_CU(cudaStreamSynchronize(s));
  return B2D_OK;
}

int b2d_map_stats(b2d_dedup* d, double out[5]) {
  if (!d || !out) return B2D_ERR_ARG;
  out[0] = (double)d->map_cap;
  out[1] = (double)d->map_size_host;
  out[2] = (double)d->map_grows;
  out[3] = d->map_grow_s;
  out[4] = d->map_alloc_s;
  return B2D_OK;
}

int b2d_pool_reserve(uint64_t bytes) {
  B2D_GUARD({
    int dev = 0;
    B2D_CU(cudaGetDevice(&dev));
    cudaMemPool_t pool = map_pool(dev);
    if (!pool) return B2D_ERR_CUDA;
    {
      std::lock_guard<std::mutex> lock(g_pool_mu);
      if ((int)g_pool_keep.size() <= dev) g_pool_keep.resize(dev + 1, 0);
      g_pool_keep[dev] = bytes;
    }
    if (bytes == 0) {
      B2D_CU(cudaMemPoolTrimTo(pool, 0));
      return B2D_OK;
    }
    // map the memory once: allocate it as one block and hand it back to the pool, which keeps
    // it (release threshold: never) and carves later map allocations out of it
    cudaStream_t s = nullptr;
    B2D_CU(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    void* p = nullptr;
    cudaError_t e = cudaMallocFromPoolAsync(&p, bytes, pool, s);
    if (e == cudaSuccess) e = cudaFreeAsync(p, s);
    const cudaError_t e2 = cudaStreamSynchronize(s);
    cudaStreamDestroy(s);
    B2D_CU(e);
    B2D_CU(e2);
    return B2D_OK;
  })
}

int b2d_memory(b2d_dedup* d, uint64_t* bytes) {
  if (!d || !bytes) return B2D_ERR_ARG;
  *bytes = handle_bytes(d);
  return B2D_OK;
}

int b2d_estimate_memory(uint64_t len, uint32_t chunk_size, int map_max_load_pct, uint64_t* bytes) {
  if (!bytes || chunk_size == 0 || len == 0) return B2D_ERR_ARG;
  if (map_max_load_pct <= 0) map_max_load_pct = 75;
  if (map_max_load_pct < 10 || map_max_load_pct > 90) return B2D_ERR_ARG;
  // the allocations prepare_checkpoint makes for a buffer of `len` bytes (checkpoint side)
  const uint64_t n = (len + chunk_size - 1) / chunk_size, N = 2 * n - 1;
  const uint64_t cap = map_capacity(2 * N, map_max_load_pct / 100.0, MAP_HEADROOM);
  uint64_t b = N * sizeof(Digest) + N + (n + 16) + ((N + 63) / 64 * 16 + 16) + n;   // tree, labels, flags
  b += (cap + 1) * MAP_SLOT_BYTES + 8;                                               // map
  b += 8 * 4 * n + 68 * 4;                                                           // lists and keys
  b += (uint64_t)64 * 4 * 2 + (uint64_t)1184 * 64 * 4 + 2 * COMPACT_GRID * 4;           // buckets, partials
  b += 64 + 16 * n + n * chunk_size;                                                 // diff
  b += sizeof(DevState);
  *bytes = b;
  return B2D_OK;
}

int b2d_batch_create(b2d_batch** out) {
  B2D_GUARD({
    if (!out) return B2D_ERR_ARG;
    *out = nullptr;
    b2d_batch* b = new b2d_batch();
    cudaError_t e = cudaGetDevice(&b->device);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&b->sm_count, cudaDevAttrMultiProcessorCount, b->device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&b->own_stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&b->cap, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->fork_ev, cudaEventDisableTiming);
    for (auto& ev : b->ev)
      if (e == cudaSuccess) e = cudaEventCreate(&ev);
    if (e != cudaSuccess) {
      delete b;
      return cuda_status(e);
    }
    b->stream = b->own_stream;
    *out = b;
    return B2D_OK;
  })
}

int b2d_batch_destroy(b2d_batch* b) {
  if (!b) return B2D_ERR_ARG;
  if (b->inflight) batch_finish(b, nullptr);
  if (b->stream) cudaStreamSynchronize(b->stream);
  delete b;
  return B2D_OK;
}

int b2d_batch_set_stream(b2d_batch* b, void* s) {
  if (!b) return B2D_ERR_ARG;
  b->stream = s ? static_cast<cudaStream_t>(s) : b->own_stream;
  return B2D_OK;
}

int b2d_batch_set_param(b2d_batch* b, const char* name, int64_t value) {
  if (!b || !name) return B2D_ERR_ARG;
  const std::string k(name);
  if (k == "leaf_stages" && value >= 0 && value <= 16) b->cur.stages = (int)value;
  else if (k == "leaf_ctas_per_sm" && value >= 0 && value <= 8) b->cur.ctas = (int)value;
  else if (k == "tiles_per_pop" && value >= 1 && value <= 1024) b->cur.tiles_per_pop = (int)value;
  else if (k == "streams" && value >= 1 && value <= 64) b->cur.streams = (int)value;
  else if (k == "shared" && (value == 0 || value == 1)) b->cur.shared = (int)value;
  else if (k == "warp_bands" && value >= 0 && value <= 3) b->cur.warp = (int)value;
  else if (k == "map_headroom_pct" && value >= 100 && value <= 1000) b->cur.headroom = (int)value;
  else if (k == "graph_cache" && value >= 1 && value <= 4096) b->graph_cap = (size_t)value;
  else if (k == "graph" && value >= 0 && value <= 2) b->graph_mode = (int)value;
  else if (k == "batch_diff" && (value == 0 || value == 1)) b->batch_diff = value != 0;
  else if (k == "batch_forest" && (value == 0 || value == 1)) b->batch_forest = value != 0;
  else if (k == "autotune" && (value == 0 || value == 1)) {
    b->autotune = value != 0;
    b->tuner.reset(b->cur);
  } else return B2D_ERR_ARG;
  return B2D_OK;
}

int b2d_batch_get_param(b2d_batch* b, const char* name, int64_t* value) {
  if (!b || !name || !value) return B2D_ERR_ARG;
  const std::string k(name);
  if (k == "leaf_stages") *value = b->cur.stages;
  else if (k == "leaf_ctas_per_sm") *value = b->cur.ctas;
  else if (k == "tiles_per_pop") *value = b->cur.tiles_per_pop;
  else if (k == "streams") *value = b->cur.streams;
  else if (k == "shared") *value = b->cur.shared;
  else if (k == "warp_bands") *value = b->cur.warp;
  else if (k == "map_headroom_pct") *value = b->cur.headroom;
  else if (k == "autotune") *value = b->autotune ? 1 : 0;
  else if (k == "tuned") *value = b->tuner.done ? 1 : 0;
  else if (k == "graph_cache") *value = (int64_t)b->graph_cap;
  else if (k == "graphs") *value = (int64_t)b->graphs.size();
  else if (k == "graph") *value = b->graph_mode;
  else if (k == "batch_diff") *value = b->batch_diff ? 1 : 0;
  else if (k == "batch_forest") *value = b->batch_forest ? 1 : 0;
  else return B2D_ERR_ARG;
  return B2D_OK;
}

int b2d_batch_checkpoint(b2d_batch* b, b2d_dedup* const* handles, const void* const* d_data, const uint64_t* lens,
                         const int* make_baseline, uint32_t count, int* rcs) {
  B2D_GUARD({
    if (!b || (count && (!handles || !d_data || !lens))) return B2D_ERR_ARG;
    int rc = batch_launch(b, handles, d_data, lens, make_baseline, count, rcs);
    if (rc != B2D_OK || count == 0) return rc;
    return batch_finish(b, rcs);
  })
}

int b2d_batch_launch(b2d_batch* b, b2d_dedup* const* handles, const void* const* d_data, const uint64_t* lens,
                     const int* make_baseline, uint32_t count, int* rcs) {
  B2D_GUARD({
    if (!b || !count || !handles || !d_data || !lens) return B2D_ERR_ARG;
    return batch_launch(b, handles, d_data, lens, make_baseline, count, rcs);
  })
}

int b2d_batch_query(b2d_batch* b, int* done) {
  if (!b || !done) return B2D_ERR_ARG;
  if (!b->inflight) {
    *done = -1;
    return B2D_OK;
  }
  const cudaError_t e = cudaEventQuery(b->ev[1]);
  if (e == cudaErrorNotReady) {
    *done = 0;
    return B2D_OK;
  }
  *done = 1;
  if (e != cudaSuccess) {
    (void)cudaGetLastError();
    return cuda_status(e);
  }
  return B2D_OK;
}

int b2d_batch_wait(b2d_batch* b, int* rcs) {
  B2D_GUARD({
    if (!b) return B2D_ERR_ARG;
    return batch_finish(b, rcs);
  })
}

int b2d_batch_times(b2d_batch* b, double out[2]) {
  if (!b || !out) return B2D_ERR_ARG;
  out[0] = b->dev_s;
  out[1] = b->host_s;
  return B2D_OK;
}

int b2d_batch_launch_count(b2d_batch* b, uint32_t* out) {
  if (!b || !out) return B2D_ERR_ARG;
  *out = b->launches;
  return B2D_OK;
}

const char* b2d_strerror(int s) {
  switch (s) {
    case B2D_OK: return "ok";
    case B2D_ERR_ARG: return "invalid argument";
    case B2D_ERR_CUDA: return "CUDA runtime error";
    case B2D_ERR_NOMEM: return "out of memory";
    case B2D_ERR_FORMAT: return "malformed diff";
    case B2D_ERR_IO: return "file I/O error";
    case B2D_ERR_MAP_FULL: return "digest map full";
    case B2D_ERR_TIMEOUT: return "bounded device wait timed out";
    case B2D_ERR_INTERNAL: return "internal invariant violated";
    case B2D_ERR_RESTART_RANGE: return "restart access outside buffer bounds (skipped)";
    case B2D_ERR_LEN_CHANGED: return "buffer length changed without a new baseline";
    case B2D_ERR_UNSUPPORTED: return "unsupported configuration";
    default: return "unknown status";
  }
}

}  // extern "C"

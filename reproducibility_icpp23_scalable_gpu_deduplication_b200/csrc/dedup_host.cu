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
};

__global__ void map_special_init_kernel(MapSlot* special) {
  special->key_lo = 0;
  special->key_hi = 0;
  special->val = ~0ull;
  special->tree = MAP_TREE_PENDING;
  special->pad = 0;   // unoccupied
}

// move every occupied slot of `from` into the (empty) table `to`
__global__ void map_rehash_kernel(MapView from, MapView to, DevStatus* st) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i <= from.cap;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const MapSlot s = from.slots[i];
    if (i == from.cap) {
      if (s.pad) to.slots[to.cap] = s;
      continue;
    }
    if (s.key_lo == MAP_EMPTY && s.key_hi == MAP_EMPTY) continue;
    Digest d;
    d.w[0] = (uint32_t)s.key_lo; d.w[1] = (uint32_t)(s.key_lo >> 32);
    d.w[2] = (uint32_t)s.key_hi; d.w[3] = (uint32_t)(s.key_hi >> 32);
    const MapRef r = map_insert(to, d, s.val, s.tree, st);
    if (r.found) {
      to.slots[r.slot].val = s.val;
      to.slots[r.slot].tree = s.tree;
    }
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
};

}  // namespace b2d

using namespace b2d;

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

  uint32_t n = 0, N = 0, D = 0;
  uint64_t F = 0, S = 0;
  uint32_t launches = 0;
  double phase[3] = {0, 0, 0};   // device time of leaves, forest, diff assembly (last checkpoint)
  bool leaf_tma = false;
  bool have_tree = false;
  LeafTuning tune;
  double map_max_load = 0.75;

  cudaStream_t own_stream = nullptr;
  cudaStream_t stream = nullptr;
  int device = 0;
  int sm_count = 148;
  cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};

  DevBuf<Digest> tree;
  DevBuf<uint8_t> lab, leaflab, push, dupflag;
  DevBuf<MapSlot> map_slots;
  uint64_t map_cap = 0;           // power of two; slots hold map_cap + 1 entries
  uint64_t map_size_host = 0;     // occupied slots after the last checkpoint
  DevBuf<unsigned long long> map_size;
  DevBuf<uint32_t> tmp_first, tmp_shift, levels;
  DevBuf<uint32_t> first_list, shift_list, region_off, sprev, skey, hist, bucket_start, partial, partial2;
  DevBuf<uint8_t> diff;
  DevBuf<DevState> state;
  PinnedBuf<DevState> state_h;
  PinnedBuf<uint8_t> diff_h;
  uint64_t diff_len = 0;
  uint32_t diff_delta = 0;
  bool diff_valid = false;

  // restart scratch
  DevBuf<uint2> r_node_list, r_rep;
  DevBuf<unsigned long long> r_dist;
  DevBuf<uint32_t> r_offs, r_partial;
  DevBuf<unsigned long long> r_cum, r_total;
  DevBuf<uint8_t> r_diff;
  PinnedBuf<uint8_t> r_stage;

  ~b2d_dedup() {
    for (auto& e : ev)
      if (e) cudaEventDestroy(e);
    if (own_stream) cudaStreamDestroy(own_stream);
  }
};

namespace {

int map_view(b2d_dedup* d, MapView& m) {
  m.slots = d->map_slots.p;
  m.cap = d->map_cap;
  m.mask = d->map_cap - 1;
  m.size = d->map_size.p;
  return B2D_OK;
}

int map_reset(b2d_dedup* d, uint64_t cap) {
  B2D_CU(d->map_slots.reserve(cap + 1));
  d->map_cap = cap;
  B2D_CU(cudaMemsetAsync(d->map_slots.p, 0xff, sizeof(MapSlot) * (cap + 1), d->stream));
  map_special_init_kernel<<<1, 1, 0, d->stream>>>(d->map_slots.p + cap);
  B2D_CU(d->map_size.reserve(1));
  B2D_CU(cudaMemsetAsync(d->map_size.p, 0, sizeof(unsigned long long), d->stream));
  d->map_size_host = 0;
  return B2D_OK;
}

uint64_t pow2_at_least(uint64_t x) {
  uint64_t c = 1024;
  while (c < x) c <<= 1;
  return c;
}

// capacity policy: the reference rehashes when capacity < size + num_nodes (:1622-1623); here
// the table keeps load <= map_max_load (default 0.75) with that reservation and grows to half
// of it
int map_ensure(b2d_dedup* d) {
  const uint64_t need = d->map_size_host + d->N;
  if (d->map_slots.p && (double)need <= d->map_max_load * (double)d->map_cap) return B2D_OK;
  const uint64_t cap = pow2_at_least((uint64_t)((double)need / (0.5 * d->map_max_load)) + 1);
  if (!d->map_slots.p || d->map_size_host == 0) return map_reset(d, cap);
  DevBuf<MapSlot> fresh;
  B2D_CU(fresh.reserve(cap + 1));
  B2D_CU(cudaMemsetAsync(fresh.p, 0xff, sizeof(MapSlot) * (cap + 1), d->stream));
  map_special_init_kernel<<<1, 1, 0, d->stream>>>(fresh.p + cap);
  DevBuf<unsigned long long> cnt;
  B2D_CU(cnt.reserve(1));
  B2D_CU(cudaMemsetAsync(cnt.p, 0, sizeof(unsigned long long), d->stream));
  MapView from, to;
  map_view(d, from);
  to.slots = fresh.p; to.cap = cap; to.mask = cap - 1; to.size = cnt.p;
  map_rehash_kernel<<<(unsigned)d->sm_count * 8u, 256, 0, d->stream>>>(from, to, &d->state.p->status);
  B2D_CU(cudaGetLastError());
  B2D_CU(cudaStreamSynchronize(d->stream));
  std::swap(d->map_slots.p, fresh.p);
  std::swap(d->map_slots.n, fresh.n);
  std::swap(d->map_size.p, cnt.p);
  std::swap(d->map_size.n, cnt.n);
  d->map_cap = cap;
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

double secs(std::chrono::high_resolution_clock::time_point a, std::chrono::high_resolution_clock::time_point b) {
  return std::chrono::duration<double>(b - a).count();
}

int do_checkpoint(b2d_dedup* d, const void* d_data, uint64_t len, bool make_baseline, bool advance) {
  using clk = std::chrono::high_resolution_clock;
  const auto t0 = clk::now();
  if (!d_data || len == 0) return B2D_ERR_ARG;
  uint64_t nc = (len + d->chunk_size - 1) / d->chunk_size;
  if (nc > 0x7fffffffull) return B2D_ERR_ARG;
  const bool baseline = (d->current_id == 0) || make_baseline;
  if (!baseline && (!d->have_tree || nc != d->n)) return B2D_ERR_LEN_CHANGED;
  if (d->current_id + 1u > MAX_BUCKETS) return B2D_ERR_UNSUPPORTED;   // source-checkpoint buckets
  d->diff_valid = false;
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
  if (d->push.n < d->N + 16ull || !d->push.p) {
    // flags stay all-zero between checkpoints (the compaction clears what it reads)
    B2D_CU(d->push.reserve(((uint64_t)d->N + 15ull) / 16ull * 16ull + 16ull));
    B2D_CU(cudaMemsetAsync(d->push.p, 0, d->push.n, d->stream));
  }
  if (baseline) {
    int rc = map_reset(d, pow2_at_least((uint64_t)((double)d->N / (0.5 * d->map_max_load)) + 1));
    if (rc) return rc;
    d->have_tree = true;
    d->baseline_id = d->current_id;
  } else {
    int rc = map_ensure(d);
    if (rc) return rc;
  }
  const uint32_t B = d->current_id + 1u;
  B2D_CU(d->first_list.reserve(d->n));
  B2D_CU(d->shift_list.reserve(d->n));
  B2D_CU(d->tmp_first.reserve(d->n));
  B2D_CU(d->tmp_shift.reserve(d->n));
  B2D_CU(d->levels.reserve(68));
  B2D_CU(d->region_off.reserve(d->n));
  B2D_CU(d->sprev.reserve(d->n));
  B2D_CU(d->skey.reserve(d->n));
  B2D_CU(d->hist.reserve(B < 64 ? 64 : B));
  B2D_CU(d->bucket_start.reserve(B < 64 ? 64 : B));
  B2D_CU(d->partial.reserve((size_t)1184 * (B < 64 ? 64 : B)));
  B2D_CU(d->partial2.reserve(2 * SCAN_GRID));
  B2D_CU(d->diff.reserve(64 + 16ull * d->n + (uint64_t)d->n * d->chunk_size));
  B2D_CU(d->state.reserve(1));
  B2D_CU(d->state_h.reserve(1));
  B2D_CU(cudaMemsetAsync(d->state.p, 0, sizeof(DevState), d->stream));
  MapView m;
  map_view(d, m);
  DevState* ds = d->state.p;
  const auto t1 = clk::now();
  d->timers[0] = secs(t0, t1);
  d->launches = 0;

  B2D_CU(cudaEventRecord(d->ev[0], d->stream));
  // dedup_data_baseline (:13-259) / dedup_data (:261-509)
  LeafArgs la{static_cast<const uint8_t*>(d_data), len, d->chunk_size, d->n, d->kind, baseline ? 1 : 0,
              d->current_id, d->tree.p, d->leaflab.p, d->dupflag.p, m, &ds->status};
  const int leaf_path = launch_leaves(la, d->sm_count, d->tune, d->stream);
  if (leaf_path < 0) return B2D_ERR_CUDA;
  d->leaf_tma = leaf_path == 1;
  d->launches += 1;
  B2D_CU(cudaEventRecord(d->ev[3], d->stream));
  ForestArgs fa{d->tree.p, d->lab.p, d->leaflab.p, d->push.p, m, &ds->status, &ds->zero_exists, d->dupflag.p,
                d->n, d->N, d->D, d->current_id, d->kind, baseline ? 1 : 0};
  B2D_CU(launch_forest(fa, 1, d->stream));
  if (baseline) {
    B2D_CU(launch_zero_exists(m, &ds->zero_exists, d->stream));
    d->launches += 1;
  }
  B2D_CU(launch_forest(fa, 2, d->stream));
  if (baseline) {
    B2D_CU(launch_baseline_inserts(fa, d->sm_count, d->stream));
    d->launches += 1;
  }
  d->launches += 2 * forest_launch_count(d->D);
  B2D_CU(cudaEventRecord(d->ev[1], d->stream));
  // collect_diff (:511-710)
  DiffArgs ga{static_cast<const uint8_t*>(d_data), len, d->chunk_size, d->n, d->N, d->D, d->current_id,
              d->baseline_id, d->tree.p, d->push.p, m, &ds->status, &ds->meta, d->first_list.p,
              d->shift_list.p, d->tmp_first.p, d->tmp_shift.p, d->levels.p, d->region_off.p, d->sprev.p, d->skey.p, d->hist.p, d->bucket_start.p,
              d->partial.p, d->partial2.p, d->diff.p};
  B2D_CU(launch_collect_diff(ga, d->sm_count, d->stream));
  d->launches += 14;
  B2D_CU(cudaEventRecord(d->ev[2], d->stream));
  B2D_CU(cudaMemcpyAsync(d->state_h.p, d->state.p, sizeof(DevState), cudaMemcpyDeviceToHost, d->stream));
  B2D_CU(cudaStreamSynchronize(d->stream));
  const DevState& st = *d->state_h.p;
  float ms_dedup = 0, ms_gather = 0, ms_leaf = 0;
  cudaEventElapsedTime(&ms_dedup, d->ev[0], d->ev[1]);
  cudaEventElapsedTime(&ms_gather, d->ev[1], d->ev[2]);
  cudaEventElapsedTime(&ms_leaf, d->ev[0], d->ev[3]);
  d->phase[0] = ms_leaf * 1e-3;
  d->phase[1] = (ms_dedup - ms_leaf) * 1e-3;
  d->phase[2] = ms_gather * 1e-3;
  d->timers[1] = ms_dedup * 1e-3;
  d->timers[2] = ms_gather * 1e-3;
  d->timers[3] = 0;
  int rc = status_code(st.status);
  d->map_size_host = st.meta.map_size;
  if (rc) {
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
  if (advance) d->current_id += 1;
  return B2D_OK;
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
  B2D_CU(d->diff_h.reserve(d->diff_len));
  rc = copy_diff(d, d->diff_h.p, d->diff_h.n);
  if (rc) return rc;
  if (diff) *diff = d->diff_h.p;
  if (diff_len) *diff_len = d->diff_len;
  return B2D_OK;
}

// write_chkpt_log (:1853-1896) with write_metadata_breakdown (src/utils.cpp:38-124); the
// checkpoint id written is the one just taken (logs are written before current_id += 1)
int write_chkpt_log(b2d_dedup* d, const uint8_t* diff, uint64_t diff_len, const std::string& logname, uint32_t id) {
  if (diff_len < 32) return B2D_ERR_FORMAT;
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
  fprintf(result, "Tree,%u,%u,%llu,%llu,%llu,%llu,%s,%s,%s,%s\n", id, d->chunk_size,
          (unsigned long long)d->data_len, (unsigned long long)(d->datasizes[0] + d->datasizes[1]),
          (unsigned long long)d->datasizes[0], (unsigned long long)d->datasizes[1], g(d->timers[0]).c_str(),
          g(d->timers[1]).c_str(), g(d->timers[2]).c_str(), g(d->timers[3]).c_str());
  fprintf(timing, "Tree,%u,%u,%s,%s,%s\n", id, d->chunk_size, g(d->timers[1]).c_str(), g(d->timers[2]).c_str(),
          g(d->timers[3]).c_str());
  fprintf(size, "Tree,%u,%u,%llu,%llu,", id, d->chunk_size, (unsigned long long)d->datasizes[0],
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
        const uint64_t off = 32 + 4ull * nf + 8ull * i + 4;
        if (off + 4 <= diff_len) memcpy(&num, diff + off, 4);
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
  fprintf(f, "Tree,%u,%u,%g,%g\n", id, d->chunk_size, d->restart_timers[0], d->restart_timers[1]);
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
               uint32_t count, uint32_t id) {
  using clk = std::chrono::high_resolution_clock;
  const auto t0 = clk::now();
  if (!d_out || !diffs || !sizes || id >= count) return B2D_ERR_ARG;
  HostHdr h;
  if (!parse_hdr(diffs[id], sizes[id], h)) return B2D_ERR_FORMAT;
  if (len < h.datalen) return B2D_ERR_ARG;
  uint64_t nc = (h.datalen + h.cs - 1) / h.cs;
  if (nc > 0x7fffffffull) return B2D_ERR_FORMAT;
  const uint32_t n = (uint32_t)nc, N = 2u * n - 1u;
  // scratch sized for the whole chain
  uint64_t max_size = 0, max_list = 0, max_ids = 0;
  {
    uint32_t ref = h.ref_id;
    for (int idx = (int)id; idx >= 0 && idx >= (int)ref; idx--) {
      HostHdr hh;
      if (!parse_hdr(diffs[idx], sizes[idx], hh)) return B2D_ERR_FORMAT;
      if (idx != (int)id) ref = hh.ref_id;
      max_size = std::max<uint64_t>(max_size, sizes[idx]);
      max_list = std::max<uint64_t>(max_list, std::max<uint64_t>(hh.F, hh.S));
      max_ids = std::max<uint64_t>(max_ids, (uint64_t)hh.chkpt_id + 1);
    }
  }
  B2D_CU(d->r_node_list.reserve(n));
  B2D_CU(d->r_rep.reserve(n));
  B2D_CU(d->r_dist.reserve(n));
  B2D_CU(d->r_offs.reserve(max_list));
  B2D_CU(d->r_partial.reserve(SCAN_GRID));
  B2D_CU(d->r_cum.reserve(max_ids));
  B2D_CU(d->r_total.reserve(1));
  B2D_CU(d->r_diff.reserve(max_size + 16));
  B2D_CU(d->state.reserve(1));
  B2D_CU(d->state_h.reserve(1));
  B2D_CU(d->r_stage.reserve(max_size + 16 + 8 * max_ids));
  B2D_CU(cudaMemsetAsync(d->state.p, 0, sizeof(DevState), d->stream));
  d->launches = 0;
  double copy_time = 0;

  RestartArgs a{};
  a.n = n;
  a.N = N;
  a.out = static_cast<uint8_t*>(d_out);
  a.out_len = h.datalen;
  a.node_list = d->r_node_list.p;
  a.dist = d->r_dist.p;
  a.rep = d->r_rep.p;
  a.offs = d->r_offs.p;
  a.partial = d->r_partial.p;
  a.total = d->r_total.p;
  a.st = &d->state.p->status;
  B2D_CU(launch_restart_init(a, d->sm_count, d->stream));

  uint32_t ref = h.ref_id;
  for (int idx = (int)id; idx >= 0 && idx >= (int)ref; idx--) {
    HostHdr hh;
    parse_hdr(diffs[idx], sizes[idx], hh);
    if (idx != (int)id) ref = hh.ref_id;
    // stage the diff (plus its repeat-table running counts) in pinned memory, then one copy
    const uint32_t delta = (uint32_t)((16u - (hh.data_off & 15u)) & 15u);
    const uint64_t ncum = (uint64_t)hh.chkpt_id + 1;
    B2D_CU(cudaStreamSynchronize(d->stream));   // the staging buffer is reused per diff
    uint8_t* stage = d->r_stage.p;
    const auto c0 = clk::now();
    memcpy(stage + delta, diffs[idx], sizes[idx]);
    std::vector<unsigned long long> cum(ncum, 0ull);
    bool bad_row = false;
    for (uint32_t i = 0; i < hh.P; i++) {
      uint32_t ck, cnt;
      memcpy(&ck, diffs[idx] + hh.count_off + 8ull * i, 4);
      memcpy(&cnt, diffs[idx] + hh.count_off + 8ull * i + 4, 4);
      if (ck < ncum) cum[ck] = cnt; else bad_row = true;
    }
    for (uint64_t t = 1; t < ncum; t++) cum[t] += cum[t - 1];
    B2D_CU(cudaMemcpyAsync(d->r_diff.p, stage, sizes[idx] + delta, cudaMemcpyHostToDevice, d->stream));
    B2D_CU(cudaMemcpyAsync(d->r_cum.p, cum.data(), sizeof(unsigned long long) * ncum, cudaMemcpyHostToDevice,
                           d->stream));
    if (idx == (int)id) {
      B2D_CU(cudaStreamSynchronize(d->stream));
      copy_time = secs(c0, clk::now());
    }
    a.diff = d->r_diff.p + delta;
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
    a.is_main = idx == (int)id;
    a.cum = d->r_cum.p;
    a.ncum = (uint32_t)ncum;
    B2D_CU(launch_restart_diff(a, &d->state.p->straddle, d->sm_count, d->stream));
    d->launches += 9 + (straddle_query(n).count ? 2 : 0);
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
    rc = write_chkpt_log(d, p, n, logname, d->current_id);
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
    rc = write_chkpt_log(d, p, n, logname, d->current_id);
    if (rc) return rc;
    FILE* f = fopen(filename, "wb");
    if (!f) return B2D_ERR_IO;
    const size_t w = fwrite(p, 1, n, f);
    const int cl = fclose(f);
    if (w != n || cl != 0) return B2D_ERR_IO;
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
  else if (k == "map_max_load_pct" && value >= 10 && value <= 90) d->map_max_load = value / 100.0;
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

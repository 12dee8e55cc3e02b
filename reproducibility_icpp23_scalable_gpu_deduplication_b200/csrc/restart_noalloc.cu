// Restart that allocates nothing.
//
// Some callers of this library cannot call cudaMalloc: a process restoring a checkpoint after
// the device ran out of memory (the moment a restart is most needed, an allocation is the
// thing most likely to fail), or a runtime that owns all device memory through its own pool
// and budget and forbids side allocations.  b2d_restart_noalloc serves them: the diffs and
// the output buffer are the caller's device memory, and the restart's scratch (per-chunk
// NodeID list, data offsets, shifted-chunk sources, region offsets, scan partials) lives in
// one file-scope __device__ array of fixed size, created with the module and held by every
// GPU that loads the library until the process exits.
//
// Limits: at most NOALLOC_MAX_CHUNKS chunks per checkpoint and checkpoint ids below
// NOALLOC_MAX_IDS; larger restarts are rejected with B2D_ERR_UNSUPPORTED.
//
// Every call looks up the array's device address (cudaGetSymbolAddress) with the caller's
// device current: the address is not cached, because a cudaDeviceReset unloads the module and
// the array can come back elsewhere.  The first call on a device should come before any stream
// capture.  Every call shares the one array and leaves its contents behind; each call clears
// what must start at zero.  Calls that overlap on the GPU (on different streams, or from
// different host threads) race on the array and must be serialised by the caller.
#include <cuda_runtime.h>

#include <cstring>

#include "../../include/b200dedup.h"
#include "restart.cuh"

namespace b2d {

constexpr uint64_t NOALLOC_MAX_CHUNKS = 1ull << 18;
constexpr uint64_t NOALLOC_MAX_IDS = 4096;

constexpr size_t na_align(size_t x) { return (x + 255) & ~size_t(255); }
constexpr size_t NA_NODE_LIST = 0;
constexpr size_t NA_MFLAG = na_align(NA_NODE_LIST + sizeof(uint2) * NOALLOC_MAX_CHUNKS);
constexpr size_t NA_DIST = na_align(NA_MFLAG + NOALLOC_MAX_CHUNKS);
constexpr size_t NA_REP = na_align(NA_DIST + sizeof(uint32_t) * NOALLOC_MAX_CHUNKS);
constexpr size_t NA_FLAG = na_align(NA_REP + sizeof(uint2) * NOALLOC_MAX_CHUNKS);
constexpr size_t NA_OFFS = na_align(NA_FLAG + NOALLOC_MAX_CHUNKS);   // offsets, starts, sources, trees
constexpr size_t NA_CUM = na_align(NA_OFFS + 4 * sizeof(uint32_t) * NOALLOC_MAX_CHUNKS);
constexpr size_t NA_PARTIAL = na_align(NA_CUM + sizeof(unsigned long long) * NOALLOC_MAX_IDS);
constexpr size_t NA_TOTAL = na_align(NA_PARTIAL + sizeof(uint32_t) * SCAN_GRID);
constexpr size_t NA_STATUS = na_align(NA_TOTAL + sizeof(unsigned long long));
constexpr size_t NA_STRADDLE = na_align(NA_STATUS + sizeof(DevStatus));
constexpr size_t NA_BYTES = na_align(NA_STRADDLE + sizeof(StraddleInfo));   // 9,996,288 bytes (about 10.0 MB)

static __device__ __align__(256) unsigned char g_restart_scratch[NA_BYTES];

namespace {

// device address of the scratch array on the current device (host code cannot use the symbol
// itself: in host code it names a host-side stand-in)
int scratch_for_current_device(unsigned char** out) {
  void* p = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&p, g_restart_scratch);
  if (e != cudaSuccess || p == nullptr) return B2D_ERR_CUDA;
  *out = static_cast<unsigned char*>(p);
  return B2D_OK;
}

struct NaHdr {
  uint32_t ref_id, chkpt_id;
  uint64_t datalen;
  uint32_t cs, F, P, S;
  uint64_t first_off, count_off, shift_off, data_off;
};

// header of a device-resident diff, read into host stack memory
int read_hdr(const void* d_diff, uint64_t size, cudaStream_t s, NaHdr& h) {
  if (!d_diff || size < 32) return B2D_ERR_FORMAT;
  uint32_t w[8];
  if (cudaMemcpyAsync(w, d_diff, 32, cudaMemcpyDeviceToHost, s) != cudaSuccess) return B2D_ERR_CUDA;
  if (cudaStreamSynchronize(s) != cudaSuccess) return B2D_ERR_CUDA;
  h.ref_id = w[0];
  h.chkpt_id = w[1];
  h.datalen = (uint64_t)w[2] | ((uint64_t)w[3] << 32);
  h.cs = w[4];
  h.F = w[5];
  h.P = w[6];
  h.S = w[7];
  h.first_off = 32;
  h.count_off = h.first_off + 4ull * h.F;
  h.shift_off = h.count_off + 8ull * h.P;
  h.data_off = h.shift_off + 8ull * h.S;
  if (h.data_off > size || h.cs == 0 || h.datalen == 0) return B2D_ERR_FORMAT;
  return B2D_OK;
}

}  // namespace
}  // namespace b2d

using namespace b2d;

extern "C" int b2d_restart_noalloc(void* d_out, uint64_t len, const void* const* d_diffs, const uint64_t* sizes,
                                   uint32_t num_diffs, uint32_t chkpt_id, void* cuda_stream) {
  if (!d_out || !d_diffs || !sizes || chkpt_id >= num_diffs) return B2D_ERR_ARG;
  cudaStream_t s = static_cast<cudaStream_t>(cuda_stream);
  unsigned char* base = nullptr;
  int rc = scratch_for_current_device(&base);
  if (rc) return rc;
  NaHdr h;
  if ((rc = read_hdr(d_diffs[chkpt_id], sizes[chkpt_id], s, h))) return rc;
  // diffs[i] must be checkpoint i, whose baseline is not after it (as b2d_restart checks)
  if (h.ref_id > h.chkpt_id || h.chkpt_id != chkpt_id) return B2D_ERR_FORMAT;
  if (len < h.datalen) return B2D_ERR_ARG;
  const uint64_t nc = (h.datalen + h.cs - 1) / h.cs;
  if (nc > NOALLOC_MAX_CHUNKS) return B2D_ERR_UNSUPPORTED;
  const uint32_t n = (uint32_t)nc, N = 2u * n - 1u;
  // every header of the chain is checked before the first launch, so a rejected call leaves
  // the output buffer untouched
  {
    uint32_t ref = h.ref_id;
    for (int idx = (int)chkpt_id; idx >= 0 && idx >= (int)ref; idx--) {
      NaHdr hh;
      if ((rc = read_hdr(d_diffs[idx], sizes[idx], s, hh))) return rc;
      if (idx != (int)chkpt_id) ref = hh.ref_id;
      if (hh.F > NOALLOC_MAX_CHUNKS || hh.S > NOALLOC_MAX_CHUNKS || (uint64_t)hh.chkpt_id + 1 > NOALLOC_MAX_IDS)
        return B2D_ERR_UNSUPPORTED;
    }
  }
  int dev = 0, sm_count = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sm_count, cudaDevAttrMultiProcessorCount, dev);

  RestartArgs a{};
  a.n = n;
  a.N = N;
  a.out = static_cast<uint8_t*>(d_out);
  a.out_len = h.datalen;
  a.node_list = reinterpret_cast<uint2*>(base + NA_NODE_LIST);
  a.mflag = base + NA_MFLAG;
  a.slot.dist = reinterpret_cast<uint32_t*>(base + NA_DIST);
  a.slot.rep = reinterpret_cast<uint2*>(base + NA_REP);
  a.slot.flag = base + NA_FLAG;
  a.offs = reinterpret_cast<uint32_t*>(base + NA_OFFS);
  a.rstart = a.offs + NOALLOC_MAX_CHUNKS;
  a.pstart = a.offs + 2 * NOALLOC_MAX_CHUNKS;
  a.rtree = a.offs + 3 * NOALLOC_MAX_CHUNKS;
  a.cum = reinterpret_cast<unsigned long long*>(base + NA_CUM);
  a.partial = reinterpret_cast<uint32_t*>(base + NA_PARTIAL);
  a.total = reinterpret_cast<unsigned long long*>(base + NA_TOTAL);
  a.st = reinterpret_cast<DevStatus*>(base + NA_STATUS);
  StraddleInfo* sd = reinterpret_cast<StraddleInfo*>(base + NA_STRADDLE);
  if (cudaMemsetAsync(a.st, 0, sizeof(DevStatus), s) != cudaSuccess) return B2D_ERR_CUDA;
  // older diffs go through the one slot: each is expanded, then walked on its own
  RestartWalk w{};
  w.main_cur = h.chkpt_id;
  w.n = n;
  w.N = N;
  w.out = a.out;
  w.out_len = h.datalen;
  w.node_list = a.node_list;
  w.mflag = a.mflag;
  w.st = a.st;

  uint32_t ref = h.ref_id;
  for (int idx = (int)chkpt_id; idx >= 0 && idx >= (int)ref; idx--) {
    NaHdr hh;
    if ((rc = read_hdr(d_diffs[idx], sizes[idx], s, hh))) return rc;
    if (idx != (int)chkpt_id) ref = hh.ref_id;
    if (hh.F > NOALLOC_MAX_CHUNKS || hh.S > NOALLOC_MAX_CHUNKS || (uint64_t)hh.chkpt_id + 1 > NOALLOC_MAX_IDS)
      return B2D_ERR_UNSUPPORTED;
    a.diff = static_cast<const uint8_t*>(d_diffs[idx]);
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
    a.is_main = idx == (int)chkpt_id;
    a.ncum = hh.chkpt_id + 1u;
    if (launch_restart_cum(a, s) != cudaSuccess) return B2D_ERR_CUDA;
    if (launch_restart_diff(a, sd, sm_count, s) != cudaSuccess) return B2D_ERR_CUDA;
    if (!a.is_main) {
      w.count = 1;
      w.cs = hh.cs;
      w.data[0] = a.diff + hh.data_off;
      w.data_len[0] = sizes[idx] - hh.data_off;
      w.datalen[0] = hh.datalen;
      w.cur[0] = hh.chkpt_id;
      w.slot[0] = a.slot;
      w.last = idx - 1 < 0 || idx - 1 < (int)ref;
      if (launch_restart_walk(w, sm_count, s) != cudaSuccess) return B2D_ERR_CUDA;
      w.dense = 1;
    }
  }
  DevStatus st;
  if (cudaMemcpyAsync(&st, a.st, sizeof(DevStatus), cudaMemcpyDeviceToHost, s) != cudaSuccess) return B2D_ERR_CUDA;
  if (cudaStreamSynchronize(s) != cudaSuccess) return B2D_ERR_CUDA;
  switch (st.error) {
    case DERR_NONE: return B2D_OK;
    case DERR_RESTART_RANGE: return B2D_ERR_RESTART_RANGE;
    default: return B2D_ERR_INTERNAL;
  }
}

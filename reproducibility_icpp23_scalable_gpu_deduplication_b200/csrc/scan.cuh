// Block-level scan helpers for the reduce-then-scan passes (no cross-CTA waiting: every
// multi-CTA scan here is three launches -- per-CTA reduce, one-CTA scan of the partials,
// per-CTA rescan + scatter -- so no kernel ever spins on another CTA).
#pragma once
#include "common.cuh"

namespace b2d {

__device__ __forceinline__ uint32_t warp_incl_scan(uint32_t v) {
  const uint32_t lane = threadIdx.x & 31u;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t t = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= (uint32_t)o) v += t;
  }
  return v;
}

// Exclusive block scan of one u32 per thread; returns the exclusive prefix, *total gets the
// block sum.  `sh` needs blockDim.x/32 + 1 words.  All threads must call it.
__device__ __forceinline__ uint32_t block_excl_scan(uint32_t v, uint32_t* sh, uint32_t* total) {
  const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5, nw = (blockDim.x + 31u) >> 5;
  const uint32_t inc = warp_incl_scan(v);
  if (lane == 31u) sh[warp] = inc;
  __syncthreads();
  if (warp == 0) {
    uint32_t s = lane < nw ? sh[lane] : 0u;
    s = warp_incl_scan(s);
    if (lane < nw) sh[lane] = s;   // inclusive per-warp sums
  }
  __syncthreads();
  const uint32_t warp_base = warp == 0 ? 0u : sh[warp - 1];
  const uint32_t tot = sh[nw - 1];
  __syncthreads();
  *total = tot;
  return warp_base + inc - v;
}

__device__ __forceinline__ uint32_t block_reduce_sum(uint32_t v, uint32_t* sh) {
  uint32_t tot;
  block_excl_scan(v, sh, &tot);
  return tot;
}

// contiguous range [beg, end) of `count` items owned by CTA b out of g
__device__ __forceinline__ void cta_range(uint64_t count, uint32_t b, uint32_t g, uint64_t& beg, uint64_t& end) {
  const uint64_t per = (count + g - 1) / g;
  beg = per * b;
  end = beg + per;
  if (beg > count) beg = count;
  if (end > count) end = count;
}

}  // namespace b2d

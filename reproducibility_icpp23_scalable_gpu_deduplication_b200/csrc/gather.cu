// Diff assembly on the device: the reference's collect_diff (src/tree_approach.cpp:511-710).
//
// Output order is the reference's sequential order (what its atomics produce with one
// thread): region roots by (level descending, node ascending); the repeat table by
// checkpoint id; shifted-duplicate entries stably bucketed by source checkpoint.
//   1. compaction of the push flags in that canonical order (reduce-then-scan, 3 launches)
//   2. first-occurrence region sizes -> exclusive chunk offsets (3 launches)
//   3. shift entries: source NodeID lookup + per-CTA histograms (1 launch)
//   4. layout: bucket starts, repeat table, header, byte offsets (1 launch, 1 CTA)
//   5. stable bucket scatter of the shift entries (1 launch, one warp per range)
//   6. first-occurrence metadata + 16-byte vectorised chunk gather (1 launch)
// Diff layout (include/utils.hpp:29-37, src/tree_approach.cpp:777-780):
//   [header 32 B][u32 first node x F][(u32 ckpt, u32 count) x P][(u32 node, u32 prev) x S][data]
// It is placed `delta` bytes into the device buffer so the data section is 16-byte aligned.
#include "dedup_kernels.cuh"
#include "map.cuh"
#include "scan.cuh"

namespace b2d {

constexpr uint32_t COMPACT_THREADS = 512;

// Every kernel below is a body over a virtual grid (bid of nb CTAs) with two launchers: one
// handle's launch (the CUDA grid) and a segmented launch over many handles' diff assembly in
// one grid, where CTA b belongs to the handle h with beg[h] <= b < beg[h+1] (batched form).
__device__ __forceinline__ uint32_t seg_locate(const SegGrid& s, uint32_t& bid, uint32_t& nb) {
  uint32_t lo = 0, hi = s.n;
  while (hi - lo > 1) {
    const uint32_t mid = (lo + hi) >> 1;
    if (s.beg[mid] <= blockIdx.x) lo = mid; else hi = mid;
  }
  bid = blockIdx.x - s.beg[lo];
  nb = s.beg[lo + 1] - s.beg[lo];
  return lo;
}
constexpr uint32_t SHIFT_GRID = 296;    // at most 2 x 148 ranges for the shift-entry passes

// Region roots are flagged in `push`: 2 bits per node (PUSH_FIRST = 1, PUSH_SHIFT = 2), 16 nodes
// per 32-bit word, zero-padded to a multiple of 64 nodes, all-zero between checkpoints (a quarter
// of the bytes of one flag byte per node, so the two passes below read 16 MB instead of 64 MB
// for a 2^26-node tree).  Compaction runs in node order with 16-byte loads of 64 nodes; since the
// canonical order is "level descending, node ascending" and node order is "level ascending,
// node ascending", the canonical list is the node-order list with its per-level runs reversed,
// which compact_permute_kernel applies after a per-level split of the node-order lists.
constexpr uint32_t PUSH_GROUP = 64;   // nodes per 16-byte load
__device__ __forceinline__ uint4 ld_push16(const uint8_t* push, uint64_t g) {
  return reinterpret_cast<const uint4*>(push)[g];
}
// one bit (the low bit of each 2-bit field) per node flagged first / shifted
__device__ __forceinline__ uint32_t push_first_bits(uint32_t w) { return w & ~(w >> 1) & 0x55555555u; }
__device__ __forceinline__ uint32_t push_shift_bits(uint32_t w) { return (w >> 1) & ~w & 0x55555555u; }
__device__ __forceinline__ void count64(uint4 v, uint32_t& cf, uint32_t& cs) {
  cf += __popc(push_first_bits(v.x)) + __popc(push_first_bits(v.y)) + __popc(push_first_bits(v.z)) +
        __popc(push_first_bits(v.w));
  cs += __popc(push_shift_bits(v.x)) + __popc(push_shift_bits(v.y)) + __popc(push_shift_bits(v.z)) +
        __popc(push_shift_bits(v.w));
}

__device__ __forceinline__ void compact_count_body(const DiffArgs& a, uint32_t bid, uint32_t nb) {
  __shared__ uint32_t sh[COMPACT_THREADS / 32 + 1];
  const uint64_t groups = ((uint64_t)a.N + PUSH_GROUP - 1u) / PUSH_GROUP;
  uint64_t beg, end;
  cta_range(groups, bid, nb, beg, end);
  uint32_t cf = 0, cs = 0;
  // two independent loads per thread per iteration
  for (uint64_t g = beg + threadIdx.x; g < end; g += 2ull * blockDim.x) {
    const uint4 v0 = ld_push16(a.push, g);
    const uint4 v1 = g + blockDim.x < end ? ld_push16(a.push, g + blockDim.x) : make_uint4(0, 0, 0, 0);
    if (v0.x | v0.y | v0.z | v0.w) count64(v0, cf, cs);
    if (v1.x | v1.y | v1.z | v1.w) count64(v1, cf, cs);
  }
  const uint32_t tf = block_reduce_sum(cf, sh);
  const uint32_t ts = block_reduce_sum(cs, sh);
  if (threadIdx.x == 0) {
    a.partial2[2 * bid] = tf;
    a.partial2[2 * bid + 1] = ts;
  }
}
__global__ void __launch_bounds__(COMPACT_THREADS) compact_count_kernel(DiffArgs a0) {
  griddep_enter();
  compact_count_body(with_round(a0), blockIdx.x, gridDim.x);
}
__global__ void __launch_bounds__(COMPACT_THREADS) compact_count_seg(SegGrid s) {
  uint32_t bid, nb;
  const uint32_t h = seg_locate(s, bid, nb);
  compact_count_body(with_round(s.args[h]), bid, nb);
}

__device__ __forceinline__ void compact_scan_body(const DiffArgs& a, uint32_t bid, uint32_t nb, uint32_t g) {
  __shared__ uint32_t sh[33];
  uint32_t tf, ts;
  const uint32_t i = threadIdx.x;
  const uint32_t vf = i < g ? a.partial2[2 * i] : 0u, vs = i < g ? a.partial2[2 * i + 1] : 0u;
  const uint32_t ef = block_excl_scan(vf, sh, &tf);
  const uint32_t es = block_excl_scan(vs, sh, &ts);
  if (i < g) {
    a.partial2[2 * i] = ef;
    a.partial2[2 * i + 1] = es;
  }
  if (i == 0) {
    a.meta->F = tf;
    a.meta->S = ts;
  }
}
__global__ void __launch_bounds__(1024) compact_scan_kernel(DiffArgs a0, uint32_t g, uint32_t bcap) {
  griddep_enter();
  compact_scan_body(with_round(a0), blockIdx.x, gridDim.x, g);
  // the per-checkpoint bucket counts start at zero
  for (uint32_t t = threadIdx.x; t < bcap; t += blockDim.x) a0.hist[t] = 0u;
}
__global__ void __launch_bounds__(1024) compact_scan_seg(SegGrid s) {
  uint32_t bid, nb;
  const uint32_t h = seg_locate(s, bid, nb);
  compact_scan_body(with_round(s.args[h]), bid, nb, s.g[h]);
  // the per-checkpoint bucket counts start at zero (the single-handle path memsets them)
  for (uint32_t t = threadIdx.x; t < s.bcap[h]; t += blockDim.x) s.args[h].hist[t] = 0u;
}

// node-order lists of first / shift roots; clears the flags it consumed.  Each thread owns one
// 64-node group of a tile, so one block scan covers COMPACT_THREADS * 64 = 32768 nodes, which
// keeps both 16-bit halves of the packed counts exact.
__device__ __forceinline__ void compact_write_body(const DiffArgs& a, uint32_t bid, uint32_t nb) {
  __shared__ uint32_t sh[COMPACT_THREADS / 32 + 1];
  const uint64_t groups = ((uint64_t)a.N + PUSH_GROUP - 1u) / PUSH_GROUP;
  uint64_t beg, end;
  cta_range(groups, bid, nb, beg, end);
  uint32_t bf = a.partial2[2 * bid], bs = a.partial2[2 * bid + 1];
  for (uint64_t t0 = beg; t0 < end; t0 += COMPACT_THREADS) {
    const uint64_t g = t0 + threadIdx.x;
    const uint4 v = g < end ? ld_push16(a.push, g) : make_uint4(0, 0, 0, 0);
    const bool nz = (v.x | v.y | v.z | v.w) != 0u;
    uint32_t cf = 0, cs = 0;
    if (nz) count64(v, cf, cs);
    uint32_t tot;
    const uint32_t ex = block_excl_scan((cf << 16) | cs, sh, &tot);
    if (nz) {
      uint32_t of = bf + (ex >> 16), os = bs + (ex & 0xffffu);
      const uint32_t w[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
      for (int k = 0; k < 4; k++) {
        const uint32_t base = (uint32_t)(PUSH_GROUP * g) + 16u * k;
        for (uint32_t m = push_first_bits(w[k]); m; m &= m - 1u) a.tmp_first[of++] = base + ((__ffs(m) - 1u) >> 1);
        for (uint32_t m = push_shift_bits(w[k]); m; m &= m - 1u) a.tmp_shift[os++] = base + ((__ffs(m) - 1u) >> 1);
      }
      reinterpret_cast<uint4*>(a.push)[g] = make_uint4(0, 0, 0, 0);
    }
    bf += tot >> 16;
    bs += tot & 0xffffu;
  }
}
__global__ void __launch_bounds__(COMPACT_THREADS) compact_write_kernel(DiffArgs a0) {
  griddep_enter();
  compact_write_body(with_round(a0), blockIdx.x, gridDim.x);
}
__global__ void __launch_bounds__(COMPACT_THREADS) compact_write_seg(SegGrid s) {
  uint32_t bid, nb;
  const uint32_t h = seg_locate(s, bid, nb);
  compact_write_body(with_round(s.args[h]), bid, nb);
}

// warp-parallel lower bound: first index of sorted v[0..cnt) with v[idx] >= key (32-ary search)
__device__ __forceinline__ uint32_t warp_lower_bound(const uint32_t* v, uint32_t cnt, uint64_t key) {
  const uint32_t lane = threadIdx.x & 31u;
  uint32_t lo = 0, hi = cnt;
  while (hi - lo > 32u) {
    const uint32_t step = (hi - lo + 31u) / 32u;
    const uint32_t probe = lo + lane * step;
    const bool below = probe < hi && v[probe] < key;
    const uint32_t c = __popc(__ballot_sync(0xffffffffu, below));
    const uint32_t nlo = c ? lo + (c - 1u) * step + 1u : lo;
    const uint32_t nhi = (c < 32u && lo + c * step < hi) ? lo + c * step : hi;
    lo = nlo;
    hi = nhi;
  }
  const bool below = lo + lane < hi && v[lo + lane] < key;
  return lo + __popc(__ballot_sync(0xffffffffu, below));
}

// level runs of the node-order lists: levels[L] = start of level L in tmp_first,
// levels[34 + L] in tmp_shift (L = 0..D+1); one warp per search
__device__ __forceinline__ void compact_levels_body(const DiffArgs& a, uint32_t bid, uint32_t nb) {
  const uint32_t gw = (bid * blockDim.x + threadIdx.x) >> 5;
  const uint32_t L = gw >> 1;
  if (L > a.D + 1u) return;
  const uint64_t key = (1ull << L) - 1ull;   // first node of level L
  if ((gw & 1u) == 0) {
    const uint32_t r = warp_lower_bound(a.tmp_first, a.meta->F, key);
    if ((threadIdx.x & 31u) == 0) a.levels[L] = r;
  } else {
    const uint32_t r = warp_lower_bound(a.tmp_shift, a.meta->S, key);
    if ((threadIdx.x & 31u) == 0) a.levels[34 + L] = r;
  }
}
__global__ void compact_levels_kernel(DiffArgs a0) {
  griddep_enter();
  compact_levels_body(with_round(a0), blockIdx.x, gridDim.x);
}
__global__ void compact_levels_seg(SegGrid s) {
  uint32_t bid, nb;
  const uint32_t h = seg_locate(s, bid, nb);
  compact_levels_body(with_round(s.args[h]), bid, nb);
}

// canonical position of node-order entry i at level L: entries of deeper levels first
__device__ __forceinline__ void compact_permute_body(const DiffArgs& a, uint32_t bid, uint32_t nb) {
  const uint32_t F = a.meta->F, S = a.meta->S;
  const uint64_t tot = (uint64_t)F + S;
  for (uint64_t i = bid * (uint64_t)blockDim.x + threadIdx.x; i < tot; i += (uint64_t)nb * blockDim.x) {
    const bool isf = i < F;
    const uint32_t j = isf ? (uint32_t)i : (uint32_t)(i - F);
    const uint32_t* lv = a.levels + (isf ? 0 : 34);
    const uint32_t cnt = isf ? F : S;
    const uint32_t node = isf ? a.tmp_first[j] : a.tmp_shift[j];
    const uint32_t L = node_level(node);
    // entries at levels deeper than L come first: cnt - (start of level L+1)
    const uint32_t pos = (cnt - lv[L + 1]) + (j - lv[L]);
    if (isf) a.first_list[pos] = node;
    else a.shift_list[pos] = node;
  }
}
__global__ void compact_permute_kernel(DiffArgs a0) {
  griddep_enter();
  compact_permute_body(with_round(a0), blockIdx.x, gridDim.x);
}
__global__ void compact_permute_seg(SegGrid s) {
  uint32_t bid, nb;
  const uint32_t h = seg_locate(s, bid, nb);
  compact_permute_body(with_round(s.args[h]), bid, nb);
}

// ---------------------------------------------------------------- region sizes and offsets
__device__ __forceinline__ void region_count_body(const DiffArgs& a, uint32_t bid, uint32_t nb) {
  __shared__ uint32_t sh[COMPACT_THREADS / 32 + 1];
  uint64_t beg, end;
  cta_range(a.meta->F, bid, nb, beg, end);
  uint32_t c = 0;
  for (uint64_t i = beg + threadIdx.x; i < end; i += blockDim.x) {
    const uint32_t node = a.first_list[i];
    c += num_leaf_descendents(node, a.N);
    // collect_diff keeps a first-occurrence region only when the map names it as the
    // owner of its digest (:548-556); the labelling guarantees it, so check it here
    const uint64_t slot = map_find(a.map, a.tree[node]);
    if (slot > a.map.cap || map_node(a.map, slot) != node || map_tree(a.map, slot) != a.cur)
      set_error(a.st, DERR_INTERNAL, 20);
  }
  const uint32_t t = block_reduce_sum(c, sh);
  if (threadIdx.x == 0) a.partial2[bid] = t;
}
__global__ void __launch_bounds__(COMPACT_THREADS) region_count_kernel(DiffArgs a0) {
  griddep_enter();
  region_count_body(with_round(a0), blockIdx.x, gridDim.x);
}
__global__ void __launch_bounds__(COMPACT_THREADS) region_count_seg(SegGrid s) {
  uint32_t bid, nb;
  const uint32_t h = seg_locate(s, bid, nb);
  region_count_body(with_round(s.args[h]), bid, nb);
}

__device__ __forceinline__ void region_scan_body(const DiffArgs& a, uint32_t bid, uint32_t nb, uint32_t g) {
  __shared__ uint32_t sh[33];
  uint32_t tot;
  const uint32_t i = threadIdx.x;
  const uint32_t v = i < g ? a.partial2[i] : 0u;
  const uint32_t e = block_excl_scan(v, sh, &tot);
  if (i < g) a.partial2[i] = e;
  if (i == 0) a.meta->T = tot;
}
__global__ void __launch_bounds__(1024) region_scan_kernel(DiffArgs a0, uint32_t g) {
  griddep_enter();
  region_scan_body(with_round(a0), blockIdx.x, gridDim.x, g);
}
__global__ void __launch_bounds__(1024) region_scan_seg(SegGrid s) {
  uint32_t bid, nb;
  const uint32_t h = seg_locate(s, bid, nb);
  region_scan_body(with_round(s.args[h]), bid, nb, s.g[h]);
}

__device__ __forceinline__ void region_write_body(const DiffArgs& a, uint32_t bid, uint32_t nb) {
  __shared__ uint32_t sh[COMPACT_THREADS / 32 + 1];
  uint64_t beg, end;
  cta_range(a.meta->F, bid, nb, beg, end);
  uint32_t base = a.partial2[bid];
  for (uint64_t t0 = beg; t0 < end; t0 += blockDim.x) {
    const uint64_t i = t0 + threadIdx.x;
    const uint32_t len = i < end ? num_leaf_descendents(a.first_list[i], a.N) : 0u;
    uint32_t tot;
    const uint32_t e = block_excl_scan(len, sh, &tot);
    if (i < end) a.region_off[i] = base + e;
    base += tot;
  }
}
__global__ void __launch_bounds__(COMPACT_THREADS) region_write_kernel(DiffArgs a0) {
  griddep_enter();
  region_write_body(with_round(a0), blockIdx.x, gridDim.x);
}
__global__ void __launch_bounds__(COMPACT_THREADS) region_write_seg(SegGrid s) {
  uint32_t bid, nb;
  const uint32_t h = seg_locate(s, bid, nb);
  region_write_body(with_round(s.args[h]), bid, nb);
}

// ---------------------------------------------------------------- shifted duplicates
// source NodeID of each entry (:572-580, :672-674) and per-range histograms by checkpoint
__device__ __forceinline__ void shift_prev_body(const DiffArgs& a, uint32_t bid, uint32_t nb, uint32_t bcap) {
  const uint32_t B = a.rs->buckets <= bcap ? a.rs->buckets : bcap;
  extern __shared__ uint32_t hs[];
  uint64_t beg, end;
  cta_range(a.meta->S, bid, nb, beg, end);
  for (uint32_t t = threadIdx.x; t < B; t += blockDim.x) hs[t] = 0;
  __syncthreads();
  for (uint64_t i = beg + threadIdx.x; i < end; i += blockDim.x) {
    const uint32_t node = a.shift_list[i];
    const uint64_t slot = map_find(a.map, a.tree[node]);
    uint32_t pn = 0, pt = 0;
    if (slot <= a.map.cap) {
      pn = map_node(a.map, slot);
      pt = map_tree(a.map, slot);
    } else {
      set_error(a.st, DERR_INTERNAL, 30);
    }
    if (pt >= B) {
      set_error(a.st, DERR_INTERNAL, 31);
      pt = 0;
    }
    a.sprev[i] = pn;
    a.skey[i] = pt;
    atomicAdd(&hs[pt], 1u);
  }
  __syncthreads();
  for (uint32_t t = threadIdx.x; t < B; t += blockDim.x) {
    const uint32_t v = hs[t];
    a.partial[(uint64_t)t * nb + bid] = v;
    if (v) atomicAdd(&a.hist[t], v);
  }
}
__global__ void __launch_bounds__(128) shift_prev_kernel(DiffArgs a0, uint32_t bcap) {
  griddep_enter();
  shift_prev_body(with_round(a0), blockIdx.x, gridDim.x, bcap);
}
__global__ void __launch_bounds__(128) shift_prev_seg(SegGrid s) {
  uint32_t bid, nb;
  const uint32_t h = seg_locate(s, bid, nb);
  shift_prev_body(with_round(s.args[h]), bid, nb, s.bcap[h]);
}

// one CTA: bucket starts, repeat table, per-range scatter bases, header, byte layout
__device__ __forceinline__ void layout_body(const DiffArgs& a, uint32_t bid, uint32_t nb, uint32_t bcap, uint32_t g) {
  const uint32_t B = a.rs->buckets <= bcap ? a.rs->buckets : bcap;
  __shared__ uint32_t sh[33];
  __shared__ uint32_t carry_start, carry_rows;
  if (threadIdx.x == 0) { carry_start = 0; carry_rows = 0; }
  __syncthreads();
  const DevMeta m0 = *a.meta;
  // count P first so the table position is known
  for (uint32_t t0 = 0; t0 < B; t0 += blockDim.x) {
    const uint32_t t = t0 + threadIdx.x;
    const uint32_t h = t < B ? a.hist[t] : 0u;
    uint32_t tot_h, tot_r;
    const uint32_t eh = block_excl_scan(h, sh, &tot_h);
    const uint32_t er = block_excl_scan(h ? 1u : 0u, sh, &tot_r);
    if (t < B) a.bucket_start[t] = carry_start + eh;
    __syncthreads();
    if (threadIdx.x == 0) { carry_start += tot_h; carry_rows += tot_r; }
    __syncthreads();
    (void)er;
  }
  const uint32_t P = carry_rows;
  const uint64_t F = m0.F, S = m0.S, T = m0.T;
  const uint64_t meta_bytes = 4 * F + 8 * (uint64_t)P + 8 * S;
  const uint32_t delta = (uint32_t)((16u - ((32u + meta_bytes) & 15u)) & 15u);
  const uint64_t first_off = delta + 32ull;
  const uint64_t count_off = first_off + 4 * F;
  const uint64_t shift_off = count_off + 8ull * P;
  const uint64_t data_off = shift_off + 8 * S;
  // repeat table rows (ckpt id, count) in ascending id order (:656-665)
  __shared__ uint32_t row_carry;
  if (threadIdx.x == 0) row_carry = 0;
  __syncthreads();
  for (uint32_t t0 = 0; t0 < B; t0 += blockDim.x) {
    const uint32_t t = t0 + threadIdx.x;
    const uint32_t h = t < B ? a.hist[t] : 0u;
    uint32_t tot_r;
    const uint32_t er = block_excl_scan(h ? 1u : 0u, sh, &tot_r);
    if (h) {
      uint32_t* row = reinterpret_cast<uint32_t*>(a.diff + count_off + 8ull * (row_carry + er));
      row[0] = t;
      row[1] = h;
    }
    __syncthreads();
    if (threadIdx.x == 0) row_carry += tot_r;
    __syncthreads();
  }
  // per-range scatter bases: bucket start + counts of earlier ranges.  `partial` is
  // bucket-major (partial[t * g + range]); one warp scans one bucket's g range counts.
  {
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (uint32_t t = warp; t < B; t += nw) {
      uint32_t carry = a.bucket_start[t];
      uint32_t* row = a.partial + (uint64_t)t * g;
#pragma unroll 4
      for (uint32_t j = 0; j < g; j += 32) {
        const uint32_t b = j + lane;
        const uint32_t v = b < g ? row[b] : 0u;
        const uint32_t inc = warp_incl_scan(v);
        if (b < g) row[b] = carry + inc - v;
        carry += __shfl_sync(0xffffffffu, inc, 31);
      }
    }
  }
  if (threadIdx.x == 0) {
    uint32_t* h32 = reinterpret_cast<uint32_t*>(a.diff + delta);
    h32[0] = a.baseline_id;                 // ref_id
    h32[1] = a.cur;                         // chkpt_id
    h32[2] = (uint32_t)a.len;               // datalen (u64, little endian)
    h32[3] = (uint32_t)(a.len >> 32);
    h32[4] = a.cs;                          // chunk_size
    h32[5] = (uint32_t)F;                   // num_first_ocur
    h32[6] = P;                             // num_prior_chkpts
    h32[7] = (uint32_t)S;                   // num_shift_dupl
    DevMeta* m = a.meta;
    m->P = P;
    m->delta = delta;
    m->first_off = first_off;
    m->count_off = count_off;
    m->shift_off = shift_off;
    m->data_off = data_off;
    m->diff_len = 32ull + meta_bytes + T * a.cs;
    m->map_size = *a.map.size;
  }
}
__global__ void __launch_bounds__(1024) layout_kernel(DiffArgs a0, uint32_t bcap, uint32_t g) {
  griddep_enter();
  layout_body(with_round(a0), blockIdx.x, gridDim.x, bcap, g);
}
__global__ void __launch_bounds__(1024) layout_seg(SegGrid s) {
  uint32_t bid, nb;
  const uint32_t h = seg_locate(s, bid, nb);
  layout_body(with_round(s.args[h]), bid, nb, s.bcap[h], s.gs[h]);
}

// stable scatter of shift entries: one warp walks its range in order
__device__ __forceinline__ void shift_write_body(const DiffArgs& a, uint32_t bid, uint32_t nb, uint32_t bcap) {
  const uint32_t B = a.rs->buckets <= bcap ? a.rs->buckets : bcap;
  extern __shared__ uint32_t run[];
  uint64_t beg, end;
  cta_range(a.meta->S, bid, nb, beg, end);
  if (beg >= end) return;
  for (uint32_t t = threadIdx.x; t < B; t += 32) run[t] = a.partial[(uint64_t)t * nb + bid];
  __syncwarp();
  const uint64_t shift_off = a.meta->shift_off;
  const uint32_t lane = threadIdx.x;
  // UNR groups of 32 entries per pass: their loads are issued together (they do
  // not depend on the running bucket positions), then the groups are placed in order
  constexpr uint32_t UNR = 4;
  for (uint64_t t0 = beg; t0 < end; t0 += 32ull * UNR) {
    uint32_t key[UNR], node[UNR], prev[UNR];
#pragma unroll
    for (uint32_t u = 0; u < UNR; u++) {
      const uint64_t i = t0 + 32ull * u + lane;
      const bool act = i < end;
      key[u] = act ? a.skey[i] : 0xffffffffu;
      node[u] = act ? a.shift_list[i] : 0u;
      prev[u] = act ? a.sprev[i] : 0u;
    }
#pragma unroll
    for (uint32_t u = 0; u < UNR; u++) {
      const bool act = t0 + 32ull * u + lane < end;
      const uint32_t peers = __match_any_sync(0xffffffffu, key[u]);
      const uint32_t rank = __popc(peers & ((1u << lane) - 1u));
      uint32_t pos = 0;
      if (act) pos = run[key[u]] + rank;
      __syncwarp();
      if (act && rank == 0) run[key[u]] += __popc(peers);
      __syncwarp();
      if (act) {
        uint32_t* e = reinterpret_cast<uint32_t*>(a.diff + shift_off + 8ull * pos);
        e[0] = node[u] - a.id_bias;
        e[1] = prev[u] - a.id_bias;
      }
    }
  }
}
__global__ void __launch_bounds__(32) shift_write_kernel(DiffArgs a0, uint32_t bcap) {
  griddep_enter();
  shift_write_body(with_round(a0), blockIdx.x, gridDim.x, bcap);
}
__global__ void __launch_bounds__(32) shift_write_seg(SegGrid s) {
  uint32_t bid, nb;
  const uint32_t h = seg_locate(s, bid, nb);
  shift_write_body(with_round(s.args[h]), bid, nb, s.bcap[h]);
}

// ---------------------------------------------------------------- metadata + data gather
__device__ __forceinline__ uint32_t find_region(const uint32_t* off, uint32_t F, uint64_t k) {
  uint32_t lo = 0, hi = F;   // largest i with off[i] <= k
  while (hi - lo > 1) {
    const uint32_t mid = (lo + hi) >> 1;
    if (off[mid] <= k) lo = mid; else hi = mid;
  }
  return lo;
}

// Data section.  Each warp owns a contiguous range [k0, k1) of diff chunks (the same share for
// every warp) and copies it with 16-byte vectors, lane after lane over consecutive 16-byte units
// of the range, GATHER_UNROLL units per lane in flight (chunk size a multiple of 16, both sides
// 16-byte aligned), whatever the region boundaries: many regions are a few chunks long.  A unit's
// source follows from its chunk's region (start in the diff, root node).  The starts and roots
// of 32 regions at a time are held one per lane, and each unit finds its region among them by a
// five-step shuffle search, so no load waits on another: looked up in memory, each group of
// chunks waited for two dependent loads before its data load could issue.  The short last chunk
// is zero-padded (:643-645).
#ifndef B2D_GATHER_UNROLL
#define B2D_GATHER_UNROLL 4
#endif
__device__ __forceinline__ void gather_vec_body(const DiffArgs& a, uint32_t bid, uint32_t nb) {
  constexpr uint32_t U = B2D_GATHER_UNROLL;
  const DevMeta m = *a.meta;
  uint8_t* dst_base = a.diff + m.data_off;
  uint32_t* first_meta = reinterpret_cast<uint32_t*>(a.diff + m.first_off);
  const uint64_t gtid = bid * (uint64_t)blockDim.x + threadIdx.x;
  const uint64_t nthr = (uint64_t)nb * blockDim.x;
  for (uint64_t i = gtid; i < m.F; i += nthr) first_meta[i] = a.first_list[i] - a.id_bias;
  if (m.T == 0) return;
  const uint32_t lane = threadIdx.x & 31u;
  const uint64_t warp = gtid >> 5, nwarps = nthr >> 5;
  uint64_t k0, k1;
  cta_range(m.T, (uint32_t)warp, (uint32_t)nwarps, k0, k1);
  if (k0 >= k1) return;
  const uint64_t T = m.T;
  const uint32_t F = m.F;
  const uint32_t units = a.cs / 16u;   // 16-byte units per chunk
  const bool pow2 = (units & (units - 1u)) == 0u;
  const uint32_t ush = __ffs(units) - 1u;
  const uint64_t last = a.n - 1ull;
  const bool short_last = (a.len % a.cs) != 0;
  const uint4* src = reinterpret_cast<const uint4*>(a.data);
  uint4* dst = reinterpret_cast<uint4*>(dst_base);
  // largest r with region_off[r] <= k0 (region_off[0] = 0)
  uint32_t r = warp_lower_bound(a.region_off, F, k0 + 1u) - 1u;
  uint64_t k = k0;
  while (k < k1) {
    // regions r .. r + 31, one per lane; chunks before `bend` lie in them
    const uint32_t rl = r + lane;
    const uint32_t off_l = rl < F ? a.region_off[rl] : (uint32_t)T;
    const uint32_t node_l = rl < F ? a.first_list[rl] : 0u;
    const uint64_t bend = r + 32u < F ? a.region_off[r + 32u] : T;
    const uint64_t kend = bend < k1 ? bend : k1;
    const uint64_t u_end = kend * units;
    for (uint64_t base = k * units; base < u_end; base += 32ull * U) {
      uint4 v[U];
      uint32_t st = 0;   // bit i: unit i is this lane's to copy
#pragma unroll
      for (uint32_t i = 0; i < U; i++) {
        const uint64_t g = base + lane + 32ull * i;
        const bool act = g < u_end;
        const uint64_t kk = act ? (pow2 ? g >> ush : g / units) : k;
        uint32_t j = 0;   // largest j with region start j <= kk
#pragma unroll
        for (uint32_t step = 16; step >= 1; step >>= 1) {
          const uint32_t o = __shfl_sync(0xffffffffu, off_l, j + step);
          if (o <= kk) j += step;
        }
        const uint32_t off = __shfl_sync(0xffffffffu, off_l, j);
        const uint32_t node = __shfl_sync(0xffffffffu, node_l, j);
        if (!act) continue;
        const uint64_t chunk = (uint64_t)(leftmost_leaf(node, a.N) - (a.n - 1u)) + (kk - off);
        const uint64_t su = chunk * units + (g - kk * units);
        if (chunk > last) {
          set_error(a.st, DERR_INTERNAL, 40);
        } else if (short_last && chunk == last) {   // bytes past the buffer's end are zero
          uint8_t tmp[16];
          for (uint32_t b = 0; b < 16; b++) tmp[b] = 16ull * su + b < a.len ? a.data[16ull * su + b] : 0u;
          uint4 w;
          memcpy(&w, tmp, 16);
          dst[g] = w;
        } else {
          st |= 1u << i;
          v[i] = __ldg(src + su);
        }
      }
#pragma unroll
      for (uint32_t i = 0; i < U; i++)
        if ((st >> i) & 1u) dst[base + lane + 32ull * i] = v[i];
    }
    k = kend;
    r += 32u;
  }
}
__global__ void __launch_bounds__(256) gather_vec_kernel(DiffArgs a0) {
  griddep_enter();
  gather_vec_body(with_round(a0), blockIdx.x, gridDim.x);
}
__global__ void __launch_bounds__(256) gather_vec_seg(SegGrid s) {
  uint32_t bid, nb;
  const uint32_t h = seg_locate(s, bid, nb);
  gather_vec_body(with_round(s.args[h]), bid, nb);
}

// any chunk size / alignment: one thread per chunk, byte copies
__device__ __forceinline__ void gather_bytes_body(const DiffArgs& a, uint32_t bid, uint32_t nb) {
  const DevMeta m = *a.meta;
  uint8_t* dst_base = a.diff + m.data_off;
  uint8_t* first_meta = a.diff + m.first_off;
  const uint64_t gtid = bid * (uint64_t)blockDim.x + threadIdx.x;
  const uint64_t nthr = (uint64_t)nb * blockDim.x;
  for (uint64_t i = gtid; i < m.F; i += nthr) {
    const uint32_t v = a.first_list[i] - a.id_bias;
    memcpy(first_meta + 4 * i, &v, 4);
  }
  for (uint64_t k = gtid; k < m.T; k += nthr) {
    const uint32_t r = find_region(a.region_off, m.F, k);
    const uint32_t node = a.first_list[r];
    const uint64_t chunk = (uint64_t)(leftmost_leaf(node, a.N) - (a.n - 1u)) + (k - a.region_off[r]);
    if (chunk >= a.n) { set_error(a.st, DERR_INTERNAL, 41); continue; }
    const uint64_t src_off = chunk * a.cs;
    const uint64_t avail = (chunk == a.n - 1u) ? a.len - src_off : a.cs;
    uint8_t* d = dst_base + k * a.cs;
    const uint8_t* s = a.data + src_off;
    for (uint64_t b = 0; b < a.cs; b++) d[b] = b < avail ? s[b] : 0u;
  }
}
__global__ void __launch_bounds__(256) gather_bytes_kernel(DiffArgs a0) {
  griddep_enter();
  gather_bytes_body(with_round(a0), blockIdx.x, gridDim.x);
}
__global__ void __launch_bounds__(256) gather_bytes_seg(SegGrid s) {
  uint32_t bid, nb;
  const uint32_t h = seg_locate(s, bid, nb);
  gather_bytes_body(with_round(s.args[h]), bid, nb);
}

static uint32_t grid_for(uint64_t units, uint64_t per_cta, uint32_t cap) {
  const uint64_t g = (units + per_cta - 1) / per_cta;
  return g < 1 ? 1u : (g > cap ? cap : (uint32_t)g);
}

// grids follow the buffer size (host-known bounds: F, S <= n), so a small buffer is not charged
// for hundreds of idle CTAs per launch; large buffers get the full grids
DiffGrids diff_grids(const DiffArgs& a, int sm_count) {
  DiffGrids r;
  r.g = grid_for(((uint64_t)a.N + 63u) / 64u, 512, COMPACT_GRID);   // ~1 64-node load per thread
  // shift-entry ranges: the layout kernel scans every range's count per bucket in one CTA, so
  // fewer, longer ranges (<= 296) keep it short; the scatter walks each range with one warp
  r.gs = grid_for(a.n, 8192, SHIFT_GRID);
  r.gl = (2u * (a.D + 2u) * 32u + 255u) / 256u;
  r.gp = grid_for(a.n, 2048, (uint32_t)sm_count * 2u);
  r.gg = grid_for((uint64_t)a.n * a.cs, 32768, (uint32_t)sm_count * 4u);
  const bool vec = (a.cs % 16u == 0) && ((reinterpret_cast<uintptr_t>(a.data) & 15u) == 0) &&
                   ((reinterpret_cast<uintptr_t>(a.diff) & 15u) == 0);
  r.variant = vec ? 0 : 1;
  return r;
}

cudaError_t launch_collect_diff_batch(const DiffBatch& b, cudaStream_t stream, uint32_t* launches) {
  if (b.max_bcap > MAX_BUCKETS || b.base.n == 0) return cudaErrorInvalidValue;
  SegGrid s = b.base;
  uint32_t c = 0;
  const size_t hsm = sizeof(uint32_t) * b.max_bcap;
  s.beg = b.beg_g;   compact_count_seg<<<b.tot_g, COMPACT_THREADS, 0, stream>>>(s); c++;
  s.beg = b.beg_one; compact_scan_seg<<<b.tot_one, 1024, 0, stream>>>(s); c++;
  s.beg = b.beg_g;   compact_write_seg<<<b.tot_g, COMPACT_THREADS, 0, stream>>>(s); c++;
  s.beg = b.beg_gl;  compact_levels_seg<<<b.tot_gl, 256, 0, stream>>>(s); c++;
  s.beg = b.beg_gp;  compact_permute_seg<<<b.tot_gp, 256, 0, stream>>>(s); c++;
  s.beg = b.beg_g;   region_count_seg<<<b.tot_g, COMPACT_THREADS, 0, stream>>>(s); c++;
  s.beg = b.beg_one; region_scan_seg<<<b.tot_one, 1024, 0, stream>>>(s); c++;
  s.beg = b.beg_g;   region_write_seg<<<b.tot_g, COMPACT_THREADS, 0, stream>>>(s); c++;
  s.beg = b.beg_gs;  shift_prev_seg<<<b.tot_gs, 128, hsm, stream>>>(s); c++;
  s.beg = b.beg_one; layout_seg<<<b.tot_one, 1024, 0, stream>>>(s); c++;
  s.beg = b.beg_gs;  shift_write_seg<<<b.tot_gs, 32, hsm, stream>>>(s); c++;
  for (int v = 0; v < GATHER_VARIANTS; v++) {
    if (!b.tot_gather[v]) continue;
    s.beg = b.beg_gather[v];
    if (v == 0) gather_vec_seg<<<b.tot_gather[v], 256, 0, stream>>>(s);
    else gather_bytes_seg<<<b.tot_gather[v], 256, 0, stream>>>(s);
    c++;
  }
  if (launches) *launches = c;
  return cudaGetLastError();
}

cudaError_t launch_collect_diff(const DiffArgs& args, uint32_t bcap, int sm_count, cudaStream_t stream,
                                bool node_order) {
  DiffArgs a = args;
  const DiffGrids dg = diff_grids(a, sm_count);
  const uint32_t g = dg.g, gs = dg.gs;
  const uint32_t B = bcap;   // capacity; each kernel reads the checkpoint's bucket count from rs
  if (B > MAX_BUCKETS) return cudaErrorInvalidValue;
  // one kernel after another, each launched to overlap its start with its predecessor's end
  // (launch_dependent); the scan kernel also clears the per-checkpoint bucket counts
  cudaError_t e;
#define B2D_LD(...)                                              \
  if ((e = launch_dependent(__VA_ARGS__)) != cudaSuccess) return e;
  B2D_LD(compact_count_kernel, g, COMPACT_THREADS, 0, stream, a)
  B2D_LD(compact_scan_kernel, 1, 1024, 0, stream, a, g, B)
  B2D_LD(compact_write_kernel, g, COMPACT_THREADS, 0, stream, a)
  if (node_order) {
    a.first_list = a.tmp_first;
    a.shift_list = a.tmp_shift;
  } else {
    B2D_LD(compact_levels_kernel, dg.gl, 256, 0, stream, a)
    B2D_LD(compact_permute_kernel, dg.gp, 256, 0, stream, a)
  }
  B2D_LD(region_count_kernel, g, COMPACT_THREADS, 0, stream, a)
  B2D_LD(region_scan_kernel, 1, 1024, 0, stream, a, g)
  B2D_LD(region_write_kernel, g, COMPACT_THREADS, 0, stream, a)
  const size_t hsm = sizeof(uint32_t) * B;   // <= 32 KB for MAX_BUCKETS
  B2D_LD(shift_prev_kernel, gs, 128, hsm, stream, a, B)
  B2D_LD(layout_kernel, 1, 1024, 0, stream, a, B, gs)
  B2D_LD(shift_write_kernel, gs, 32, hsm, stream, a, B)
  const uint32_t gblocks = dg.gg;
  const bool vec = (a.cs % 16u == 0) && ((reinterpret_cast<uintptr_t>(a.data) & 15u) == 0) &&
                   ((reinterpret_cast<uintptr_t>(a.diff) & 15u) == 0);
  if (vec) {
    B2D_LD(gather_vec_kernel, gblocks, 256, 0, stream, a)
  } else {
    B2D_LD(gather_bytes_kernel, gblocks, 256, 0, stream, a)
  }
#undef B2D_LD
  return cudaSuccess;
}

}  // namespace b2d

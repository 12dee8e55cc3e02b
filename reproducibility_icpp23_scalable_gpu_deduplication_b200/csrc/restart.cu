// Restart: rebuild checkpoint `id` from the diffs ref_id..id (host-view restart of the
// reference, src/tree_approach.cpp:712-1128).
//
// The reference keeps two hash maps per diff (NodeID -> data offset for every node under a
// first-occurrence region, node -> source NodeID for every shifted leaf) and walks the diffs
// newest to oldest, one pass over all chunks per diff.  Every lookup the restart makes is for a
// leaf, so here both maps become dense per-leaf arrays with a flag byte per leaf (only the
// flags are cleared for each diff), and the passes over the older diffs are fused:
//   main diff   : its region lists are expanded one thread per chunk; the chunks it names get
//                 their NodeID in node_list (flag mflag) and, where the main diff holds their
//                 data, their copy (:822-939)
//   older diffs : up to RESTART_WINDOW at a time are expanded into window slots, then one walk
//                 kernel takes every chunk's NodeID through the window's diffs in the
//                 reference's order -- each diff acts on the chunks whose NodeID names it
//                 (:1083-1118) -- and copies the chunk from the diff that resolves it.  Between
//                 windows node_list carries every chunk's NodeID.
// A chunk's NodeID depends only on its own history, so the per-chunk walk makes the same
// decisions as the reference's per-diff passes; where a malformed chain resolves a chunk twice,
// the later copy wins as it does there.
//
// Region lists are expanded after an exclusive scan of the region sizes; each entry's leftmost
// leaves and source checkpoint are computed once, in the scan's write pass.  Chunk copies are
// made by whole warps: consecutive lanes move consecutive 16/8/4-byte pieces of the warp's
// chunks, so the diffs can be read where they lie (a data section need only be 4-byte aligned;
// the stores stay 16 bytes wide) and every load and store instruction covers whole sectors.
// Every index and copy is bounds-checked: a diff that would make the reference read or write
// outside a buffer sets DERR_RESTART_RANGE and the access is skipped.
#include "restart.cuh"
#include "scan.cuh"

namespace b2d {

constexpr uint32_t R_THREADS = 256;

// pieces in flight per lane of a warp copy, and the resident CTAs per SM the copying kernels
// are compiled for (register cap)
#ifndef B2D_RESTART_UNROLL
#define B2D_RESTART_UNROLL 4
#endif
#ifndef B2D_RESTART_MINB
#define B2D_RESTART_MINB 4
#endif
constexpr uint32_t R_UNROLL = B2D_RESTART_UNROLL;
constexpr unsigned R_FULL = 0xffffffffu;

__device__ __forceinline__ uint32_t rd_u32(const uint8_t* p) {
  uint32_t v;
  memcpy(&v, p, 4);
  return v;
}
// a node id of the diff as a heap index: list diffs name chunk c, whose leaf is n-1+c; a chunk
// id outside the checkpoint maps to N, one past the last node, which every use rejects
__device__ __forceinline__ uint32_t rd_node(const RestartArgs& a, const uint8_t* p) {
  const uint32_t v = rd_u32(p);
  if (!a.id_bias) return v;
  return v < a.n ? v + a.id_bias : a.N;
}

__device__ __forceinline__ void copy_bytes(uint8_t* dst, const uint8_t* src, uint64_t nb) {
  if ((((uintptr_t)dst | (uintptr_t)src) & 15u) == 0) {
    const uint64_t nv = nb / 16u;
    uint4* d4 = reinterpret_cast<uint4*>(dst);
    const uint4* s4 = reinterpret_cast<const uint4*>(src);
    for (uint64_t i = 0; i < nv; i++) d4[i] = s4[i];
    for (uint64_t i = nv * 16u; i < nb; i++) dst[i] = src[i];
  } else {
    for (uint64_t i = 0; i < nb; i++) dst[i] = src[i];
  }
}

// source of a copy of nb bytes from data-section offset src_off to out[dst_off..], or null (and
// DERR_RESTART_RANGE) when either side would leave its buffer
__device__ __forceinline__ const uint8_t* checked_src(const uint8_t* data, uint64_t data_len, uint64_t out_len,
                                                      uint64_t dst_off, uint64_t src_off, uint64_t nb,
                                                      DevStatus* st) {
  if (dst_off > out_len || nb > out_len - dst_off || src_off > data_len || nb > data_len - src_off) {
    set_error(st, DERR_RESTART_RANGE, 1);
    return nullptr;
  }
  return data + src_off;
}

// 16 bytes from a 4-byte aligned address, in the widest loads its alignment allows; never
// touches a byte outside [a, a+16)
__device__ __forceinline__ uint4 load16(const uint8_t* a) {
  const uint32_t m = (uint32_t)(uintptr_t)a & 15u;
  if (m == 0) return __ldg(reinterpret_cast<const uint4*>(a));
  if ((m & 7u) == 0) {
    const uint2 x = __ldg(reinterpret_cast<const uint2*>(a));
    const uint2 y = __ldg(reinterpret_cast<const uint2*>(a + 8));
    return make_uint4(x.x, x.y, y.x, y.y);
  }
  const uint32_t x = __ldg(reinterpret_cast<const uint32_t*>(a));
  const uint2 y = __ldg(reinterpret_cast<const uint2*>(a + 4));
  const uint32_t z = __ldg(reinterpret_cast<const uint32_t*>(a + 12));
  return make_uint4(x, y.x, y.y, z);
}
template <class V>
__device__ __forceinline__ V load_piece(const uint8_t* a) {
  return __ldg(reinterpret_cast<const V*>(a));
}
template <>
__device__ __forceinline__ uint4 load_piece<uint4>(const uint8_t* a) {
  return load16(a);
}

// the warp's whole chunks in pieces of V: piece p belongs to the chunk of lane p / per
template <class V>
__device__ __forceinline__ void warp_pieces(uint8_t* out, uint32_t per, uint32_t per_log2, uint64_t dst,
                                            const uint8_t* src) {
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t total = 32u * per;
  const unsigned long long s_lane = reinterpret_cast<unsigned long long>(src);
  for (uint32_t p0 = 0; p0 < total; p0 += 32u * R_UNROLL) {
    V v[R_UNROLL];
    uint8_t* d[R_UNROLL];
#pragma unroll
    for (uint32_t u = 0; u < R_UNROLL; u++) {
      const uint32_t p = p0 + 32u * u + lane;
      const uint32_t j = per_log2 != 0xffu ? p >> per_log2 : p / per;
      const uint32_t q = p - j * per;
      const unsigned long long s = __shfl_sync(R_FULL, s_lane, j & 31u);
      const uint64_t t = __shfl_sync(R_FULL, dst, j & 31u);
      d[u] = nullptr;
      if (p < total && s != 0ull) {
        v[u] = load_piece<V>(reinterpret_cast<const uint8_t*>(s + (uint64_t)q * sizeof(V)));
        d[u] = out + t + (uint64_t)q * sizeof(V);
      }
    }
#pragma unroll
    for (uint32_t u = 0; u < R_UNROLL; u++)
      if (d[u]) *reinterpret_cast<V*>(d[u]) = v[u];
  }
}

// Copies one chunk per lane: out[dst..dst+nb) <- src[0..nb), src null for a lane with nothing
// to copy (ranges already checked).  All lanes of the warp call it together.  Whole chunks
// (nb == cs) go through warp_pieces; a short last chunk, or every chunk when no piece width
// fits, is copied by its own lane.
__device__ __forceinline__ void warp_copy(uint8_t* out, uint32_t cs, uint32_t width, uint32_t per, uint32_t per_log2,
                                          uint64_t dst, const uint8_t* src, uint64_t nb) {
  if (src && (width == 0 || nb != cs)) {
    copy_bytes(out + dst, src, nb);
    src = nullptr;
  }
  if (width == 0 || !__any_sync(R_FULL, src != nullptr)) return;
  if (width == 16) warp_pieces<uint4>(out, per, per_log2, dst, src);
  else if (width == 8) warp_pieces<uint2>(out, per, per_log2, dst, src);
  else warp_pieces<uint32_t>(out, per, per_log2, dst, src);
}

// warp-uniform grid-stride loop over items in groups of 32 (lane i takes item base + i)
#define R_WARP_LOOP(base, count)                                                            \
  const uint32_t lane = threadIdx.x & 31u;                                                  \
  const uint64_t w0_ = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;              \
  const uint64_t nw_ = ((uint64_t)gridDim.x * blockDim.x) >> 5;                             \
  for (uint64_t base = w0_ * 32u; base < (count); base += nw_ * 32u)

__device__ __forceinline__ uint32_t shift_tree(const RestartArgs& a, uint64_t i) {
  // smallest checkpoint id whose inclusive running count exceeds i, else 0 (:879-885)
  uint32_t lo = 0, hi = a.ncum;
  while (lo < hi) {
    const uint32_t mid = (lo + hi) >> 1;
    if (a.cum[mid] > i) hi = mid; else lo = mid + 1;
  }
  return lo < a.ncum ? lo : 0u;
}

// leaves covered by region entry i; with want_meta it also records the entry's leftmost leaves
// (and for a shift entry its source checkpoint)
__device__ __forceinline__ uint32_t entry_len(const RestartArgs& a, uint64_t i, int which, bool want_meta) {
  if (which == 0) {
    uint32_t lo, hi;
    leaf_range(rd_node(a, a.diff + a.first_off + 4 * i), a.N, lo, hi);
    if (want_meta) a.rstart[i] = lo;
    return hi - lo + 1u;
  }
  const uint32_t node = rd_node(a, a.diff + a.shift_off + 8 * i);
  const uint32_t prev = rd_node(a, a.diff + a.shift_off + 8 * i + 4);
  uint32_t nlo, nhi, plo, phi;
  leaf_range(node, a.N, nlo, nhi);
  leaf_range(prev, a.N, plo, phi);
  if (want_meta) {
    a.rstart[i] = nlo;
    a.pstart[i] = plo;
    a.rtree[i] = shift_tree(a, i);
  }
  // the main diff copies num_leaf_descendents(prev) leaves (:906), older diffs map
  // num_leaf_descendents(node) leaves (:1067)
  return a.is_main ? phi - plo + 1u : nhi - nlo + 1u;
}

__global__ void __launch_bounds__(R_THREADS) r_count_kernel(RestartArgs a, int which) {
  __shared__ uint32_t sh[R_THREADS / 32 + 1];
  uint64_t beg, end;
  cta_range(which == 0 ? a.F : a.S, blockIdx.x, gridDim.x, beg, end);
  uint32_t c = 0;
  for (uint64_t i = beg + threadIdx.x; i < end; i += blockDim.x) c += entry_len(a, i, which, false);
  const uint32_t t = block_reduce_sum(c, sh);
  if (threadIdx.x == 0) a.partial[blockIdx.x] = t;
}

__global__ void __launch_bounds__(1024) r_scan_kernel(RestartArgs a, uint32_t g) {
  __shared__ uint32_t sh[33];
  uint32_t tot;
  const uint32_t i = threadIdx.x;
  const uint32_t v = i < g ? a.partial[i] : 0u;
  const uint32_t e = block_excl_scan(v, sh, &tot);
  if (i < g) a.partial[i] = e;
  if (i == 0) *a.total = tot;
}

__global__ void __launch_bounds__(R_THREADS) r_write_kernel(RestartArgs a, int which) {
  __shared__ uint32_t sh[R_THREADS / 32 + 1];
  uint64_t beg, end;
  cta_range(which == 0 ? a.F : a.S, blockIdx.x, gridDim.x, beg, end);
  uint32_t base = a.partial[blockIdx.x];
  for (uint64_t t0 = beg; t0 < end; t0 += blockDim.x) {
    const uint64_t i = t0 + threadIdx.x;
    const uint32_t len = i < end ? entry_len(a, i, which, true) : 0u;
    uint32_t tot;
    const uint32_t e = block_excl_scan(len, sh, &tot);
    if (i < end) a.offs[i] = base + e;
    base += tot;
  }
}

// largest i in [lo, hi) with off[i] <= k (off[lo] <= k)
__device__ __forceinline__ uint32_t find_entry(const uint32_t* off, uint32_t lo, uint32_t hi, uint64_t k) {
  while (hi - lo > 1) {
    const uint32_t mid = (lo + hi) >> 1;
    if (off[mid] <= k) lo = mid; else hi = mid;
  }
  return lo;
}

// Region-list expansion: warp w takes one contiguous range of expanded positions k, in windows
// of 32 (lane i takes k = base + i).  The entry of the range's first k is searched once; the 32
// positions of a window lie in at most the 32 entries from the previous window's last one (every
// entry covers at least one position), so each lane then searches only those -- one cache line
// for the whole warp.  A list diff, whose entries are single chunks, would otherwise pay a search
// over millions of entries per chunk.
// With a.id_bias (list diffs) every entry is one chunk: position k is entry k, no search.
#define R_EXPAND_LOOP(base, count, off, cnt)                                                      \
  const uint32_t lane = threadIdx.x & 31u;                                                        \
  const uint64_t w0_ = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;                    \
  const uint64_t nw_ = ((uint64_t)gridDim.x * blockDim.x) >> 5;                                   \
  const uint64_t per_ = ((count) + nw_ * 32u - 1u) / (nw_ * 32u) * 32u;                           \
  const uint64_t beg_ = w0_ * per_;                                                               \
  const uint64_t end_ = beg_ + per_ < (count) ? beg_ + per_ : (count);                            \
  uint32_t ib_ = (!a.id_bias && beg_ < end_) ? find_entry((off), 0u, (cnt), beg_) : 0u;          \
  for (uint64_t base = beg_; base < end_; base += 32u)

// entry of position k of the current window, whose first position lies in entry ib; an entry
// covering no position (only a malformed diff has one) sends the search past the window
__device__ __forceinline__ uint32_t window_entry(const uint32_t* off, uint32_t ib, uint32_t cnt, uint64_t k) {
  const uint32_t hi = ib + 32u < cnt ? ib + 32u : cnt;
  uint32_t i = find_entry(off, ib, hi, k);
  if (i + 1u == hi && hi < cnt && off[hi] <= k) i = find_entry(off, hi, cnt, k);
  return i;
}
#define R_WINDOW_ENTRY(off, cnt, k) window_entry((off), ib_, (cnt), (k))

// first-occurrence regions: dist for every leaf; the main diff also fills node_list and copies
// the chunk (:822-865 main, :1005-1030 older)
__global__ void __launch_bounds__(R_THREADS, B2D_RESTART_MINB) r_expand_first_kernel(RestartArgs a) {
  const uint64_t T = a.id_bias ? (uint64_t)a.F : *a.total;
  const uint8_t* data = a.diff + a.data_off;
  const uint64_t data_len = a.diff_size - a.data_off;
  R_EXPAND_LOOP(kb, T, a.offs, a.F) {
    const uint64_t k = kb + lane;
    uint64_t dst = 0, nb = 0;
    const uint8_t* src = nullptr;
    uint32_t i = ib_;
    if (k < end_) {
      uint32_t start, j, off0;
      if (a.id_bias) {   // one chunk per entry, at data offset k (src/list_approach.cpp:331-351)
        i = (uint32_t)k;
        start = rd_node(a, a.diff + a.first_off + 4ull * k);
        j = 0;
        off0 = (uint32_t)k;
      } else {
        i = R_WINDOW_ENTRY(a.offs, a.F, k);
        start = a.rstart[i];
        off0 = a.offs[i];
        j = (uint32_t)(k - off0);
      }
      const uint64_t c = (uint64_t)start - (a.n - 1u) + j;
      if (start < a.n - 1u || c >= a.n) {
        set_error(a.st, DERR_RESTART_RANGE, 2);
      } else {
        const uint32_t off = off0 + j;   // u32 like the reference (:846, :1018)
        a.slot.dist[c] = off;
        a.slot.flag[c] = R_HAS_DIST;   // the diff's first writer of this flag
        if (a.is_main) {
          a.node_list[c] = make_uint2((uint32_t)c, a.cur_id);
          a.mflag[c] = 1;
          dst = c * a.cs;
          nb = (c == a.n - 1u) ? a.datalen - dst : a.cs;
          src = checked_src(data, data_len, a.out_len, dst, (uint64_t)off * a.cs, nb, a.st);
        }
      }
    }
    if (a.is_main) warp_copy(a.out, a.cs, a.width, a.per, a.per_log2, dst, src, nb);
    ib_ = __shfl_sync(R_FULL, i, 31);
  }
}

// Leaves on the shallower level under a region root that spans two depths (only possible
// when the chunk count is not a power of two): the reference inserts them with an offset
// computed in wrapping u32 arithmetic (:844-846, :1016-1018).  Reproduced so later lookups
// of those leaves behave the same.
StraddleQuery straddle_query(uint32_t n) {
  StraddleQuery q;
  q.count = 0;
  if (n < 3 || (n & (n - 1)) == 0) return q;
  uint32_t x = n - 2, y = n - 1;
  while (x != y) {
    if (x > y) x = (x - 1) / 2;
    else y = (y - 1) / 2;
  }
  for (;;) {
    q.anc[q.count++] = x;
    if (x == 0 || q.count == 32) break;
    x = (x - 1) / 2;
  }
  return q;
}

__global__ void r_straddle_find_kernel(RestartArgs a, StraddleQuery q, StraddleInfo* sd) {
  const uint32_t D = node_level(a.N - 1u);
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < a.F; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t node = rd_u32(a.diff + a.first_off + 4 * i);
    bool hit = false;
    for (uint32_t k = 0; k < q.count; k++) hit |= q.anc[k] == node;
    if (!hit) continue;
    // leaves of level D-1 under this root
    const uint32_t k = (D - 1u) - node_level(node);
    const uint64_t lo_all = ((uint64_t)node << k) + (1ull << k) - 1ull;
    const uint64_t hi_all = lo_all + (1ull << k) - 1ull;
    const uint64_t lo = lo_all > (uint64_t)a.n - 1u ? lo_all : (uint64_t)a.n - 1u;
    const uint64_t lvl_end = (1ull << D) - 2ull;
    const uint64_t hi = hi_all < lvl_end ? hi_all : lvl_end;
    if (lo <= hi) {
      sd->root = node;
      sd->region_off = a.offs[i];
      sd->lo = (uint32_t)lo;
      sd->hi = (uint32_t)hi;
      __threadfence();
      sd->present = 1;
    }
  }
}

__global__ void r_straddle_kernel(RestartArgs a, const StraddleInfo* sd) {
  if (!sd->present) return;
  const uint32_t root = sd->root, region_off = sd->region_off, lo = sd->lo, hi = sd->hi;
  const uint32_t start = leftmost_leaf(root, a.N);
  for (uint64_t u = lo + blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; u <= hi; u += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t c = u - (a.n - 1u);
    if (c < a.n) {
      a.slot.dist[c] = region_off + (uint32_t)u - start;
      a.slot.flag[c] |= R_HAS_DIST;
    }
  }
}

// shifted-duplicate entries (:888-927 main, :1049-1075 older)
__global__ void __launch_bounds__(R_THREADS, B2D_RESTART_MINB) r_expand_shift_kernel(RestartArgs a) {
  const uint64_t T = a.id_bias ? (uint64_t)a.S : *a.total;
  const uint8_t* data = a.diff + a.data_off;
  const uint64_t data_len = a.diff_size - a.data_off;
  R_EXPAND_LOOP(kb, T, a.offs, a.S) {
    const uint64_t k = kb + lane;
    uint64_t dst = 0, nb = 0;
    const uint8_t* src = nullptr;
    uint32_t i = ib_;
    if (k < end_) {
      uint32_t j, node_start, prev_start, tree;
      if (a.id_bias) {   // one chunk per entry (src/list_approach.cpp:371-408, :501-513)
        i = (uint32_t)k;
        j = 0;
        node_start = rd_node(a, a.diff + a.shift_off + 8ull * k);
        prev_start = rd_node(a, a.diff + a.shift_off + 8ull * k + 4);
        tree = shift_tree(a, k);
      } else {
        i = R_WINDOW_ENTRY(a.offs, a.S, k);
        j = (uint32_t)(k - a.offs[i]);
        node_start = a.rstart[i];
        prev_start = a.pstart[i];
        tree = a.rtree[i];
      }
      const uint64_t c = (uint64_t)node_start + j - (a.n - 1u);
      if (node_start < a.n - 1u || c >= a.n) {
        set_error(a.st, DERR_RESTART_RANGE, 3);
      } else if (a.is_main) {
        a.node_list[c] = make_uint2(prev_start + j, tree);
        a.mflag[c] = 1;
        if (tree == a.cur_id) {
          // offset of NodeID(prev, cur) = offset of prev's leftmost leaf; absent -> 0 (:898-901)
          uint64_t base = 0;
          const uint64_t pc = (uint64_t)prev_start - (a.n - 1u);
          if (prev_start >= a.n - 1u && pc < a.n && (a.slot.flag[pc] & R_HAS_DIST))
            base = (uint64_t)a.slot.dist[pc] * a.cs;
          dst = c * a.cs;
          nb = (c == a.n - 1u) ? a.out_len - dst : a.cs;
          src = checked_src(data, data_len, a.out_len, dst, base + (uint64_t)j * a.cs, nb, a.st);
        }
      } else {
        a.slot.rep[c] = make_uint2(prev_start + j, tree);
        a.slot.flag[c] |= R_HAS_REP;   // after the first-occurrence expansion of the same diff
      }
    }
    if (a.is_main) warp_copy(a.out, a.cs, a.width, a.per, a.per_log2, dst, src, nb);
    ib_ = __shfl_sync(R_FULL, i, 31);
  }
}

// Every chunk through the window's diffs, newest first (:1083-1118 per diff): a diff acts on a
// chunk whose NodeID names it -- copy from its data when the leaf is a first occurrence there
// (or a shifted copy of one in the same diff), follow a shifted leaf to its source NodeID, or
// pass the leaf on to the previous checkpoint.  Chunks the main diff does not name start at
// (their leaf, main id - 1), as the reference's node_list does (:933-939).  A chunk's NodeID
// usually stays its own leaf all the way down, so that leaf's flags in every slot are loaded up
// front, side by side; another leaf's flags are loaded when the walk reaches it.
__global__ void __launch_bounds__(R_THREADS, B2D_RESTART_MINB) r_walk_kernel(RestartWalk w) {
  R_WARP_LOOP(cb, w.n) {
    const uint64_t c = cb + lane;
    const uint64_t dst = c * w.cs;
    uint64_t nb = 0;
    const uint8_t* src = nullptr;
    if (c < w.n) {
      const uint32_t own = (uint32_t)c + w.n - 1u;   // heap index of chunk c's leaf
      uint32_t pf = 0;                                // 2 flag bits per slot for leaf `own`
#pragma unroll
      for (uint32_t k = 0; k < RESTART_WINDOW; k++)
        if (k < w.count) pf |= (uint32_t)w.slot[k].flag[c] << (2u * k);
      uint2 id;
      if (w.dense) {
        id = w.node_list[c];
      } else {
        id = make_uint2(own, w.main_cur - 1u);
        if (w.mflag[c]) {
          const uint2 m = w.node_list[c];
          if (m.x != 0xffffffffu) id = m;
        }
      }
      const uint2 id0 = id;
#pragma unroll
      for (uint32_t k = 0; k < RESTART_WINDOW; k++) {
        if (k >= w.count) break;
        const uint32_t cur = w.cur[k];
        if (id.y != cur) continue;
        const RestartSlot s = w.slot[k];
        uint64_t ws = w.cs;
        if (dst + ws > w.datalen[k]) ws = w.datalen[k] - dst;
        const uint64_t lc = (uint64_t)id.x - (w.n - 1u);
        const bool leaf = id.x >= w.n - 1u && lc < w.n;
        const uint32_t f = !leaf ? 0u : id.x == own ? (pf >> (2u * k)) & 3u : (uint32_t)s.flag[lc];
        if (f & R_HAS_DIST) {
          const uint8_t* p =
              checked_src(w.data[k], w.data_len[k], w.out_len, dst, (uint64_t)s.dist[lc] * w.cs, ws, w.st);
          if (p) {
            src = p;
            nb = ws;
          }
        } else if ((f & R_HAS_REP) && s.rep[lc].x != 0xffffffffu) {
          const uint2 prev = s.rep[lc];
          if (prev.y == cur) {
            const uint64_t pc = (uint64_t)prev.x - (w.n - 1u);
            if (prev.x >= w.n - 1u && pc < w.n && (s.flag[pc] & R_HAS_DIST)) {
              const uint8_t* p =
                  checked_src(w.data[k], w.data_len[k], w.out_len, dst, (uint64_t)s.dist[pc] * w.cs, ws, w.st);
              if (p) {
                src = p;
                nb = ws;
              }
            } else {
              set_error(w.st, DERR_RESTART_RANGE, 4);
            }
          } else {
            id = prev;
          }
        } else {
          id = make_uint2(id.x, cur - 1u);
        }
      }
      if (!w.last && (!w.dense || id.x != id0.x || id.y != id0.y)) w.node_list[c] = id;
    }
    warp_copy(w.out, w.cs, w.width, w.per, w.per_log2, dst, src, nb);
  }
}

// running shift counts per checkpoint id from a device-resident diff's (ckpt, count) table:
// the last row for an id wins, then an inclusive scan over ids (:871-885); rows naming an id
// beyond the diff's own are outside the reference's array and are reported
__global__ void r_cum_kernel(RestartArgs a) {
  unsigned long long* cum = const_cast<unsigned long long*>(a.cum);
  for (uint32_t t = threadIdx.x; t < a.ncum; t += blockDim.x) cum[t] = 0;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (uint32_t i = 0; i < a.P; i++) {
      const uint32_t ck = rd_u32(a.diff + a.count_off + 8ull * i);
      const uint32_t cnt = rd_u32(a.diff + a.count_off + 8ull * i + 4);
      if (ck < a.ncum) cum[ck] = cnt;
      else set_error(a.st, DERR_RESTART_RANGE, 5);
    }
    unsigned long long run = 0;
    for (uint32_t t = 0; t < a.ncum; t++) {
      run += cum[t];
      cum[t] = run;
    }
  }
}

cudaError_t launch_restart_cum(const RestartArgs& a, cudaStream_t s) {
  r_cum_kernel<<<1, 256, 0, s>>>(a);
  return cudaGetLastError();
}

static uint32_t grid_for(uint64_t work, int sm_count) {
  uint64_t b = ceil_div_u64(work ? work : 1, R_THREADS);
  const uint64_t cap = (uint64_t)sm_count * 8u;
  return (uint32_t)(b > cap ? cap : b);
}

// piece width of the warp copies.  16-byte pieces need the chunk size and the output 16-byte
// aligned and every source 4-byte aligned (a data section starts 32 + 4F + 8P + 8S bytes into
// its diff, so a diff read where it lies is often only 4-byte aligned; load16 reads such a
// source in narrower loads); otherwise the widest of 8/4 bytes dividing everything.
static void copy_width(uint64_t dst_al, uint64_t src_al, uint32_t cs, uint32_t& width, uint32_t& per,
                       uint32_t& per_log2) {
  const uint64_t al = dst_al | src_al | cs;
  if (((dst_al | cs) & 15u) == 0 && (src_al & 3u) == 0) width = 16;
  else width = (al & 7u) == 0 ? 8u : (al & 3u) == 0 ? 4u : 0u;
  if (width && cs / width > (1u << 26)) width = 0;   // keeps 32 x pieces per chunk in u32
  per = width ? cs / width : 0u;
  per_log2 = 0xffu;
  if (per && (per & (per - 1u)) == 0) per_log2 = (uint32_t)__builtin_ctz(per);
}

int restart_diff_launches(uint32_t n, bool list) { return list ? 2 : 8 + (straddle_query(n).count ? 2 : 0); }

cudaError_t launch_restart_diff(const RestartArgs& args, StraddleInfo* sd, int sm_count, cudaStream_t s) {
  RestartArgs a = args;
  copy_width((uint64_t)(uintptr_t)a.out, (uint64_t)(uintptr_t)(a.diff + a.data_off), a.cs, a.width, a.per,
             a.per_log2);
  cudaError_t e = cudaMemsetAsync(a.slot.flag, 0, a.n, s);
  if (e == cudaSuccess && a.is_main) e = cudaMemsetAsync(a.mflag, 0, a.n, s);
  if (e != cudaSuccess) return e;
  const uint32_t g = SCAN_GRID;
  const bool scan = !a.id_bias;   // list entries are single chunks: offsets are the entry indices
  // first-occurrence regions
  if (scan) {
    r_count_kernel<<<g, R_THREADS, 0, s>>>(a, 0);
    r_scan_kernel<<<1, 1024, 0, s>>>(a, g);
    r_write_kernel<<<g, R_THREADS, 0, s>>>(a, 0);
  }
  r_expand_first_kernel<<<grid_for(a.n, sm_count), R_THREADS, 0, s>>>(a);
  const StraddleQuery q = a.id_bias ? StraddleQuery{} : straddle_query(a.n);   // list regions are single leaves
  if (q.count) {
    e = cudaMemsetAsync(sd, 0, sizeof(StraddleInfo), s);
    if (e != cudaSuccess) return e;
    r_straddle_find_kernel<<<grid_for(a.F, sm_count), R_THREADS, 0, s>>>(a, q, sd);
    r_straddle_kernel<<<(uint32_t)sm_count * 4u, R_THREADS, 0, s>>>(a, sd);
  }
  // shifted duplicates
  if (scan) {
    r_count_kernel<<<g, R_THREADS, 0, s>>>(a, 1);
    r_scan_kernel<<<1, 1024, 0, s>>>(a, g);
    r_write_kernel<<<g, R_THREADS, 0, s>>>(a, 1);
  }
  r_expand_shift_kernel<<<grid_for(a.n, sm_count), R_THREADS, 0, s>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_restart_walk(const RestartWalk& walk, int sm_count, cudaStream_t s) {
  RestartWalk w = walk;
  if (w.count == 0 || w.count > RESTART_WINDOW) return cudaErrorInvalidValue;
  uint64_t src_al = 0;
  for (uint32_t k = 0; k < w.count; k++) src_al |= (uint64_t)(uintptr_t)w.data[k];
  copy_width((uint64_t)(uintptr_t)w.out, src_al, w.cs, w.width, w.per, w.per_log2);
  r_walk_kernel<<<grid_for(w.n, sm_count), R_THREADS, 0, s>>>(w);
  return cudaGetLastError();
}

}  // namespace b2d

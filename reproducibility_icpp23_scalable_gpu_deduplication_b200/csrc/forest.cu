// Merkle forest stages, level-fused.
//
// The reference walks the heap one level per launch, twice (src/tree_approach.cpp:116-224
// baseline, :371-477 incremental): ~2 log2(N) launches.  Here one launch reduces 12 levels:
// a CTA of 256 threads owns the subtree of 4096 input nodes under one node 12 levels up;
//   * each thread folds 16 consecutive input labels through 4 levels in registers,
//   * each warp folds its 32 thread results through 5 levels with shuffles,
//   * warp 0 folds the 8 warp results through the last 3 levels.
// Labels cross band boundaries through `lab` (only band outputs are written).  A subtree whose
// 16 inputs are all FIXED (phase 2) or contain no first occurrence (phase 1) is folded without
// touching memory, which is the common case of an incremental checkpoint.  The few levels left
// above the last full band (and trees with fewer than 12 levels) use forest_band_kernel, which
// walks a band level by level through shared memory.
//
// Phase 1 (FIRST forest): relabel leaves whose digest's lowest-index owner is another leaf
//   ("Choose first occurrences", :100-114 / :353-369), then every inner node with two
//   first-occurrence children becomes one, is hashed and inserted (:116-145 / :371-404).
// Phase 2 (region forest, :147-224 / :406-477): the label of each inner node follows from its
//   children's labels; differing children become region roots (push flags), two shifted
//   children merge only if the parent digest is already known.  The baseline tests the
//   parent digest before computing it (stale zero digest, :202), then hashes and inserts
//   every inner node (:218-224); this is reproduced with `zero_exists`.
// Map priorities reproduce the sequential insert order: leaves 0, phase-1 parents
// 1 + height, baseline per-level inserts 64 + height (height = D - level).
// `push` holds 2-bit flags, set with atomicOr (16 nodes share a word): it is all-zero between
// checkpoints (the compaction clears what it reads), so a region-free subtree writes nothing.
#include <vector>

#include "dedup_kernels.cuh"
#include "hash.cuh"
#include "map.cuh"

namespace b2d {

// resident CTAs per SM the band kernels are compiled for (register budget): phase 1 at 8
// (32 registers) measured ~6% faster on its launches than the unconstrained 40 registers; the
// phase-2 band at 4 (64 registers, no spills) took 0.29 instead of 0.30 ms of forest time per
// 4 GiB step once its first band ran on a resident grid (3 CTAs per SM before)
#ifndef B2D_FF_MINB
#define B2D_FF_MINB 8
#endif
#ifndef B2D_FAST_MINB
#define B2D_FAST_MINB 4
#endif

constexpr uint32_t FOREST_THREADS = 512;
constexpr uint32_t FAST_THREADS = 256;
constexpr uint32_t FAST_LEVELS = 12;      // 4 in-thread + 5 warp + 3 CTA
constexpr uint8_t NONE_LABEL = 5;         // node index beyond the tree

__device__ __forceinline__ uint8_t push_flag(uint8_t label) {
  return label == SHIFT_DUPL ? PUSH_SHIFT : (label == FIRST_OCUR ? PUSH_FIRST : PUSH_NONE);
}
// region-root flag of node x: 2 bits per node, 16 nodes per word (gather.cu reads them)
__device__ __forceinline__ void push_set(uint8_t* push, uint64_t x, uint32_t flag) {
  atomicOr(reinterpret_cast<uint32_t*>(push) + (x >> 4), flag << (2u * (uint32_t)(x & 15u)));
}

// phase-1 parent insert, priority 1 + height (:133, :390).  The rare heavy paths (hashing,
// map probes) are kept out of line so the label folds stay small in the instruction cache.
__device__ __noinline__ void insert_first_parent(const ForestArgs& a, uint32_t x, const Digest& d) {
  const uint32_t height = a.D - node_level(x);
  const unsigned long long v = ((unsigned long long)(1u + height) << 32) | x;
  const MapRef ref = map_insert(a.map, d, v, a.cur, a.st);
  if (ref.found && !ref.inserted) map_merge_current(a.map, ref.slot, v, a.cur);
}

// Phase-1 parents are inserted together at the end of a band (or warp task), up to FF_GROUP
// per thread at once.  B2D_FF_GROUPED 1: map_insert_group (all home reads, then all claims in
// flight together); 0: one insert after another, each waiting for a DRAM read of its home slot
// and then its atomics.  Measured with groups of 2: forest 0.173 against 0.176 ms per 4 GiB
// step, batched step 12.67 against 12.87 ms; groups of 4 spill registers.  Prefetching each
// group's home slots into L2 before inserting them one at a time was slower (0.185 ms and 13.30
// ms; on the MD5 series 1.68 against 1.44 ms of forest per step).
#ifndef B2D_FF_GROUPED
#define B2D_FF_GROUPED 1
#endif
constexpr int FF_GROUP = 2;
__device__ __forceinline__ void insert_first_parents(const ForestArgs& a, const uint32_t (&x)[FF_GROUP],
                                                     const Digest (&d)[FF_GROUP], uint32_t cnt) {
#if B2D_FF_GROUPED
  Key128 k[FF_GROUP];
  unsigned long long pv[FF_GROUP];
  MapRef r[FF_GROUP];
#pragma unroll
  for (int j = 0; j < FF_GROUP; j++) {
    k[j] = digest_key(d[j]);
    pv[j] = map_pack(((unsigned long long)(1u + a.D - node_level(x[j])) << 32) | x[j], a.cur);
  }
  map_insert_group<FF_GROUP>(a.map, k, pv, cnt, r, a.st);
#pragma unroll
  for (int j = 0; j < FF_GROUP; j++)
    if ((uint32_t)j < cnt && r[j].found && !r[j].inserted)
      map_merge_current(a.map, r[j].slot, ((unsigned long long)(1u + a.D - node_level(x[j])) << 32) | x[j], a.cur);
#else
#pragma unroll
  for (int j = 0; j < FF_GROUP; j++)
    if ((uint32_t)j < cnt) insert_first_parent(a, x[j], d[j]);
#endif
}

__device__ __noinline__ void hash_first_parent(const ForestArgs& a, uint32_t x) {
  const Digest d = hash_pair(a.kind, a.tree[2u * x + 1u], a.tree[2u * x + 2u]);
  a.tree[x] = d;
  insert_first_parent(a, x, d);
}

// two shifted children: the parent is a shifted duplicate only if its digest is already known;
// the baseline tests the stale (zero) digest instead (:202 vs :459)
__device__ __noinline__ uint8_t shift_pair(const ForestArgs& a, uint32_t x) {
  const uint32_t l = 2u * x + 1u, r = 2u * x + 2u;
  bool exists;
  if (a.baseline) {
    exists = *a.zero_exists != 0;
  } else {
    const Digest d = hash_pair(a.kind, a.tree[l], a.tree[r]);
    a.tree[x] = d;
    exists = map_find(a.map, d) <= a.map.cap;
  }
  if (exists) return SHIFT_DUPL;
  push_set(a.push, l, PUSH_SHIFT);
  push_set(a.push, r, PUSH_SHIFT);
  return DONE;
}

// baseline "Insert entries" (:218-224) for a parent that is not a first occurrence (those were
// hashed and inserted by phase 1 with a lower priority, so re-inserting them changes nothing):
// hash, insert with priority 64 + height
__device__ __noinline__ void baseline_parent(const ForestArgs& a, uint32_t x) {
  const Digest d = hash_pair(a.kind, a.tree[2u * x + 1u], a.tree[2u * x + 2u]);
  a.tree[x] = d;
  const uint32_t height = a.D - node_level(x);
  const unsigned long long v = ((unsigned long long)(64u + height) << 32) | x;
  const MapRef ref = map_insert(a.map, d, v, a.cur, a.st);
  if (ref.found && !ref.inserted) map_merge_current(a.map, ref.slot, v, a.cur);
}

template <int PHASE>
__device__ __forceinline__ uint8_t forest_node(const ForestArgs& a, uint32_t x, uint8_t ll, uint8_t rl) {
  if constexpr (PHASE == 1) {
    if (ll == FIRST_OCUR && rl == FIRST_OCUR) {
      hash_first_parent(a, x);
      return FIRST_OCUR;
    }
    return DONE;
  } else {
    uint8_t out;
    if (ll != rl) {
      out = DONE;
      const uint8_t pl = push_flag(ll), pr = push_flag(rl);
      if (pl) push_set(a.push, 2u * x + 1u, pl);
      if (pr) push_set(a.push, 2u * x + 2u, pr);
    } else if (ll == SHIFT_DUPL) {
      out = shift_pair(a, x);
    } else {
      out = ll;   // FIXED, FIRST or DONE pairs keep the label
    }
    if (a.baseline && out != FIRST_OCUR) baseline_parent(a, x);
    return out;
  }
}

// label of a leaf as seen by this phase: phase 1 applies the lowest-index relabel to the
// few first occurrences the leaf stage flagged as sharing their digest; every other first
// occurrence is already its digest's owner
template <int PHASE>
__device__ __forceinline__ uint8_t leaf_view(const ForestArgs& a, uint32_t x, uint8_t lab) {
  if constexpr (PHASE == 1) {
    const uint32_t c = x - (a.n - 1u);
    if (lab == FIRST_OCUR && a.dupflag[c]) {
      a.dupflag[c] = 0;
      const uint64_t slot = map_find(a.map, a.tree[x]);
      if (slot <= a.map.cap) {
        if (map_tree(a.map, slot) == a.cur && map_node(a.map, slot) != x) {
          lab = SHIFT_DUPL;
          a.leaflab[c] = lab;
        }
      } else {
        set_error(a.st, DERR_INTERNAL, 10);
      }
    }
  }
  return lab;
}
template <int PHASE>
__device__ __forceinline__ uint8_t forest_leaf(const ForestArgs& a, uint32_t x) {
  return leaf_view<PHASE>(a, x, a.leaflab[x - (a.n - 1u)]);
}

// label of node x given its children's labels: absent node, leaf (level D-1 leaves of a tree
// whose chunk count is not a power of two), or inner node
template <int PHASE>
__device__ __forceinline__ uint8_t combine(const ForestArgs& a, uint64_t x, uint8_t ll, uint8_t rl) {
  if (x >= a.N) return NONE_LABEL;
  if (x >= (uint64_t)a.n - 1u) return forest_leaf<PHASE>(a, (uint32_t)x);
  return forest_node<PHASE>(a, (uint32_t)x, ll, rl);
}

// label of an input node of a band: a leaf, or the output of the band below
template <int PHASE>
__device__ __forceinline__ uint8_t input_label(const ForestArgs& a, uint64_t x) {
  if (x >= a.N) return NONE_LABEL;
  if (x >= (uint64_t)a.n - 1u) return forest_leaf<PHASE>(a, (uint32_t)x);
  return a.lab[x];
}

// band output: hand the label to the next band, or settle the whole-tree region at the root
// (first = [0] when the root is a first occurrence, :127-129 / :392-399)
template <int PHASE>
__device__ __forceinline__ void band_output(const ForestArgs& a, uint64_t x, uint8_t lab) {
  if (x == 0) {
    if (PHASE == 2 && a.n >= 2u && lab == FIRST_OCUR) push_set(a.push, 0, PUSH_FIRST);
  } else if (x < (uint64_t)a.n - 1u) {
    a.lab[x] = lab;
  }
}

// pair-AND of a bit mask: bit j of the result = bits 2j and 2j+1 of m (m has 2w bits)
__device__ __forceinline__ uint32_t pair_and(uint32_t m, int w) {
  uint32_t r = 0;
#pragma unroll
  for (int j = 0; j < 8; j++)
    if (j < w) r |= ((m >> (2 * j)) & (m >> (2 * j + 1)) & 1u) << j;
  return r;
}

// Phase-1 band: 10 levels above the inputs at level `in` (1024 inputs per CTA of 256 threads:
// 2 levels in registers, 5 by warp shuffles, 3 through shared memory).  A parent is a first
// occurrence iff both children are; its digest is computed where its label is, from the
// children's digests held in registers (shuffled between lanes), so a run of new chunks costs
// one hash per node with no memory round trip between levels.  The parents found are recorded
// in a per-CTA bit set and inserted into the map at the end, spread evenly over the threads.
constexpr uint32_t FF_LEVELS = 10;
constexpr uint32_t FF_WORDS = 32;          // 1023 bits: band heights 1..10
__device__ __forceinline__ uint32_t ff_base(uint32_t k) {   // first bit of band height k
  return 1024u - (2048u >> k);
}
__device__ __forceinline__ void ff_set(uint32_t* ff, uint32_t k, uint32_t i) {
  const uint32_t bit = ff_base(k) + i;
  atomicOr(&ff[bit >> 5], 1u << (bit & 31u));
}
__device__ __forceinline__ Digest shfl_down_digest(const Digest& d, uint32_t delta) {
  Digest r;
#pragma unroll
  for (int k = 0; k < 4; k++) r.w[k] = __shfl_down_sync(0xffffffffu, d.w[k], delta);
  return r;
}

__device__ __forceinline__ void forest_first_body(const ForestArgs& a, uint32_t bid, uint32_t in) {
  __shared__ uint32_t ff[FF_WORDS];
  __shared__ uint32_t wbit[FAST_THREADS / 32];
  __shared__ Digest wdig[FAST_THREADS / 32];
  __shared__ uint32_t wpre[FF_WORDS + 1];
  const uint32_t t = threadIdx.x, lane = t & 31u, warp = t >> 5;
  if (t < FF_WORDS) ff[t] = 0;
  __syncthreads();
  const uint64_t root = ((1ull << (in - FF_LEVELS)) - 1ull) + bid;
  const uint64_t x0 = (root << FF_LEVELS) + ((1ull << FF_LEVELS) - 1ull) + 4ull * t;
  const uint64_t p0 = (x0 - 1ull) >> 1;
  uint32_t m0 = 0;   // first-occurrence inputs
  const bool aligned = in == a.D && (a.n & (a.n - 1u)) == 0;
  if (aligned) {
    // power-of-two leaf count, leaf band: inputs are chunks 4t.. of this CTA's 1024
    const uint32_t w = *reinterpret_cast<const uint32_t*>(a.leaflab + (x0 - (a.n - 1u)));
    const uint32_t z = ~(((w & 0x7f7f7f7fu) + 0x7f7f7f7fu) | w | 0x7f7f7f7fu);   // exact: byte == FIRST (0)
    m0 = ((z >> 7) & 1u) | ((z >> 14) & 2u) | ((z >> 21) & 4u) | ((z >> 28) & 8u);
    if (m0) {   // lowest-index relabel of the first occurrences flagged by the leaf stage
#pragma unroll
      for (int j = 0; j < 4; j++)
        if ((m0 >> j) & 1u)
          if (leaf_view<1>(a, (uint32_t)(x0 + j), FIRST_OCUR) != FIRST_OCUR) m0 &= ~(1u << j);
    }
  } else {
#pragma unroll
    for (int j = 0; j < 4; j++) m0 |= (uint32_t)(input_label<1>(a, x0 + j) == FIRST_OCUR) << j;
  }
  // no first occurrence among the inputs: nothing to hash or insert, the band root is DONE
  // (unless level D-1 holds leaves, which the first band of a non-power-of-two tree reads below)
  if ((aligned || in < a.D) && !__syncthreads_or(m0 != 0u)) {
    if (t == 0) band_output<1>(a, root, DONE);
    return;
  }
  // band height 1: nodes p0, p0 + 1
  Digest d1[2];
  uint32_t m1 = 0;
#pragma unroll
  for (int j = 0; j < 2; j++) {
    const uint64_t p = p0 + j;
    d1[j].w[0] = d1[j].w[1] = d1[j].w[2] = d1[j].w[3] = 0u;
    if (!aligned && p >= a.N) continue;
    if (!aligned && p >= (uint64_t)a.n - 1u) {   // a leaf on level D-1 (chunk count not a power of two)
      if (forest_leaf<1>(a, (uint32_t)p) == FIRST_OCUR) {
        d1[j] = a.tree[p];
        m1 |= 1u << j;
      }
      continue;
    }
    if (((m0 >> (2 * j)) & 3u) == 3u) {
      d1[j] = hash_pair(a.kind, a.tree[x0 + 2 * j], a.tree[x0 + 2 * j + 1]);
      a.tree[p] = d1[j];
      m1 |= 1u << j;
      ff_set(ff, 1, 2u * t + j);
    }
  }
  // band height 2: node (root << 8) + 255 + t
  uint64_t y = (p0 - 1ull) >> 1;
  uint32_t b = 0;
  Digest dg;
  dg.w[0] = dg.w[1] = dg.w[2] = dg.w[3] = 0u;
  if (m1 == 3u) {
    dg = hash_pair(a.kind, d1[0], d1[1]);
    a.tree[y] = dg;
    b = 1;
    ff_set(ff, 2, t);
  }
  // band heights 3..7: warp shuffles
  if (__any_sync(0xffffffffu, b)) {
#pragma unroll
    for (int s = 0; s < 5; s++) {
      const uint32_t rb = __shfl_down_sync(0xffffffffu, b, 1u << s);
      const Digest rd = shfl_down_digest(dg, 1u << s);
      if ((lane & ((2u << s) - 1u)) == 0) {
        y = (y - 1ull) >> 1;
        b &= rb;
        if (b) {
          dg = hash_pair(a.kind, dg, rd);
          a.tree[y] = dg;
          ff_set(ff, 3 + s, t >> (s + 1));
        }
      }
    }
  } else {
    b = 0;
  }
  if (lane == 0) {
    wbit[warp] = b;
    wdig[warp] = dg;
  }
  __syncthreads();
  // band heights 8..10: the 8 warp results
  if (warp == 0) {
    b = lane < FAST_THREADS / 32 ? wbit[lane] : 0u;
    if (lane < FAST_THREADS / 32) dg = wdig[lane];
    y = (root << 3) + 7ull + lane;
#pragma unroll
    for (int s = 0; s < 3; s++) {
      const uint32_t rb = __shfl_down_sync(0xffffffffu, b, 1u << s);
      const Digest rd = shfl_down_digest(dg, 1u << s);
      if ((lane & ((2u << s) - 1u)) == 0 && lane < FAST_THREADS / 32) {
        y = (y - 1ull) >> 1;
        b &= rb;
        if (b) {
          dg = hash_pair(a.kind, dg, rd);
          a.tree[y] = dg;
          ff_set(ff, 8 + s, lane >> (s + 1));
        }
      }
    }
    if (lane == 0) band_output<1>(a, root, b ? FIRST_OCUR : DONE);
  }
  __syncthreads();
  // inserts: rank the set bits (prefix of per-word counts), thread t takes ranks t, t+256, ...
  static_assert(FF_WORDS == 32, "one word per lane of warp 0");
  if (warp == 0) {
    uint32_t c = __popc(ff[lane]);
#pragma unroll
    for (uint32_t o = 1; o < 32; o <<= 1) {
      const uint32_t v = __shfl_up_sync(0xffffffffu, c, o);
      if (lane >= o) c += v;
    }
    wpre[lane + 1] = c;
    if (lane == 0) wpre[0] = 0;
  }
  __syncthreads();
  const uint32_t total = wpre[FF_WORDS];
  for (uint32_t r0 = t; r0 < total; r0 += FAST_THREADS * FF_GROUP) {
    uint32_t xs[FF_GROUP], c = 0;
    Digest ds[FF_GROUP];
#pragma unroll
    for (int j = 0; j < FF_GROUP; j++) {
      const uint32_t r = r0 + FAST_THREADS * j;
      xs[j] = 0;
      ds[j].w[0] = ds[j].w[1] = ds[j].w[2] = ds[j].w[3] = 0u;
      if (r >= total) continue;
      uint32_t lo = 0, hi = FF_WORDS;   // word with wpre[w] <= r < wpre[w+1]
      while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (wpre[mid] <= r) lo = mid; else hi = mid;
      }
      uint32_t word = ff[lo], skip = r - wpre[lo];
      while (skip--) word &= word - 1u;   // drop the lower set bits
      const uint32_t bit = lo * 32u + (__ffs(word) - 1u);
      uint32_t k = 1;                     // band height of this bit
      while (k < FF_LEVELS && bit >= ff_base(k + 1)) k++;
      const uint64_t first = (root << (FF_LEVELS - k)) + (1ull << (FF_LEVELS - k)) - 1ull;
      xs[j] = (uint32_t)(first + (bit - ff_base(k)));
      ds[j] = a.tree[xs[j]];
      c = j + 1;
    }
    insert_first_parents(a, xs, ds, c);
  }
}
// The first band of a phase has one band per 1024 (phase 1) or 4096 (phase 2) leaves, most of
// them without work at low change rates.  With B2D_FOREST_PERSIST the launch is one resident
// grid whose CTAs take bands in turn (a barrier between bands: shared memory is reused), so
// tens of thousands of short-lived CTAs are not scheduled one by one.
#ifndef B2D_FOREST_PERSIST
#define B2D_FOREST_PERSIST 1
#endif
__global__ void __launch_bounds__(FAST_THREADS, B2D_FF_MINB) forest_first_kernel(ForestArgs a0, uint32_t in,
                                                                                  uint32_t nbands) {
  griddep_enter();
  const ForestArgs a = with_round(a0);
  for (uint32_t bid = blockIdx.x; bid < nbands; bid += gridDim.x) {
    forest_first_body(a, bid, in);
    __syncthreads();
  }
}
__global__ void __launch_bounds__(FAST_THREADS, B2D_FF_MINB) forest_first_seg(ForestSeg s) {
  uint32_t bid, nb;
  const uint32_t h = seg_find(s.beg, s.n, bid, nb);
  forest_first_body(with_round(s.args[h]), bid, s.p0[h]);
}

// Fast band: inputs at level `in`, outputs at level in - 12.
template <int PHASE>
__device__ __forceinline__ void forest_fast_body(const ForestArgs& a, uint32_t bid, uint32_t in) {
  __shared__ uint8_t wlab[FAST_THREADS / 32];
  const uint32_t t = threadIdx.x, lane = t & 31u, warp = t >> 5;
  const uint64_t root = ((1ull << (in - FAST_LEVELS)) - 1ull) + bid;
  const uint64_t x0 = (root << FAST_LEVELS) + ((1ull << FAST_LEVELS) - 1ull) + 16ull * t;
  uint8_t v[16];
  bool fast = !a.baseline;
  if (in == a.D && (a.n & (a.n - 1u)) == 0) {
    // power-of-two leaf count, leaf band: the 16 inputs are chunks 16t.. of this CTA's 4096,
    // one aligned 16-byte load; FIXED = 0x01 bytes, FIRST = 0x00 bytes
    const uint4 w = *reinterpret_cast<const uint4*>(a.leaflab + (x0 - (a.n - 1u)));
    if (PHASE == 2) {
      fast = fast && w.x == 0x01010101u && w.y == 0x01010101u && w.z == 0x01010101u && w.w == 0x01010101u;
    } else {
      const uint32_t zx = (w.x - 0x01010101u) & ~w.x, zy = (w.y - 0x01010101u) & ~w.y;
      const uint32_t zz = (w.z - 0x01010101u) & ~w.z, zw = (w.w - 0x01010101u) & ~w.w;
      fast = fast && (((zx | zy | zz | zw) & 0x80808080u) == 0);   // no zero byte at all: no FIRST
    }
    if (!fast) {
      const uint32_t ws[4] = {w.x, w.y, w.z, w.w};
#pragma unroll
      for (int j = 0; j < 16; j++) v[j] = leaf_view<PHASE>(a, (uint32_t)(x0 + j), (uint8_t)(ws[j >> 2] >> (8 * (j & 3))));
    }
  } else {
#pragma unroll
    for (int j = 0; j < 16; j++) v[j] = input_label<PHASE>(a, x0 + j);
#pragma unroll
    for (int j = 0; j < 16; j++) {
      if (PHASE == 2) fast = fast && v[j] == FIXED_DUPL;
      else fast = fast && v[j] != FIRST_OCUR && v[j] != NONE_LABEL;
    }
  }
  // every input of the band unchanged (phase 2: all FIXED; phase 1: no first occurrence): the
  // whole subtree folds to one label without further work
  if (!__syncthreads_or(!fast)) {
    if (t == 0) band_output<PHASE>(a, root, PHASE == 2 ? FIXED_DUPL : DONE);
    return;
  }
  uint8_t lab;
  if (fast) {
    lab = PHASE == 2 ? FIXED_DUPL : DONE;
  } else {
    uint64_t first = x0;
#pragma unroll
    for (int width = 8; width >= 1; width >>= 1) {
      first = (first - 1ull) >> 1;
#pragma unroll
      for (int j = 0; j < width; j++) {
        // two FIXED children: an inner node, FIXED in an incremental checkpoint (fixed_or_node)
        if (PHASE == 2 && !a.baseline && v[2 * j] == FIXED_DUPL && v[2 * j + 1] == FIXED_DUPL) v[j] = FIXED_DUPL;
        else v[j] = combine<PHASE>(a, first + j, v[2 * j], v[2 * j + 1]);
      }
    }
    lab = v[0];
  }
  // warp: 5 levels
  uint64_t y = (root << 8) + 255ull + t;
#pragma unroll
  for (int s = 0; s < 5; s++) {
    __syncwarp();   // digests written by the partner lane at the previous level are visible
    const uint8_t rl = (uint8_t)__shfl_down_sync(0xffffffffu, (uint32_t)lab, 1u << s);
    if ((lane & ((2u << s) - 1u)) == 0) {
      y = (y - 1ull) >> 1;
      if (!(PHASE == 2 && !a.baseline && lab == FIXED_DUPL && rl == FIXED_DUPL) &&
          !(PHASE == 1 && !a.baseline && lab != FIRST_OCUR && lab != NONE_LABEL && rl != NONE_LABEL))
        lab = combine<PHASE>(a, y, lab, rl);
      else if (PHASE == 1)
        lab = DONE;
    }
  }
  if (lane == 0) wlab[warp] = lab;
  __syncthreads();
  if (warp == 0) {
    lab = lane < FAST_THREADS / 32 ? wlab[lane] : NONE_LABEL;
    y = (root << 3) + 7ull + lane;
#pragma unroll
    for (int s = 0; s < 3; s++) {
      __syncwarp();
      const uint8_t rl = (uint8_t)__shfl_down_sync(0xffffffffu, (uint32_t)lab, 1u << s);
      if ((lane & ((2u << s) - 1u)) == 0 && lane < FAST_THREADS / 32) {
        y = (y - 1ull) >> 1;
        lab = combine<PHASE>(a, y, lab, rl);
      }
    }
    if (lane == 0) band_output<PHASE>(a, root, lab);
  }
}
template <int PHASE>
__global__ void __launch_bounds__(FAST_THREADS, B2D_FAST_MINB) forest_fast_kernel(ForestArgs a0, uint32_t in,
                                                                                  uint32_t nbands) {
  griddep_enter();
  const ForestArgs a = with_round(a0);
  for (uint32_t bid = blockIdx.x; bid < nbands; bid += gridDim.x) {
    forest_fast_body<PHASE>(a, bid, in);
    __syncthreads();
  }
}
template <int PHASE>
__global__ void __launch_bounds__(FAST_THREADS, B2D_FAST_MINB) forest_fast_seg(ForestSeg s) {
  uint32_t bid, nb;
  const uint32_t h = seg_find(s.beg, s.n, bid, nb);
  forest_fast_body<PHASE>(with_round(s.args[h]), bid, s.p0[h]);
}

// Warp bands: the first band of each phase of a tree whose chunk count is a power of two, as
// independent warp tasks (no CTA barrier).  A CTA band stalls all its warps on three barriers
// per band and a CTA takes its bands one after another, so most of a band's time was load and
// barrier latency; a warp task folds its leaves in registers and by shuffles only, and each
// warp loads the next task's labels before it works on the current one.
//   phase 1: 128 leaves per task (4 per lane, one 32-bit label load), 7 levels: 2 in registers
//            (with the parents' digests), 5 by shuffles; a parent is hashed and inserted where
//            its label is decided
//   phase 2: 512 leaves per task (16 per lane, one 16-byte label load), 9 levels: 4 in
//            registers, 5 by shuffles
// A task writes its root's label to `lab` for the band above (which is a CTA band again: few
// nodes are left there).  Same per-node rules as the CTA bands, so the labels, digests, map
// entries and push flags are the same.
// Which phases start with one is a runtime mask (B2D_WARP_BANDS, the default, in dedup_kernels.cuh).
constexpr uint32_t WB1_LEVELS = 7;
constexpr uint32_t WB2_LEVELS = 9;
constexpr uint32_t WB_THREADS = 256;
// resident CTAs per SM the warp bands are compiled for (phase 1: 5, 48 registers; phase 2: 4,
// 64 registers)
#ifndef B2D_WB1_MINB
#define B2D_WB1_MINB 5
#endif
#ifndef B2D_WB2_MINB
#define B2D_WB2_MINB 4
#endif

static bool warp_bands(uint32_t n, uint32_t D, int phase, int mask) {
  return (mask & (phase == 1 ? 1 : 2)) && n >= 2u && (n & (n - 1u)) == 0 &&
         D >= (phase == 1 ? WB1_LEVELS : WB2_LEVELS);
}

// Parents a phase-1 warp task created, inserted into the map together once the task's hashing is
// done (spread over the lanes): inserting each where it is hashed put a chain of dependent map
// round trips on the lanes that carry the upper levels.  At most 127 per task of 128 leaves.
struct WarpInserts {
  uint32_t* node;   // 128 entries of this warp's buffer in shared memory
  Digest* dig;
  uint32_t* count;
};
__device__ __forceinline__ void wi_add(const WarpInserts& wi, uint32_t x, const Digest& d) {
  const uint32_t pos = atomicAdd(wi.count, 1u);
  wi.node[pos] = x;
  wi.dig[pos] = d;
}
__device__ __forceinline__ void wi_flush(const ForestArgs& a, const WarpInserts& wi, uint32_t lane) {
  __syncwarp();
  const uint32_t cnt = *wi.count;
  // lane takes entries lane, lane + 32, ... in groups of FF_GROUP
  for (uint32_t r0 = lane; r0 < cnt; r0 += 32u * FF_GROUP) {
    uint32_t x[FF_GROUP], c = 0;
    Digest d[FF_GROUP];
#pragma unroll
    for (int j = 0; j < FF_GROUP; j++) {
      const uint32_t r = r0 + 32u * j;
      x[j] = 0;
      d[j].w[0] = d[j].w[1] = d[j].w[2] = d[j].w[3] = 0u;
      if (r < cnt) {
        x[j] = wi.node[r];
        d[j] = wi.dig[r];
        c = j + 1;
      }
    }
    insert_first_parents(a, x, d, c);
  }
  __syncwarp();
  if (lane == 0) *wi.count = 0;
  __syncwarp();
}

__device__ __forceinline__ void warp1_task(const ForestArgs& a, uint32_t task, uint32_t lane, uint32_t w,
                                           const WarpInserts& wi) {
  const uint64_t root = ((1ull << (a.D - WB1_LEVELS)) - 1ull) + task;
  const uint32_t c0 = task * 128u + 4u * lane;          // first chunk of this lane
  const uint64_t x0 = (uint64_t)(a.n - 1u) + c0;        // its leaf (a left child)
  const uint32_t z = ~(((w & 0x7f7f7f7fu) + 0x7f7f7f7fu) | w | 0x7f7f7f7fu);   // exact: byte == FIRST (0)
  uint32_t m0 = ((z >> 7) & 1u) | ((z >> 14) & 2u) | ((z >> 21) & 4u) | ((z >> 28) & 8u);
  if (!__any_sync(0xffffffffu, m0 != 0u)) {
    if (lane == 0) band_output<1>(a, root, DONE);
    return;
  }
  // the leaf digests of both pairs are loaded together with the duplicate flags (a relabel
  // below only drops pairs, and rarely)
  Digest lv[4];
#pragma unroll
  for (int j = 0; j < 4; j++) lv[j].w[0] = lv[j].w[1] = lv[j].w[2] = lv[j].w[3] = 0u;
  if (m0) {
    const uint32_t df = *reinterpret_cast<const uint32_t*>(a.dupflag + c0);
#pragma unroll
    for (int j = 0; j < 2; j++)
      if (((m0 >> (2 * j)) & 3u) == 3u) {
        lv[2 * j] = a.tree[x0 + 2 * j];
        lv[2 * j + 1] = a.tree[x0 + 2 * j + 1];
      }
    if (df) {
      // lowest-index relabel of the first occurrences the leaf stage flagged as sharing a digest
#pragma unroll
      for (int j = 0; j < 4; j++)
        if ((m0 >> j) & 1u)
          if (leaf_view<1>(a, (uint32_t)(x0 + j), FIRST_OCUR) != FIRST_OCUR) m0 &= ~(1u << j);
    }
  }
  // height 1: nodes p0, p0 + 1; height 2: node y
  const uint64_t p0 = (x0 - 1ull) >> 1;
  Digest d1[2];
  uint32_t m1 = 0;
#pragma unroll
  for (int j = 0; j < 2; j++) {
    d1[j].w[0] = d1[j].w[1] = d1[j].w[2] = d1[j].w[3] = 0u;
    if (((m0 >> (2 * j)) & 3u) == 3u) {
      d1[j] = hash_pair(a.kind, lv[2 * j], lv[2 * j + 1]);
      a.tree[p0 + j] = d1[j];
      wi_add(wi, (uint32_t)(p0 + j), d1[j]);
      m1 |= 1u << j;
    }
  }
  uint64_t y = (p0 - 1ull) >> 1;
  uint32_t b = 0;
  Digest dg;
  dg.w[0] = dg.w[1] = dg.w[2] = dg.w[3] = 0u;
  if (m1 == 3u) {
    dg = hash_pair(a.kind, d1[0], d1[1]);
    a.tree[y] = dg;
    wi_add(wi, (uint32_t)y, dg);
    b = 1;
  }
  // heights 3..7: shuffles; lane 0 ends at the task root
  if (__any_sync(0xffffffffu, b)) {
#pragma unroll
    for (int s = 0; s < 5; s++) {
      const uint32_t rb = __shfl_down_sync(0xffffffffu, b, 1u << s);
      const Digest rd = shfl_down_digest(dg, 1u << s);
      if ((lane & ((2u << s) - 1u)) == 0) {
        y = (y - 1ull) >> 1;
        b &= rb;
        if (b) {
          dg = hash_pair(a.kind, dg, rd);
          a.tree[y] = dg;
          wi_add(wi, (uint32_t)y, dg);
        }
      }
    }
  } else {
    b = 0;
  }
  if (lane == 0) band_output<1>(a, root, b ? FIRST_OCUR : DONE);
  wi_flush(a, wi, lane);
}

// Phase-2 parent of two FIXED children in an incremental checkpoint: FIXED, with nothing pushed
// or looked up, so the call is skipped.  A task of 512 leaves almost always holds a few scattered
// shifted copies (0.5 % of the plain series' chunks), so most tasks take the slow path, and most
// of their nodes are still FIXED pairs.
__device__ __forceinline__ uint8_t fixed_or_node(const ForestArgs& a, uint32_t x, uint8_t ll, uint8_t rl) {
  if (!a.baseline && ll == FIXED_DUPL && rl == FIXED_DUPL) return FIXED_DUPL;
  return forest_node<2>(a, x, ll, rl);
}

__device__ __forceinline__ void warp2_task(const ForestArgs& a, uint32_t task, uint32_t lane, const uint4& w) {
  const uint64_t root = ((1ull << (a.D - WB2_LEVELS)) - 1ull) + task;
  const uint32_t c0 = task * 512u + 16u * lane;
  const uint64_t x0 = (uint64_t)(a.n - 1u) + c0;
  bool fast = !a.baseline && w.x == 0x01010101u && w.y == 0x01010101u && w.z == 0x01010101u &&
              w.w == 0x01010101u;   // all 16 leaves FIXED
  if (__all_sync(0xffffffffu, fast)) {
    if (lane == 0) band_output<2>(a, root, FIXED_DUPL);
    return;
  }
  uint8_t lab = FIXED_DUPL;
  if (!fast) {
    uint8_t v[16];
    const uint32_t ws[4] = {w.x, w.y, w.z, w.w};
#pragma unroll
    for (int j = 0; j < 16; j++) v[j] = (uint8_t)(ws[j >> 2] >> (8 * (j & 3)));
    uint64_t first = x0;
#pragma unroll
    for (int width = 8; width >= 1; width >>= 1) {
      first = (first - 1ull) >> 1;
#pragma unroll
      for (int j = 0; j < width; j++) v[j] = fixed_or_node(a, (uint32_t)(first + j), v[2 * j], v[2 * j + 1]);
    }
    lab = v[0];
  }
  uint64_t y = ((x0 + 1ull) >> 4) - 1ull;   // the lane's 16-leaf subtree root
#pragma unroll
  for (int s = 0; s < 5; s++) {
    __syncwarp();   // digests written by the partner lane at the previous level are visible
    const uint8_t rl = (uint8_t)__shfl_down_sync(0xffffffffu, (uint32_t)lab, 1u << s);
    if ((lane & ((2u << s) - 1u)) == 0) {
      y = (y - 1ull) >> 1;
      if (a.baseline || lab != FIXED_DUPL || rl != FIXED_DUPL) lab = forest_node<2>(a, (uint32_t)y, lab, rl);
    }
  }
  if (lane == 0) band_output<2>(a, root, lab);
}

// Resident grid of warps over the tasks.  B2D_WARP_QUEUE 1 (default): two passes per CTA.
//   scan: warp w of the grid tests tasks w, w + G, w + 2G, ... four at a time (their labels
//         loaded while the previous four are handled), writes the output of every task without
//         work and queues the others in the CTA's shared memory;
//   work: after one CTA barrier the CTA's 8 warps take the queued tasks in turn.
// A run of changed chunks covers consecutive tasks, which the stride spreads over warps, and
// the queue evens out each CTA's share of work tasks over its warps: with one fixed task per
// warp and step, a launch waited for the warps that drew the most work.  Groups of consecutive
// tasks taken from a global counter measured slower than either (a run's tasks then fall to one
// warp).  Where a CTA's tasks could overflow its queue (more than WB_QUEUE, from 2^27 chunks at
// a resident grid) and with B2D_WARP_QUEUE 0, warp w runs tasks w, w + G, ... itself, the next
// one's labels loaded first.
#ifndef B2D_WARP_QUEUE
#define B2D_WARP_QUEUE 1
#endif
constexpr uint32_t WB_QUEUE = 1024;   // queued tasks per CTA
constexpr uint32_t WB_SCAN = 4;       // tasks tested per scan step of a warp
constexpr uint32_t WB_FULL = 0xffffffffu;

#define B2D_WARP_INSERT_BUFFERS                                                                 \
  __shared__ uint32_t wi_node_[WB_THREADS / 32u][128];                                          \
  __shared__ Digest wi_dig_[WB_THREADS / 32u][128];                                             \
  __shared__ uint32_t wi_count_[WB_THREADS / 32u];                                              \
  const WarpInserts wi{wi_node_[threadIdx.x >> 5], wi_dig_[threadIdx.x >> 5], &wi_count_[threadIdx.x >> 5]}; \
  if ((threadIdx.x & 31u) == 0) *wi.count = 0;                                                  \
  __syncwarp();

// the CTA's task queue: entries, reserved count, taken count
#define B2D_WARP_QUEUE_BUFFERS                                                                  \
  __shared__ uint32_t wq_[WB_QUEUE];                                                            \
  __shared__ uint32_t wq_n_, wq_h_;                                                             \
  if (threadIdx.x == 0) {                                                                       \
    wq_n_ = 0;                                                                                  \
    wq_h_ = 0;                                                                                  \
  }                                                                                             \
  __syncthreads();

__device__ __forceinline__ bool has_zero_byte(uint32_t w) {
  return ((w - 0x01010101u) & ~w & 0x80808080u) != 0u;
}
// lane 0 queues `task` (the launch guarantees room: at most WB_QUEUE tasks per CTA)
__device__ __forceinline__ void wq_push(uint32_t* q, uint32_t* n, uint32_t task, uint32_t lane) {
  if (lane == 0) {
    const uint32_t pos = atomicAdd(n, 1u);
    if (pos < WB_QUEUE) q[pos] = task;
  }
}
// next queued task for this warp, or ~0 once the queue is drained
__device__ __forceinline__ uint32_t wq_pop(const uint32_t* q, uint32_t* h, uint32_t n, uint32_t lane) {
  uint32_t i = 0;
  if (lane == 0) i = atomicAdd(h, 1u);
  i = __shfl_sync(WB_FULL, i, 0);
  return i < (n < WB_QUEUE ? n : WB_QUEUE) ? q[i] : ~0u;
}
// tasks of one CTA of a resident grid of `grid` CTAs fit its queue
static bool wq_fits(uint32_t ntasks, uint32_t grid) {
  const uint64_t warps = (uint64_t)grid * (WB_THREADS / 32u);
  return B2D_WARP_QUEUE && ((uint64_t)ntasks + warps - 1u) / warps * (WB_THREADS / 32u) <= WB_QUEUE;
}

__global__ void __launch_bounds__(WB_THREADS, B2D_WB1_MINB)
    forest_warp1_kernel(ForestArgs a0, uint32_t ntasks, uint32_t queue) {
  griddep_enter();
  B2D_WARP_INSERT_BUFFERS
  B2D_WARP_QUEUE_BUFFERS
  const ForestArgs a = with_round(a0);
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t G = (gridDim.x * WB_THREADS) >> 5;
  const uint32_t w0 = (blockIdx.x * WB_THREADS + threadIdx.x) >> 5;
  const uint32_t* lab32 = reinterpret_cast<const uint32_t*>(a.leaflab);
  if (!queue) {
    uint32_t w = w0 < ntasks ? lab32[w0 * 32u + lane] : 0u;
    for (uint32_t task = w0; task < ntasks; task += G) {
      const uint32_t next = task + G;
      const uint32_t wn = next < ntasks ? lab32[next * 32u + lane] : 0u;
      warp1_task(a, task, lane, w, wi);
      w = wn;
    }
    return;
  }
  const uint64_t root0 = (1ull << (a.D - WB1_LEVELS)) - 1ull;
  uint32_t wn[WB_SCAN];
#pragma unroll
  for (uint32_t k = 0; k < WB_SCAN; k++) {
    const uint32_t t = w0 + k * G;
    wn[k] = t < ntasks ? lab32[t * 32u + lane] : 0x01010101u;
  }
  for (uint32_t t0 = w0; t0 < ntasks; t0 += WB_SCAN * G) {
    uint32_t work = 0;   // bit k: task t0 + kG holds a first occurrence
#pragma unroll
    for (uint32_t k = 0; k < WB_SCAN; k++)
      if (__any_sync(WB_FULL, has_zero_byte(wn[k]))) work |= 1u << k;
#pragma unroll
    for (uint32_t k = 0; k < WB_SCAN; k++) {
      const uint32_t t = t0 + (WB_SCAN + k) * G;
      wn[k] = t < ntasks ? lab32[t * 32u + lane] : 0x01010101u;
    }
#pragma unroll
    for (uint32_t k = 0; k < WB_SCAN; k++) {
      const uint32_t t = t0 + k * G;
      if (t >= ntasks) break;
      if ((work >> k) & 1u) wq_push(wq_, &wq_n_, t, lane);
      else if (lane == 0) band_output<1>(a, root0 + t, DONE);
    }
  }
  __syncthreads();
  const uint32_t qn = wq_n_;
  for (uint32_t t = wq_pop(wq_, &wq_h_, qn, lane); t != ~0u; t = wq_pop(wq_, &wq_h_, qn, lane))
    warp1_task(a, t, lane, lab32[t * 32u + lane], wi);
}
__global__ void __launch_bounds__(WB_THREADS, B2D_WB2_MINB)
    forest_warp2_kernel(ForestArgs a0, uint32_t ntasks, uint32_t queue) {
  griddep_enter();
  B2D_WARP_QUEUE_BUFFERS
  const ForestArgs a = with_round(a0);
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t G = (gridDim.x * WB_THREADS) >> 5;
  const uint32_t w0 = (blockIdx.x * WB_THREADS + threadIdx.x) >> 5;
  const uint4* lab128 = reinterpret_cast<const uint4*>(a.leaflab);
  if (!queue) {
    uint4 w = w0 < ntasks ? lab128[w0 * 32u + lane] : make_uint4(0, 0, 0, 0);
    for (uint32_t task = w0; task < ntasks; task += G) {
      const uint32_t next = task + G;
      const uint4 wn = next < ntasks ? lab128[next * 32u + lane] : make_uint4(0, 0, 0, 0);
      warp2_task(a, task, lane, w);
      w = wn;
    }
    return;
  }
  const uint64_t root0 = (1ull << (a.D - WB2_LEVELS)) - 1ull;
  const uint4 fixed4 = make_uint4(0x01010101u, 0x01010101u, 0x01010101u, 0x01010101u);
  uint4 wn[WB_SCAN];
#pragma unroll
  for (uint32_t k = 0; k < WB_SCAN; k++) {
    const uint32_t t = w0 + k * G;
    wn[k] = t < ntasks ? lab128[t * 32u + lane] : fixed4;
  }
  for (uint32_t t0 = w0; t0 < ntasks; t0 += WB_SCAN * G) {
    uint32_t work = 0;   // bit k: task t0 + kG has a leaf that is not FIXED (every task of a baseline)
#pragma unroll
    for (uint32_t k = 0; k < WB_SCAN; k++) {
      const bool fast = !a.baseline && wn[k].x == 0x01010101u && wn[k].y == 0x01010101u &&
                        wn[k].z == 0x01010101u && wn[k].w == 0x01010101u;
      if (!__all_sync(WB_FULL, fast)) work |= 1u << k;
    }
#pragma unroll
    for (uint32_t k = 0; k < WB_SCAN; k++) {
      const uint32_t t = t0 + (WB_SCAN + k) * G;
      wn[k] = t < ntasks ? lab128[t * 32u + lane] : fixed4;
    }
#pragma unroll
    for (uint32_t k = 0; k < WB_SCAN; k++) {
      const uint32_t t = t0 + k * G;
      if (t >= ntasks) break;
      if ((work >> k) & 1u) wq_push(wq_, &wq_n_, t, lane);
      else if (lane == 0) band_output<2>(a, root0 + t, FIXED_DUPL);
    }
  }
  __syncthreads();
  const uint32_t qn = wq_n_;
  for (uint32_t t = wq_pop(wq_, &wq_h_, qn, lane); t != ~0u; t = wq_pop(wq_, &wq_h_, qn, lane))
    warp2_task(a, t, lane, lab128[t * 32u + lane]);
}

// Segmented warp bands (batched form): CTA b of a handle's range holds its tasks 8b .. 8b+7,
// one per warp.
__global__ void __launch_bounds__(WB_THREADS) forest_warp1_seg(ForestSeg s) {
  B2D_WARP_INSERT_BUFFERS
  uint32_t bid, nb;
  const uint32_t h = seg_find(s.beg, s.n, bid, nb);
  const ForestArgs a = with_round(s.args[h]);
  const uint32_t task = bid * (WB_THREADS / 32u) + (threadIdx.x >> 5);
  if (task >= (a.n >> WB1_LEVELS)) return;
  const uint32_t lane = threadIdx.x & 31u;
  warp1_task(a, task, lane, reinterpret_cast<const uint32_t*>(a.leaflab)[task * 32u + lane], wi);
}
__global__ void __launch_bounds__(WB_THREADS) forest_warp2_seg(ForestSeg s) {
  uint32_t bid, nb;
  const uint32_t h = seg_find(s.beg, s.n, bid, nb);
  const ForestArgs a = with_round(s.args[h]);
  const uint32_t task = bid * (WB_THREADS / 32u) + (threadIdx.x >> 5);
  if (task >= (a.n >> WB2_LEVELS)) return;
  const uint32_t lane = threadIdx.x & 31u;
  warp2_task(a, task, lane, reinterpret_cast<const uint4*>(a.leaflab)[task * 32u + lane]);
}

// General band: levels [top, bot] (top <= bot <= D), level by level through shared memory.
// Nodes at level `bot` are leaves or combine children at level bot+1 read from `lab`.
template <int PHASE>
__device__ __forceinline__ void forest_band_body(const ForestArgs& a, uint32_t bid, uint32_t top, uint32_t bot) {
  __shared__ uint8_t buf[2][1u << (FOREST_BAND_LEVELS - 1)];
  const uint32_t H = bot - top;
  const uint64_t root = ((1ull << top) - 1ull) + bid;
  uint8_t* below = buf[0];
  uint8_t* here = buf[1];
  for (int k = (int)H; k >= 0; k--) {
    const uint64_t width = 1ull << k;
    const uint64_t base = (root << k) + width - 1ull;
    for (uint64_t i = threadIdx.x; i < width; i += blockDim.x) {
      const uint64_t x = base + i;
      uint8_t lab;
      if (k == (int)H) {
        if (x >= a.N || x >= (uint64_t)a.n - 1u) lab = input_label<PHASE>(a, x);
        else lab = combine<PHASE>(a, x, a.lab[2 * x + 1], a.lab[2 * x + 2]);
      } else {
        lab = combine<PHASE>(a, x, below[2 * i], below[2 * i + 1]);
      }
      if (k > 0) here[i] = lab;
      else band_output<PHASE>(a, x, lab);
    }
    __syncthreads();
    uint8_t* t = below;
    below = here;
    here = t;
  }
}
template <int PHASE>
__global__ void __launch_bounds__(FOREST_THREADS) forest_band_kernel(ForestArgs a0, uint32_t top, uint32_t bot) {
  griddep_enter();
  forest_band_body<PHASE>(with_round(a0), blockIdx.x, top, bot);
}
template <int PHASE>
__global__ void __launch_bounds__(FOREST_THREADS) forest_band_seg(ForestSeg s) {
  uint32_t bid, nb;
  const uint32_t h = seg_find(s.beg, s.n, bid, nb);
  forest_band_body<PHASE>(with_round(s.args[h]), bid, s.p0[h], s.p1[h]);
}

static uint32_t band_levels(int phase) { return phase == 1 ? FF_LEVELS : FAST_LEVELS; }

// The launches of one phase for a tree of depth D whose labels at level `in` are known (the
// leaves, in = D, or a warp band's outputs): full bands of band_levels(phase) levels up from
// `in` (kind 0, p0 = input level), then general bands of up to FOREST_BAND_LEVELS levels
// (kind 1, p0 = top, p1 = bottom level) for what is left above.
static void forest_steps_from(uint32_t D, uint32_t in, uint64_t N, int phase, std::vector<ForestStep>& out) {
  out.clear();
  if (N <= 1) return;   // one chunk: no inner nodes; the reference never pushes a region
  const uint32_t L = band_levels(phase);
  while (in >= L) {
    out.push_back(ForestStep{0, in, 0, 1u << (in - L)});
    in -= L;
  }
  if (in == 0) return;  // the root was a full band's output
  // remaining levels [0, bot]: bot = D when no full band ran (start from the leaves), else in-1
  int bot = (in == D) ? (int)D : (int)in - 1;
  while (bot >= 0) {
    int top = bot - (int)FOREST_BAND_LEVELS + 1;
    if (top < 0) top = 0;
    out.push_back(ForestStep{1, (uint32_t)top, (uint32_t)bot, 1u << top});
    bot = top - 1;
  }
}
void forest_steps(uint32_t D, uint64_t N, int phase, std::vector<ForestStep>& out) {
  forest_steps_from(D, D, N, phase, out);
}
void forest_steps_batch(uint32_t n, uint32_t D, uint64_t N, int phase, std::vector<ForestStep>& out,
                        int warp_mask) {
  if (!warp_bands(n, D, phase, warp_mask)) {
    forest_steps(D, N, phase, out);
    return;
  }
  const uint32_t levels = phase == 1 ? WB1_LEVELS : WB2_LEVELS;
  std::vector<ForestStep> rest;
  forest_steps_from(D, D - levels, N, phase, rest);
  out.clear();
  out.push_back(ForestStep{2, D, 0, ((n >> levels) + WB_THREADS / 32u - 1u) / (WB_THREADS / 32u)});
  out.insert(out.end(), rest.begin(), rest.end());
}

// resident CTAs per SM of a first-band kernel (queried once)
template <class K>
static uint32_t resident_ctas(K kernel) {
  int nb = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kernel, FAST_THREADS, 0) != cudaSuccess || nb < 1) {
    (void)cudaGetLastError();
    nb = 1;
  }
  return (uint32_t)nb;
}

cudaError_t launch_forest(const ForestArgs& a, int phase, cudaStream_t stream, int sm_count, int warp_mask) {
  static const uint32_t res_first = resident_ctas(forest_first_kernel);
  static const uint32_t res_fast = resident_ctas(forest_fast_kernel<2>);
  std::vector<ForestStep> steps;
  if (warp_bands(a.n, a.D, phase, warp_mask)) {
    static const uint32_t res_w1 = resident_ctas(forest_warp1_kernel);
    static const uint32_t res_w2 = resident_ctas(forest_warp2_kernel);
    const uint32_t levels = phase == 1 ? WB1_LEVELS : WB2_LEVELS;
    const uint32_t ntasks = a.n >> levels;
    const uint32_t want = (ntasks + WB_THREADS / 32u - 1u) / (WB_THREADS / 32u);
    const uint32_t cap = (phase == 1 ? res_w1 : res_w2) * (uint32_t)(sm_count > 0 ? sm_count : 1);
    const uint32_t grid = want < cap ? want : cap;
    const uint32_t queue = wq_fits(ntasks, grid) ? 1u : 0u;
    cudaError_t e = phase == 1 ? launch_dependent(forest_warp1_kernel, grid, WB_THREADS, 0, stream, a, ntasks, queue)
                               : launch_dependent(forest_warp2_kernel, grid, WB_THREADS, 0, stream, a, ntasks, queue);
    if (e != cudaSuccess) return e;
    forest_steps_from(a.D, a.D - levels, a.N, phase, steps);
  } else {
    forest_steps(a.D, a.N, phase, steps);
  }
  for (const ForestStep& st : steps) {
    cudaError_t e;
    if (st.kind == 0) {
      uint32_t grid = st.ctas;
      const uint32_t cap = (phase == 1 ? res_first : res_fast) * (uint32_t)(sm_count > 0 ? sm_count : 0);
      if (B2D_FOREST_PERSIST && cap && grid > cap) grid = cap;
      e = phase == 1 ? launch_dependent(forest_first_kernel, grid, FAST_THREADS, 0, stream, a, st.p0, st.ctas)
                     : launch_dependent(forest_fast_kernel<2>, grid, FAST_THREADS, 0, stream, a, st.p0, st.ctas);
    } else {
      e = phase == 1 ? launch_dependent(forest_band_kernel<1>, st.ctas, FOREST_THREADS, 0, stream, a, st.p0, st.p1)
                     : launch_dependent(forest_band_kernel<2>, st.ctas, FOREST_THREADS, 0, stream, a, st.p0, st.p1);
    }
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

int forest_launch_count(uint32_t n, uint32_t D, int phase, int warp_mask) {
  std::vector<ForestStep> steps;
  if (warp_bands(n, D, phase, warp_mask)) {
    forest_steps_from(D, D - (phase == 1 ? WB1_LEVELS : WB2_LEVELS), 2, phase, steps);
    return 1 + (int)steps.size();
  }
  forest_steps(D, D == 0 ? 1 : 2, phase, steps);
  return (int)steps.size();
}

cudaError_t launch_forest_seg(const ForestSeg& s, int phase, int kind, uint32_t ctas, cudaStream_t stream) {
  if (ctas == 0) return cudaSuccess;
  if (kind == 2) {
    if (phase == 1) forest_warp1_seg<<<ctas, WB_THREADS, 0, stream>>>(s);
    else forest_warp2_seg<<<ctas, WB_THREADS, 0, stream>>>(s);
  } else if (kind == 0) {
    if (phase == 1) forest_first_seg<<<ctas, FAST_THREADS, 0, stream>>>(s);
    else forest_fast_seg<2><<<ctas, FAST_THREADS, 0, stream>>>(s);
  } else {
    if (phase == 1) forest_band_seg<1><<<ctas, FOREST_THREADS, 0, stream>>>(s);
    else forest_band_seg<2><<<ctas, FOREST_THREADS, 0, stream>>>(s);
  }
  return cudaGetLastError();
}

__device__ __forceinline__ void zero_exists_kernel_body(int* flag, const RoundState* rs) {
  if (!rs->baseline) return;   // only the baseline tests the stale zero digest
  Digest z;
  z.w[0] = z.w[1] = z.w[2] = z.w[3] = 0u;
  const MapView m = rs->map;
  *flag = map_find(m, z) <= m.cap ? 1 : 0;
}
__global__ void zero_exists_kernel(int* flag, const RoundState* rs) {
  griddep_enter();
  zero_exists_kernel_body(flag, rs);
}

__global__ void zero_exists_seg(const ForestArgs* args, uint32_t n) {
  const uint32_t h = blockIdx.x * blockDim.x + threadIdx.x;
  if (h < n) zero_exists_kernel_body(const_cast<int*>(args[h].zero_exists), args[h].rs);   // the flag this step sets
}

cudaError_t launch_zero_exists_seg(const ForestArgs* args, uint32_t n, cudaStream_t stream) {
  zero_exists_seg<<<(n + 127) / 128, 128, 0, stream>>>(args, n);
  return cudaGetLastError();
}

cudaError_t launch_zero_exists(int* flag, const RoundState* rs, cudaStream_t stream) {
  return launch_dependent(zero_exists_kernel, 1, 1, 0, stream, flag, rs);
}

// List approach (src/list_approach.cpp:41-71): a changed chunk whose digest was new is a first
// occurrence, one whose digest existed is a shifted duplicate.  The leaf stage labelled every
// changed chunk of a digest shared within this checkpoint a first occurrence and flagged it;
// in the reference's sequential order the lowest chunk index inserts first, which is the map
// entry's owner after the leaf stage's minimum, so the others become shifted duplicates.  The
// region flags for the diff are set per chunk (its leaf), and the duplicate flags are cleared.
__global__ void list_label_kernel(ForestArgs a0) {
  griddep_enter();
  const ForestArgs a = with_round(a0);
  for (uint64_t c = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; c < a.n; c += (uint64_t)gridDim.x * blockDim.x) {
    uint8_t lab = a.leaflab[c];
    const uint32_t leaf = a.n - 1u + (uint32_t)c;
    if (a.dupflag[c]) {
      a.dupflag[c] = 0;
      if (lab == FIRST_OCUR) {
        const uint64_t slot = map_find(a.map, a.tree[leaf]);
        if (slot <= a.map.cap) {
          if (map_tree(a.map, slot) == a.cur && map_node(a.map, slot) != leaf) {
            lab = SHIFT_DUPL;
            a.leaflab[c] = lab;
          }
        } else {
          set_error(a.st, DERR_INTERNAL, 11);
        }
      }
    }
    if (lab == FIRST_OCUR) push_set(a.push, leaf, PUSH_FIRST);
    else if (lab == SHIFT_DUPL) push_set(a.push, leaf, PUSH_SHIFT);
  }
}

cudaError_t launch_list_label(const ForestArgs& a, int sm_count, cudaStream_t stream) {
  const uint64_t want = ((uint64_t)a.n + 255u) / 256u;
  const uint64_t cap = (uint64_t)sm_count * 8u;
  const uint32_t grid = (uint32_t)(want < cap ? (want ? want : 1) : cap);
  return launch_dependent(list_label_kernel, grid, 256, 0, stream, a);
}



}  // namespace b2d

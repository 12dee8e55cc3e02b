// Leaf stage: hash every chunk, label it FIXED / FIRST / SHIFT against the prior checkpoint,
// record first occurrences in the digest map.
//
// Restates the reference's "Leaves" kernels (src/tree_approach.cpp:54-94 baseline,
// :305-351 incremental).  Two implementations share the per-leaf decision (leaf_finish):
//   * leaf_tma_kernel: persistent, warp-specialised.  One producer warp streams the buffer
//     into shared memory with TMA tensor copies (cp.async.bulk.tensor, 128/64/32-byte
//     swizzle so each lane's chunk row is read without bank conflicts) through an mbarrier
//     ring; eight consumer warps hash one chunk per lane.  Used when the chunk size is a
//     multiple of 16 bytes (MD5: 64) and the buffer is 16-byte aligned.
//   * leaf_generic_kernel: one thread per chunk with byte-granular loads, for any chunk
//     size or alignment, and for the short last chunk.
#include <cuda.h>
#include "dedup_kernels.cuh"
#include "hash.cuh"
#include "map.cuh"

namespace b2d {

// Several leaves of this checkpoint with one new digest: the lowest index owns it ("Choose
// first occurrences", :100-114 / :353-369).  Every atomicMin that finds a value already in the
// slot flags both its own leaf and the value it saw, so after the launch every leaf that
// shares a new digest is flagged; only flagged leaves need the owner lookup in the forest.
__device__ __forceinline__ void flag_shared(const LeafArgs& a, uint32_t chunk, unsigned long long prev) {
  if (prev != ~0ull) {
    a.dupflag[chunk] = 1;
    const uint32_t other = (uint32_t)prev - (a.n - 1u);
    if (other < a.n) a.dupflag[other] = 1;
  }
}

// Per-leaf decision, same order of tests as the reference:
//  baseline:    insert, then compare with the (fresh, all-zero) tree entry
//  incremental: compare with the prior digest first; FIXED leaves skip the insert because
//               their digest is already present from the checkpoint that stored it.
__device__ __forceinline__ void leaf_finish(const LeafArgs& a, uint32_t chunk, const Digest& d, const Digest& old) {
  const uint32_t leaf = a.n - 1u + chunk;
  uint8_t label = DONE;
  const bool fixed = a.baseline ? digest_zero(d) : digest_eq(d, old);
  if (a.baseline || !fixed) {
    const MapRef r = map_insert(a.map, d, (unsigned long long)leaf, a.cur, a.st);
    unsigned long long prev = ~0ull;
    if (r.inserted) {
      label = FIRST_OCUR;
      prev = r.prev;
    } else if (r.found) {
      label = map_merge_current(a.map, r.slot, leaf, a.cur, &prev) ? FIRST_OCUR : SHIFT_DUPL;
    }
    if (label == FIRST_OCUR && !fixed) flag_shared(a, chunk, prev);
    if (r.found) a.tree[leaf] = d;
  }
  if (fixed) {
    label = FIXED_DUPL;
    if (a.baseline) a.tree[leaf] = d;
  }
  a.leaflab[chunk] = label;
}

// Map insert of a lane's changed chunk spread over the lane's next tiles (B2D_LEAF_PIPE 1): the
// read of the digest's home slot is issued once the chunk is hashed and examined after the next
// tile is hashed (a claim, if the slot is empty, then costs an atomic round trip on a line already
// in L2); the owner update's old value, which only the shared-digest flags need, is examined one
// tile later still.  Inserting where the chunk is hashed, a lane with many changed chunks (30 % on
// the MD5 series, 10 % on the batched workload) waited a DRAM read and two atomic round trips per
// changed chunk with its hashing stopped.  (Issuing the claim itself ahead, as a CAS whose old
// value tells an empty slot, this key and another apart, was much slower: the MD5 series' moved
// zero pages all share one digest, and their claims serialise on its slot, where reads do not.)
// Labels, digests, map contents and flags are those of leaf_finish: the map merges values by
// atomicMin and tells a checkpoint's own entries from older ones by their checkpoint field,
// whatever the order of the inserts.
#ifndef B2D_LEAF_PIPE
#define B2D_LEAF_PIPE 1
#endif
struct LeafPipe {
  bool c_on, c_fixed, m_on;   // an insert in flight (and its FIXED test); an owner update in flight
  uint32_t c_chunk, m_chunk;
  Digest c_d;
  uint64_t c_home;
  unsigned long long c_lo, c_hi;   // the home slot's key as read
  unsigned long long m_prev;
};
__device__ __forceinline__ void pipe_init(LeafPipe& p) { p.c_on = p.c_fixed = p.m_on = false; }
// the owner update issued a tile ago: flag shared digests
__device__ __forceinline__ void pipe_flags(const LeafArgs& a, LeafPipe& p) {
  if (p.m_on) flag_shared(a, p.m_chunk, p.m_prev);
  p.m_on = false;
}
// the insert whose home slot was read a tile ago: claim, label, tree digest, owner update
__device__ __forceinline__ void pipe_claim(const LeafArgs& a, LeafPipe& p) {
  if (!p.c_on) return;
  p.c_on = false;
  const uint32_t chunk = p.c_chunk, leaf = a.n - 1u + chunk;
  const unsigned long long val = map_pack((unsigned long long)leaf, a.cur);
  const Key128 k = digest_key(p.c_d);
  MapRef r{p.c_home, true, false, ~0ull};
  bool next = false;   // the home slot holds another key: probe on
  if (p.c_lo != k.lo || p.c_hi != k.hi) {
    if (p.c_lo == MAP_EMPTY || p.c_hi == MAP_EMPTY) {   // empty or being claimed: resolved by the CAS
      const Key128 old = atomicCAS(map_key(a.map, p.c_home), Key128{MAP_EMPTY, MAP_EMPTY}, k);
      if (old.lo == MAP_EMPTY && old.hi == MAP_EMPTY) r.inserted = true;
      else next = old.lo != k.lo || old.hi != k.hi;
    } else {
      next = true;
    }
  }
  if (next) r = map_probe_from(a.map, k, val, map_next(p.c_home, a.map.cap), 1, a.st);
  uint8_t label = DONE;
  if (r.inserted && !next) {   // claimed the home slot: the owner update's old value is read later
    p.m_prev = atomicMin(map_val(a.map, p.c_home), val);
    count_insert(a.map.size);
    label = FIRST_OCUR;
    p.m_on = !p.c_fixed;
    p.m_chunk = chunk;
  } else {
    unsigned long long prev = ~0ull;
    if (r.inserted) {
      label = FIRST_OCUR;
      prev = r.prev;
    } else if (r.found) {
      label = map_merge_current(a.map, r.slot, leaf, a.cur, &prev) ? FIRST_OCUR : SHIFT_DUPL;
    }
    if (label == FIRST_OCUR && !p.c_fixed) flag_shared(a, chunk, prev);
  }
  if (r.found || p.c_fixed) a.tree[leaf] = p.c_d;   // the baseline keeps a FIXED (zero) digest too
  a.leaflab[chunk] = p.c_fixed ? FIXED_DUPL : label;
}
// a hashed chunk: FIXED at once, else the read of its home slot is issued (keys with an all-ones
// half, which a read cannot tell from a slot being claimed, take leaf_finish)
__device__ __forceinline__ void pipe_issue(const LeafArgs& a, LeafPipe& p, uint32_t chunk, const Digest& d,
                                           const Digest& old) {
  const bool fixed = a.baseline ? digest_zero(d) : digest_eq(d, old);
  if (fixed && !a.baseline) {
    a.leaflab[chunk] = FIXED_DUPL;
    return;
  }
  const Key128 k = digest_key(d);
  if (k.lo == MAP_EMPTY || k.hi == MAP_EMPTY) {
    leaf_finish(a, chunk, d, old);
    return;
  }
  p.c_on = true;
  p.c_fixed = fixed;
  p.c_chunk = chunk;
  p.c_d = d;
  p.c_home = map_home(k, a.map.cap);
  const Key128* slot = map_key(a.map, p.c_home);
  p.c_lo = *reinterpret_cast<const volatile unsigned long long*>(&slot->lo);
  p.c_hi = *reinterpret_cast<const volatile unsigned long long*>(&slot->hi);
}
__device__ __forceinline__ void pipe_drain(const LeafArgs& a, LeafPipe& p) {
  pipe_flags(a, p);
  pipe_claim(a, p);
  pipe_flags(a, p);
}

// prior digest of a leaf (the incremental FIXED test); the baseline compares against zero
__device__ __forceinline__ Digest prior_digest(const LeafArgs& a, uint64_t chunk) {
  Digest z;
  z.w[0] = z.w[1] = z.w[2] = z.w[3] = 0u;
  return a.baseline ? z : a.tree[a.n - 1u + chunk];
}

__global__ void leaf_generic_kernel(LeafArgs a0, uint32_t c_begin, uint32_t c_end) {
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
  const LeafArgs a = with_round(a0);
  for (uint64_t c = (uint64_t)c_begin + blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; c < c_end;
       c += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t off = c * a.cs;
    const uint64_t nb = (c == a.n - 1u) ? a.len - off : a.cs;
    const Digest old = prior_digest(a, c);
    const Digest d = hash_bytes(a.kind, a.data + off, nb);
    leaf_finish(a, (uint32_t)c, d, old);
  }
}

// ------------------------------------------------------------------ PTX helpers (sm_90+)
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ bool mbar_test_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
constexpr uint32_t MBAR_WAIT_POLLS = 1u << 24;
// Bounded wait: gives up after MBAR_WAIT_POLLS polls (each try_wait may suspend for a while in
// hardware), or early once another warp of the CTA has given up, records the timeout and
// returns false.  Never spins forever.  `test_polls` != 0 replaces the bound by that many
// non-blocking polls (a test of this give-up path: the first stage has not landed that soon).
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity, DevStatus* st,
                                                  volatile int* abort_flag, uint32_t test_polls = 0) {
  if (test_polls) {
    for (uint32_t i = 0; i < test_polls; i++)
      if (mbar_test_wait(bar, parity)) return true;
  } else {
    for (uint32_t i = 0; i < MBAR_WAIT_POLLS; i++) {
      if (mbar_try_wait(bar, parity)) return true;
      if ((i & 1023u) == 1023u && *abort_flag) return false;
    }
  }
  set_error(st, DERR_WAIT_TIMEOUT, 1);
  *abort_flag = 1;
  return false;
}
// A consumer warp's wait for a staged tile: every lane polls, and the warp goes on together if
// any lane saw the phase complete (completion is monotonic: the phase cannot move on before
// this warp releases the stage), so no lane leaves while the others reach a __syncwarp.
__device__ __forceinline__ bool warp_wait_full(uint64_t* bar, uint32_t parity, DevStatus* st,
                                               volatile int* abort_flag, uint32_t test_polls) {
  const bool ok = mbar_wait_bounded(bar, parity, st, abort_flag, test_polls);
  return __any_sync(0xffffffffu, ok);
}
// Wait for a copy this CTA issued, before the CTA may exit: copies in flight write into its
// shared memory.  Unlike mbar_wait_bounded it does not give up because another warp did (that
// is when it runs), only after the full bound, which a copy from valid memory never reaches.
__device__ __forceinline__ void mbar_wait_drain(uint64_t* bar, uint32_t parity, DevStatus* st) {
  for (uint32_t i = 0; i < MBAR_WAIT_POLLS; i++)
    if (mbar_try_wait(bar, parity)) return;
  set_error(st, DERR_WAIT_TIMEOUT, 2);
}
// a tensor map read from global memory (written there by a copy before this launch)
__device__ __forceinline__ void tensormap_acquire(const CUtensorMap* map) {
  asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"(reinterpret_cast<uint64_t>(map))
               : "memory");
}

__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, uint64_t* bar, int c0, int c1,
                                            int c2) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5}], "
      "[%2];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(bar)), "r"(c0), "r"(c1), "r"(c2)
      : "memory");
}

// physical shared-memory offset of logical byte offset `o` under the tensor map's swizzle
template <int U>
__device__ __forceinline__ uint32_t swz(uint32_t o) {
  if constexpr (U == 128) return o ^ (((o >> 7) & 7u) << 4);
  else if constexpr (U == 64) return o ^ (((o >> 7) & 3u) << 4);
  else if constexpr (U == 32) return o ^ (((o >> 7) & 1u) << 4);
  else return o;
}

// MD5 data blocks with part of each step on the multiply-add pipe (md5_compress_t); 0: all of
// it on the integer ALU
#ifndef B2D_MD5_SPLIT
#define B2D_MD5_SPLIT 1
#endif

// fold the U-byte segment of row `row` of a staged tile into a lane's running digest state
template <int U, int KIND>
__device__ __forceinline__ void hash_segment(const uint8_t* stage, uint32_t row, Murmur3& mm, uint32_t md[4],
                                             uint32_t one) {
  const uint32_t base = row * U;
  if constexpr (KIND == HASH_MD5) {
#pragma unroll
    for (uint32_t blk = 0; blk < U / 64u; blk++) {
      uint32_t m[16];
#pragma unroll
      for (uint32_t j = 0; j < 4; j++) {
        const uint4 v = *reinterpret_cast<const uint4*>(stage + swz<U>(base + blk * 64u + 16u * j));
        m[4 * j + 0] = v.x; m[4 * j + 1] = v.y; m[4 * j + 2] = v.z; m[4 * j + 3] = v.w;
      }
      md5_compress_t<B2D_MD5_SPLIT>(md, m, one);
    }
  } else {
#pragma unroll
    for (uint32_t j = 0; j < U / 16u; j++) {
      const uint4 v = *reinterpret_cast<const uint4*>(stage + swz<U>(base + 16u * j));
      mm.block_words(v.x, v.y, v.z, v.w);
    }
  }
}
template <int KIND>
__device__ __forceinline__ Digest finish_segments(Murmur3& mm, uint32_t md[4], uint32_t cs) {
  if constexpr (KIND == HASH_MD5) {
    md5_pad_block64(md, cs);
    return md5_digest(md);
  } else {
    return mm.finish(cs);
  }
}

// Tile = R = 32 * TMA_CONSUMER_WARPS chunks; stage = one U-byte segment of each chunk of a
// tile (R x U bytes); a chunk of cs bytes takes S = cs / U stages.
template <int U, int KIND>
__global__ void __launch_bounds__((TMA_CONSUMER_WARPS + 1) * 32)
    leaf_tma_kernel(const __grid_constant__ CUtensorMap tmap, LeafArgs a0, uint32_t nfull, uint32_t S,
                    uint32_t stages) {
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
  const LeafArgs a = with_round(a0);
  constexpr uint32_t R = 32u * TMA_CONSUMER_WARPS;
  constexpr uint32_t STAGE_BYTES = R * U;
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023u) & ~uintptr_t(1023));
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + (size_t)stages * STAGE_BYTES);
  uint64_t* empty = full + stages;
  __shared__ int abort_flag;

  const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
  if (threadIdx.x == 0) {
    abort_flag = 0;
    for (uint32_t s = 0; s < stages; s++) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], TMA_CONSUMER_WARPS);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();

  const uint32_t ntiles = (nfull + R - 1) / R;
  if (warp == TMA_CONSUMER_WARPS) {
    // ---------------- producer warp: one elected lane issues the TMA copies
    if (lane == 0) {
      asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&tmap)) : "memory");
      uint32_t k = 0;
      bool ok = true;
      for (uint32_t t = blockIdx.x; t < ntiles && ok; t += gridDim.x) {
        for (uint32_t g = 0; g < S; g++, k++) {
          const uint32_t s = k % stages, ph = (k / stages) & 1u;
          if (k >= stages && !mbar_wait_bounded(&empty[s], ph ^ 1u, a.st, &abort_flag, a.wait_polls)) {
            ok = false;
            break;
          }
          mbar_arrive_expect_tx(&full[s], STAGE_BYTES);
          tma_load_3d(smem + (size_t)s * STAGE_BYTES, &tmap, &full[s], 0, (int)g, (int)(t * R));
        }
      }
      // wait for this CTA's copies still in flight before the CTA may exit
      const uint32_t issued = k;
      const uint32_t first = issued > stages ? issued - stages : 0;
      for (uint32_t q = first; q < issued; q++) mbar_wait_drain(&full[q % stages], (q / stages) & 1u, a.st);
      // the short last chunk (len not a multiple of cs) is hashed here with byte loads
      if (ok && blockIdx.x == 0 && nfull < a.n) {
        for (uint64_t c = nfull; c < a.n; c++) {
          const uint64_t off = c * a.cs;
          const uint64_t nb = (c == a.n - 1u) ? a.len - off : a.cs;
          leaf_finish(a, (uint32_t)c, hash_bytes(a.kind, a.data + off, nb), prior_digest(a, c));
        }
      }
    }
    return;
  }

  // ---------------- consumer warps: lane = chunk row of the tile
  // MD5's hashing of a tile is long enough to hide an insert; Murmur3's is not, and its registers
  // are better spent on the loads in flight
  constexpr bool PIPE = B2D_LEAF_PIPE && KIND == HASH_MD5;
  LeafPipe pipe;
  pipe_init(pipe);
  uint32_t k = 0;
  const uint32_t row = warp * 32u + lane;
  for (uint32_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const uint32_t chunk = t * R + row;
    const bool valid = chunk < nfull;
    // issue the prior-digest load now so its latency hides behind the hashing
    Digest old;
    old.w[0] = old.w[1] = old.w[2] = old.w[3] = 0u;
    if (valid) old = prior_digest(a, chunk);
    Murmur3 mm;
    mm.init();
    uint32_t md[4];
    md5_init(md);
    for (uint32_t g = 0; g < S; g++, k++) {
      const uint32_t s = k % stages, ph = (k / stages) & 1u;
      if (!warp_wait_full(&full[s], ph, a.st, &abort_flag, a.wait_polls)) return;
      const uint8_t* stage = smem + (size_t)s * STAGE_BYTES;
      if (valid) hash_segment<U, KIND>(stage, row, mm, md, a.one);
      __syncwarp();
      if (lane == 0) mbar_arrive(&empty[s]);
    }
    if (PIPE) {
      pipe_flags(a, pipe);
      pipe_claim(a, pipe);
      if (valid) pipe_issue(a, pipe, chunk, finish_segments<KIND>(mm, md, a.cs), old);
    } else if (valid) {
      leaf_finish(a, chunk, finish_segments<KIND>(mm, md, a.cs), old);
    }
  }
  if (PIPE) pipe_drain(a, pipe);
}

// Batched form: one persistent launch hashes the chunks of many buffers.  The producer lane
// pulls work from a global queue of (buffer, tile) items -- `tiles_per_pop` tiles at a time --
// and passes each stage's owner to the consumers through shared memory next to the ring; a
// sentinel stage ends the consumers.  Every buffer has its own tensor map, state and round.
template <int U, int KIND>
__global__ void __launch_bounds__((TMA_CONSUMER_WARPS + 1) * 32)
    leaf_tma_batch_kernel(const BatchLeafItem* items, uint32_t nitems, uint32_t total_tiles, uint32_t tiles_per_pop,
                          unsigned int* queue, uint32_t stages, DevStatus* st) {
  constexpr uint32_t R = 32u * TMA_CONSUMER_WARPS;
  constexpr uint32_t STAGE_BYTES = R * U;
  constexpr uint32_t NO_ITEM = 0xffffffffu;
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023u) & ~uintptr_t(1023));
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + (size_t)stages * STAGE_BYTES);
  uint64_t* empty = full + stages;
  __shared__ uint32_t tbeg[BATCH_MAX_ITEMS + 1];
  __shared__ uint32_t slot_item[16], slot_tile[16], slot_seg[16];
  __shared__ int abort_flag;
  const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
  for (uint32_t i = threadIdx.x; i < nitems; i += blockDim.x) tbeg[i] = items[i].tile_begin;
  if (threadIdx.x == 0) {
    tbeg[nitems] = total_tiles;
    abort_flag = 0;
    for (uint32_t s = 0; s < stages; s++) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], TMA_CONSUMER_WARPS);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();

  if (warp == TMA_CONSUMER_WARPS) {
    if (lane == 0) {
      uint32_t k = 0, last = NO_ITEM;
      bool ok = true;
      while (ok) {
        const uint32_t base = atomicAdd(queue, tiles_per_pop);
        if (base >= total_tiles) break;
        const uint32_t stop = base + tiles_per_pop < total_tiles ? base + tiles_per_pop : total_tiles;
        for (uint32_t tg = base; tg < stop && ok; tg++) {
          uint32_t lo = 0, hi = nitems;   // item with tbeg[i] <= tg < tbeg[i+1]
          while (hi - lo > 1) {
            const uint32_t mid = (lo + hi) >> 1;
            if (tbeg[mid] <= tg) lo = mid; else hi = mid;
          }
          const uint32_t tile = tg - tbeg[lo];
          const uint32_t S = items[lo].S;
          if (lo != last) {
            tensormap_acquire(&items[lo].map);
            last = lo;
          }
          for (uint32_t g = 0; g < S; g++, k++) {
            const uint32_t s = k % stages, ph = (k / stages) & 1u;
            if (k >= stages && !mbar_wait_bounded(&empty[s], ph ^ 1u, st, &abort_flag)) { ok = false; break; }
            slot_item[s] = lo;
            slot_tile[s] = tile;
            slot_seg[s] = g;
            mbar_arrive_expect_tx(&full[s], STAGE_BYTES);
            tma_load_3d(smem + (size_t)s * STAGE_BYTES, &items[lo].map, &full[s], 0, (int)g, (int)(tile * R));
          }
        }
      }
      const uint32_t issued = k;
      // wait for this CTA's copies still in flight (before the sentinel reuses a stage's barrier)
      const uint32_t first = issued > stages ? issued - stages : 0;
      for (uint32_t q = first; q < issued; q++) mbar_wait_drain(&full[q % stages], (q / stages) & 1u, st);
      if (ok) {   // sentinel: a stage with no data whose owner says "done"
        const uint32_t s = k % stages, ph = (k / stages) & 1u;
        if (k < stages || mbar_wait_bounded(&empty[s], ph ^ 1u, st, &abort_flag)) {
          slot_item[s] = NO_ITEM;
          mbar_arrive(&full[s]);
        }
      }
      // short last chunks (len not a multiple of cs), one buffer per CTA in turn
      for (uint32_t i = blockIdx.x; i < nitems; i += gridDim.x) {
        const LeafArgs a = with_round(items[i].args);
        for (uint64_t c = items[i].nfull; c < a.n; c++) {
          const uint64_t off = c * a.cs;
          const uint64_t nb = (c == a.n - 1u) ? a.len - off : a.cs;
          leaf_finish(a, (uint32_t)c, hash_bytes(a.kind, a.data + off, nb), prior_digest(a, c));
        }
      }
    }
    return;
  }

  const uint32_t row = warp * 32u + lane;
  const uint32_t one = items[0].args.one;
  Murmur3 mm;
  uint32_t md[4];
  Digest old;
  uint32_t chunk = 0;
  bool valid = false;
  for (uint32_t k = 0;; k++) {
    const uint32_t s = k % stages, ph = (k / stages) & 1u;
    if (!warp_wait_full(&full[s], ph, st, &abort_flag, 0)) return;
    const uint32_t it = slot_item[s];
    if (it == NO_ITEM) break;
    const uint32_t tile = slot_tile[s], g = slot_seg[s];
    const uint32_t S = items[it].S;
    if (g == 0) {   // a new tile: this lane's chunk, its prior digest, fresh digest state
      chunk = tile * R + row;
      valid = chunk < items[it].nfull;
      mm.init();
      md5_init(md);
      old.w[0] = old.w[1] = old.w[2] = old.w[3] = 0u;
      if (valid) old = prior_digest(with_round(items[it].args), chunk);
    }
    if (valid) hash_segment<U, KIND>(smem + (size_t)s * STAGE_BYTES, row, mm, md, one);
    __syncwarp();
    if (lane == 0) mbar_arrive(&empty[s]);
    if (g + 1 == S && valid) {
      const LeafArgs a = with_round(items[it].args);
      leaf_finish(a, chunk, finish_segments<KIND>(mm, md, a.cs), old);
    }
  }
}

// ------------------------------------------------------------------ host side
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static EncodeTiledFn get_encode_fn() {
  static EncodeTiledFn fn = nullptr;
  static bool tried = false;
  if (!tried) {
    tried = true;
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(p);
  }
  return fn;
}

static int choose_unit(uint32_t cs, int kind) {
  if (kind == HASH_MD5) {
    if (cs % 128u == 0) return 128;
    if (cs % 64u == 0) return 64;
    return 0;
  }
  if (cs % 128u == 0) return 128;
  if (cs % 64u == 0) return 64;
  if (cs % 32u == 0) return 32;
  if (cs % 16u == 0) return 16;
  return 0;
}

template <int U, int KIND>
static cudaError_t launch_tma(const CUtensorMap& map, const LeafArgs& a, uint32_t nfull, uint32_t S,
                              int sm_count, const LeafTuning& tune, cudaStream_t stream) {
  constexpr uint32_t R = 32u * TMA_CONSUMER_WARPS;
  constexpr uint32_t STAGE_BYTES = R * U;
  // default: a 64 KB ring per CTA and 3 CTAs per SM (measured best for 128 B chunks: more
  // resident consumer warps beat a deeper ring); Murmur3 on 64-byte segments (52 registers): a
  // 48 KB ring and 4 CTAs per SM (64 B chunks: 1.019 against 1.057 ms per 4 GiB launch)
  const bool four = U == 64 && KIND == HASH_MURMUR3;
  uint32_t stages = tune.stages > 0 ? (uint32_t)tune.stages : (four ? 3u : (64u * 1024u) / STAGE_BYTES);
  if (stages < 2) stages = 2;
  if (stages > 16) stages = 16;
  while (stages > 2 && (size_t)stages * STAGE_BYTES > 200u * 1024u) stages--;
  const size_t smem = (size_t)stages * STAGE_BYTES + 2 * stages * sizeof(uint64_t) + 1024;
  auto kern = leaf_tma_kernel<U, KIND>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  const uint32_t ntiles = (nfull + R - 1) / R;
  uint32_t grid = (uint32_t)sm_count * (uint32_t)(tune.ctas_per_sm > 0 ? tune.ctas_per_sm : (four ? 4 : 3));
  if (grid > ntiles) grid = ntiles;
  if (grid == 0) grid = 1;
  kern<<<grid, (TMA_CONSUMER_WARPS + 1) * 32, smem, stream>>>(map, a, nfull, S, stages);
  return cudaGetLastError();
}

static bool encode_map(const LeafArgs& a, int U, CUtensorMap& map) {
  EncodeTiledFn enc = get_encode_fn();
  if (!enc) return false;
  const uint32_t nfull = (uint32_t)(a.len / a.cs);
  const cuuint64_t S = a.cs / (uint32_t)U;
  cuuint64_t dims[3] = {(cuuint64_t)U, S, (cuuint64_t)nfull};
  cuuint64_t strides[2] = {(cuuint64_t)U, (cuuint64_t)a.cs};
  cuuint32_t box[3] = {(cuuint32_t)U, 1u, 32u * TMA_CONSUMER_WARPS};
  cuuint32_t estr[3] = {1u, 1u, 1u};
  CUtensorMapSwizzle sw = U == 128 ? CU_TENSOR_MAP_SWIZZLE_128B
                        : U == 64  ? CU_TENSOR_MAP_SWIZZLE_64B
                        : U == 32  ? CU_TENSOR_MAP_SWIZZLE_32B
                                   : CU_TENSOR_MAP_SWIZZLE_NONE;
  return enc(&map, CU_TENSOR_MAP_DATA_TYPE_UINT8, 3, const_cast<uint8_t*>(a.data), dims, strides, box, estr,
             CU_TENSOR_MAP_INTERLEAVE_NONE, sw, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

int batch_leaf_item(const LeafArgs& a, BatchLeafItem& item) {
  const uint32_t nfull = (uint32_t)(a.len / a.cs);
  const int U = choose_unit(a.cs, a.kind);
  if (U == 0 || nfull == 0 || (reinterpret_cast<uintptr_t>(a.data) & 15u) != 0) return 0;
  if (!encode_map(a, U, item.map)) return 0;
  item.args = a;
  item.nfull = nfull;
  item.S = a.cs / (uint32_t)U;
  item.ntiles = (nfull + 32u * TMA_CONSUMER_WARPS - 1) / (32u * TMA_CONSUMER_WARPS);
  return U;
}

template <int U, int KIND>
static cudaError_t launch_batch(const BatchLeafItem* d_items, uint32_t nitems, uint32_t total_tiles,
                                unsigned int* queue, DevStatus* st, int sm_count, const LeafTuning& tune,
                                uint32_t tiles_per_pop, cudaStream_t stream) {
  constexpr uint32_t STAGE_BYTES = 32u * TMA_CONSUMER_WARPS * U;
  uint32_t stages = tune.stages > 0 ? (uint32_t)tune.stages : (64u * 1024u) / STAGE_BYTES;
  if (stages < 2) stages = 2;
  if (stages > 16) stages = 16;
  while (stages > 2 && (size_t)stages * STAGE_BYTES > 200u * 1024u) stages--;
  const size_t smem = (size_t)stages * STAGE_BYTES + 2 * stages * sizeof(uint64_t) + 1024;
  auto kern = leaf_tma_batch_kernel<U, KIND>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  uint32_t grid = (uint32_t)sm_count * (uint32_t)(tune.ctas_per_sm > 0 ? tune.ctas_per_sm : 3);
  if (grid == 0) grid = 1;
  kern<<<grid, (TMA_CONSUMER_WARPS + 1) * 32, smem, stream>>>(d_items, nitems, total_tiles,
                                                              tiles_per_pop ? tiles_per_pop : 1u, queue, stages, st);
  return cudaGetLastError();
}

cudaError_t launch_leaves_batch(const BatchLeafItem* d_items, uint32_t nitems, uint32_t total_tiles, int U, int kind,
                                unsigned int* queue, DevStatus* st, int sm_count, const LeafTuning& tune,
                                uint32_t tiles_per_pop, cudaStream_t stream) {
  if (nitems == 0 || nitems > BATCH_MAX_ITEMS) return cudaErrorInvalidValue;
  if (kind == HASH_MD5) {
    if (U == 128) return launch_batch<128, HASH_MD5>(d_items, nitems, total_tiles, queue, st, sm_count, tune, tiles_per_pop, stream);
    if (U == 64) return launch_batch<64, HASH_MD5>(d_items, nitems, total_tiles, queue, st, sm_count, tune, tiles_per_pop, stream);
    return cudaErrorInvalidValue;
  }
  switch (U) {
    case 128: return launch_batch<128, HASH_MURMUR3>(d_items, nitems, total_tiles, queue, st, sm_count, tune, tiles_per_pop, stream);
    case 64: return launch_batch<64, HASH_MURMUR3>(d_items, nitems, total_tiles, queue, st, sm_count, tune, tiles_per_pop, stream);
    case 32: return launch_batch<32, HASH_MURMUR3>(d_items, nitems, total_tiles, queue, st, sm_count, tune, tiles_per_pop, stream);
    case 16: return launch_batch<16, HASH_MURMUR3>(d_items, nitems, total_tiles, queue, st, sm_count, tune, tiles_per_pop, stream);
    default: return cudaErrorInvalidValue;
  }
}

// Returns 1 if the staged TMA path was used, 0 for the generic path, negative on error.
int launch_leaves(const LeafArgs& a, int sm_count, const LeafTuning& tune, cudaStream_t stream) {
  const uint32_t nfull = (uint32_t)(a.len / a.cs);
  int U = choose_unit(a.cs, a.kind);
  // a narrower requested unit (must divide the chunk; MD5 needs whole 64-byte blocks)
  if (U > 0 && tune.unit > 0 && tune.unit < U && a.cs % (uint32_t)tune.unit == 0 &&
      (a.kind != HASH_MD5 || tune.unit >= 64))
    U = tune.unit;
  const bool aligned = (reinterpret_cast<uintptr_t>(a.data) & 15u) == 0;
  CUtensorMap map;
  if (tune.allow_tma && U > 0 && aligned && nfull > 0) {
    const cuuint64_t S = a.cs / (uint32_t)U;
    if (encode_map(a, U, map)) {
      cudaError_t e;
      const uint32_t s32 = (uint32_t)S;
      if (a.kind == HASH_MD5) {
        e = U == 128 ? launch_tma<128, HASH_MD5>(map, a, nfull, s32, sm_count, tune, stream)
                     : launch_tma<64, HASH_MD5>(map, a, nfull, s32, sm_count, tune, stream);
      } else {
        switch (U) {
          case 128: e = launch_tma<128, HASH_MURMUR3>(map, a, nfull, s32, sm_count, tune, stream); break;
          case 64: e = launch_tma<64, HASH_MURMUR3>(map, a, nfull, s32, sm_count, tune, stream); break;
          case 32: e = launch_tma<32, HASH_MURMUR3>(map, a, nfull, s32, sm_count, tune, stream); break;
          default: e = launch_tma<16, HASH_MURMUR3>(map, a, nfull, s32, sm_count, tune, stream); break;
        }
      }
      return e == cudaSuccess ? 1 : -1;
    }
  }
  const uint32_t threads = 256;
  uint64_t blocks = ceil_div_u64(a.n, threads);
  const uint64_t cap = (uint64_t)sm_count * 16u;
  if (blocks > cap) blocks = cap;
  if (blocks == 0) blocks = 1;
  leaf_generic_kernel<<<(uint32_t)blocks, threads, 0, stream>>>(a, 0u, a.n);
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

}  // namespace b2d

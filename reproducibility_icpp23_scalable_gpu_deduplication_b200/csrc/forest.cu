// Merkle forest stages, level-fused.
//
// The reference walks the heap one level per launch, twice (src/tree_approach.cpp:116-224
// baseline, :371-477 incremental): ~2 log2(N) launches.  Here a launch covers a band of up to
// FOREST_BAND_LEVELS levels: each CTA owns the subtree under one node of the band's top
// level, keeps the labels of the level it is working on in shared memory, and climbs the
// band with one __syncthreads per level.  Labels cross band boundaries through `lab` (only
// the band-top nodes are written).  A 2^25-chunk tree needs three bands per stage.
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
#include "dedup_kernels.cuh"
#include "hash.cuh"
#include "map.cuh"

namespace b2d {

constexpr uint32_t FOREST_THREADS = 512;

__device__ __forceinline__ uint8_t push_flag(uint8_t label) {
  return label == SHIFT_DUPL ? PUSH_SHIFT : (label == FIRST_OCUR ? PUSH_FIRST : PUSH_NONE);
}

template <int PHASE>
__device__ __forceinline__ uint8_t forest_node(const ForestArgs& a, uint32_t x, uint8_t ll, uint8_t rl) {
  const uint32_t l = 2u * x + 1u, r = 2u * x + 2u;
  const uint32_t height = a.D - node_level(x);
  if constexpr (PHASE == 1) {
    if (ll == FIRST_OCUR && rl == FIRST_OCUR) {
      const Digest d = hash_pair(a.kind, a.tree[l], a.tree[r]);
      a.tree[x] = d;
      const unsigned long long v = ((unsigned long long)(1u + height) << 32) | x;
      const MapRef ref = map_insert(a.map, d, v, a.cur, a.st);
      if (ref.found && !ref.inserted) map_merge_current(a.map, ref.slot, v, a.cur);
      return FIRST_OCUR;
    }
    return DONE;
  } else {
    uint8_t out = DONE;
    uint8_t pl = PUSH_NONE, pr = PUSH_NONE;
    if (ll != rl) {
      out = DONE;
      pl = push_flag(ll);
      pr = push_flag(rl);
    } else if (ll == FIXED_DUPL) {
      out = FIXED_DUPL;
    } else if (ll == SHIFT_DUPL) {
      bool exists;
      if (a.baseline) {
        exists = *a.zero_exists != 0;
      } else {
        const Digest d = hash_pair(a.kind, a.tree[l], a.tree[r]);
        a.tree[x] = d;
        exists = map_find(a.map, d) <= a.map.cap;
      }
      if (exists) {
        out = SHIFT_DUPL;
      } else {
        out = DONE;
        pl = PUSH_SHIFT;
        pr = PUSH_SHIFT;
      }
    } else if (ll == FIRST_OCUR) {
      out = FIRST_OCUR;
    }
    a.push[l] = pl;
    a.push[r] = pr;
    if (a.baseline) {
      const Digest d = hash_pair(a.kind, a.tree[l], a.tree[r]);
      a.tree[x] = d;
      const unsigned long long v = ((unsigned long long)(64u + height) << 32) | x;
      const MapRef ref = map_insert(a.map, d, v, a.cur, a.st);
      if (ref.found && !ref.inserted) map_merge_current(a.map, ref.slot, v, a.cur);
    }
    return out;
  }
}

// label of a leaf as seen by this phase (phase 1 applies the lowest-index relabel)
template <int PHASE>
__device__ __forceinline__ uint8_t forest_leaf(const ForestArgs& a, uint32_t x) {
  uint8_t lab = a.lab[x];
  if constexpr (PHASE == 1) {
    if (lab == FIRST_OCUR) {
      const uint64_t slot = map_find(a.map, a.tree[x]);
      if (slot <= a.map.cap) {
        if (map_tree(a.map, slot) == a.cur && map_node(a.map, slot) != x) {
          lab = SHIFT_DUPL;
          a.lab[x] = lab;
        }
      } else {
        set_error(a.st, DERR_INTERNAL, 10);
      }
    }
  }
  return lab;
}

// One band: levels [top, bot] (top <= bot <= D).  CTA b owns node (2^top - 1 + b).
template <int PHASE>
__global__ void __launch_bounds__(FOREST_THREADS) forest_band_kernel(ForestArgs a, uint32_t top, uint32_t bot) {
  __shared__ uint8_t buf[2][1u << (FOREST_BAND_LEVELS - 1)];
  const uint32_t H = bot - top;
  const uint64_t root = ((1ull << top) - 1ull) + blockIdx.x;
  uint8_t* below = buf[0];
  uint8_t* here = buf[1];
  for (int k = (int)H; k >= 0; k--) {
    const uint64_t width = 1ull << k;
    const uint64_t base = (root << k) + width - 1ull;
    for (uint64_t i = threadIdx.x; i < width; i += blockDim.x) {
      const uint64_t x = base + i;
      uint8_t lab = DONE;
      if (x < a.N) {
        if (x >= (uint64_t)a.n - 1u) {
          lab = forest_leaf<PHASE>(a, (uint32_t)x);
        } else {
          uint8_t ll, rl;
          if (k == (int)H) {   // children belong to the band below (written to lab)
            ll = a.lab[2u * (uint32_t)x + 1u];
            rl = a.lab[2u * (uint32_t)x + 2u];
          } else {
            ll = below[2 * i];
            rl = below[2 * i + 1];
          }
          lab = forest_node<PHASE>(a, (uint32_t)x, ll, rl);
        }
      }
      if (k > 0) here[i] = lab;
      else if (x < a.N) {
        // band top: hand the label to the next band up; the tree root decides the
        // whole-buffer first-occurrence region (:127-129 / :392-399)
        if (x == 0) {
          if (PHASE == 2) a.push[0] = (a.n >= 2u && lab == FIRST_OCUR) ? PUSH_FIRST : PUSH_NONE;
        } else {
          if (x < (uint64_t)a.n - 1u) a.lab[x] = lab;   // leaves already hold their label
        }
      }
    }
    __syncthreads();
    uint8_t* t = below;
    below = here;
    here = t;
  }
}

cudaError_t launch_forest(const ForestArgs& a, int phase, cudaStream_t stream) {
  if (a.N <= 1) {   // one chunk: no inner nodes; the reference never pushes a region
    if (phase == 2) return cudaMemsetAsync(a.push, 0, 1, stream);
    return cudaSuccess;
  }
  int bot = (int)a.D;
  while (bot >= 0) {
    int top = bot - (int)FOREST_BAND_LEVELS + 1;
    if (top < 0) top = 0;
    const uint32_t ctas = 1u << top;
    if (phase == 1) forest_band_kernel<1><<<ctas, FOREST_THREADS, 0, stream>>>(a, (uint32_t)top, (uint32_t)bot);
    else forest_band_kernel<2><<<ctas, FOREST_THREADS, 0, stream>>>(a, (uint32_t)top, (uint32_t)bot);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    bot = top - 1;
  }
  return cudaSuccess;
}

__global__ void zero_exists_kernel(MapView m, int* flag) {
  Digest z;
  z.w[0] = z.w[1] = z.w[2] = z.w[3] = 0u;
  *flag = map_find(m, z) <= m.cap ? 1 : 0;
}

cudaError_t launch_zero_exists(const MapView& m, int* flag, cudaStream_t stream) {
  zero_exists_kernel<<<1, 1, 0, stream>>>(m, flag);
  return cudaGetLastError();
}

}  // namespace b2d

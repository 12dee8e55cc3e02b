// Shared device definitions for the B200 tree deduplicator.
//
// Layout of the per-instance state in HBM (one deduplicator = one checkpointed buffer):
//   tree   : Digest[N]       implicit heap of N = 2n-1 node digests, leaves at [n-1, 2n-2]
//                            (include/kokkos_merkle_tree.hpp:30-33 of the reference)
//   lab    : uint8_t[N]      per-node labels (leaf labels + band-top labels), rewritten
//                            every checkpoint (include/utils.hpp:51-57 Label values)
//   push   : 2 bits per node region-root flags set by each node's parent: 1 first-occurrence
//                            root, 2 shifted-duplicate root (16 nodes per 32-bit word)
//   map    : cap+1 keys (16 B) then cap+1 values (8 B): open-addressing digest -> NodeID
//            table, 24 B per slot (map.cuh)
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace b2d {

enum Label : uint8_t { FIRST_OCUR = 0, FIXED_DUPL = 1, SHIFT_DUPL = 2, FIRST_DUPL = 3, DONE = 4 };
enum HashKind : int { HASH_MURMUR3 = 0, HASH_MD5 = 1 };
enum PushFlag : uint8_t { PUSH_NONE = 0, PUSH_FIRST = 1, PUSH_SHIFT = 2 };

struct __align__(16) Digest {
  uint32_t w[4];
};

__host__ __device__ __forceinline__ bool digest_eq(const Digest& a, const Digest& b) {
  return a.w[0] == b.w[0] && a.w[1] == b.w[1] && a.w[2] == b.w[2] && a.w[3] == b.w[3];
}
__host__ __device__ __forceinline__ bool digest_zero(const Digest& a) {
  return (a.w[0] | a.w[1] | a.w[2] | a.w[3]) == 0u;
}

// Device-side error word.  Kernels never trap: they record the first error here and skip.
enum DevError : uint32_t {
  DERR_NONE = 0,
  DERR_MAP_FULL = 1,       // probe sequence exhausted the table
  DERR_WAIT_TIMEOUT = 2,   // a bounded barrier wait gave up
  DERR_INTERNAL = 3,       // an invariant of the reference algorithm did not hold
  DERR_RESTART_RANGE = 4,  // a restart copy/index fell outside its buffer (corrupt diff)
};

struct DevStatus {
  uint32_t error;
  uint32_t detail;
};

__device__ __forceinline__ void set_error(DevStatus* st, uint32_t code, uint32_t detail) {
  if (atomicCAS(&st->error, 0u, code) == 0u) st->detail = detail;
}

// -----------------------------------------------------------------------------------------
// Tree index math, restating include/kokkos_merkle_tree.hpp:102-142 of the reference:
// descend from a node's children until the leftmost index leaves the tree, step back one
// level, clamp the right end.  For a power-of-two leaf count this is the node's leaf range;
// for other counts a node whose subtree spans two depths reports only its deepest level,
// and the diff format inherits that (the GPU path reproduces it bit for bit).
// -----------------------------------------------------------------------------------------
__host__ __device__ __forceinline__ void leaf_range(uint32_t node, uint32_t num_nodes,
                                                    uint32_t& lo, uint32_t& hi) {
  uint32_t l = 2u * node + 1u, r = 2u * node + 2u;
  while (l < num_nodes) {
    l = 2u * l + 1u;
    r = 2u * r + 2u;
  }
  l = (l - 1u) / 2u;
  r = (r - 2u) / 2u;
  if (r > num_nodes) r = num_nodes - 1u;
  lo = l;
  hi = r;
}
__host__ __device__ __forceinline__ uint32_t num_leaf_descendents(uint32_t node, uint32_t num_nodes) {
  uint32_t lo, hi;
  leaf_range(node, num_nodes, lo, hi);
  return hi - lo + 1u;
}
__host__ __device__ __forceinline__ uint32_t leftmost_leaf(uint32_t node, uint32_t num_nodes) {
  uint32_t lo, hi;
  leaf_range(node, num_nodes, lo, hi);
  return lo;
}
// level of a heap index: floor(log2(i+1))
__host__ __device__ __forceinline__ uint32_t node_level(uint32_t i) {
#ifdef __CUDA_ARCH__
  return 31u - __clz(i + 1u);
#else
  return 31u - (uint32_t)__builtin_clz(i + 1u);
#endif
}

__host__ __device__ __forceinline__ uint64_t ceil_div_u64(uint64_t a, uint64_t b) { return (a + b - 1) / b; }

}  // namespace b2d

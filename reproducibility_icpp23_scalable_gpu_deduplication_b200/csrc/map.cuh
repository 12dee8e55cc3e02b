// Open-addressing device map: 128-bit chunk/node digest -> NodeID{node, checkpoint}.
//
// Replaces the reference's DigestNodeIDDeviceMap (include/map_helpers.hpp:105-113, a
// Kokkos::UnorderedMap<HashDigest, NodeID>).  Contract kept from the reference tree path:
//   insert(key, value): insert-if-absent; reports inserted vs existing plus the slot;
//   the slot's value stays mutable for the lowest-index update (tree_approach.cpp:85,339).
//
// Table layout (cap + 1 slots in one allocation), one of two, chosen at build time:
//   B2D_MAP_SPLIT 0 (default): a 32-byte slot per entry, the 128-bit key then its u64 value, so
//     an insert's value update lands in the sector its key claim already brought in;
//   B2D_MAP_SPLIT 1: all keys, then all values (24 bytes per slot): a probe reads only keys,
//     eight to a line, but every value update is a second DRAM access (measured slower on the
//     checkpoint path, which inserts or looks up every changed chunk).
// keys: the 128-bit digest, claimed with one 128-bit atomicCAS (EMPTY = all ones).
// values: u64 = priority << 45 | checkpoint << 32 | node.  Every insert of the current
//   checkpoint applies atomicMin to it; within one checkpoint the checkpoint field is the same,
//   so the value left behind is the one the reference's sequential execution order inserts first
//   (leaves by index, then first-occurrence parents by level and index, then the baseline's
//   per-level inserts).  One atomic sets the owner and its checkpoint together.  All ones
//   (checkpoint field MAP_TREE_PENDING) while the inserting thread has claimed the key but not
//   yet merged its value: readers treat that as "this checkpoint".  Checkpoint ids are below
//   MAP_TREE_PENDING.
// The digest equal to the EMPTY pattern is kept in the extra slot `cap`: present once its value
// is no longer all ones.
#pragma once
#include "common.cuh"

#ifndef B2D_MAP_SPLIT
#define B2D_MAP_SPLIT 0
#endif
#ifndef B2D_MAP_CAS_FIRST
#define B2D_MAP_CAS_FIRST 0
#endif

namespace b2d {

struct __align__(16) Key128 {
  unsigned long long lo, hi;
};
constexpr uint64_t MAP_SLOT_BYTES = B2D_MAP_SPLIT ? sizeof(Key128) + sizeof(unsigned long long) : 32;
constexpr uint64_t MAP_STRIDE = B2D_MAP_SPLIT ? 1 : 2;   // Key128 units from one slot's key to the next

constexpr unsigned long long MAP_EMPTY = ~0ull;
constexpr uint32_t MAP_TREE_BITS = 13;
constexpr uint32_t MAP_TREE_PENDING = (1u << MAP_TREE_BITS) - 1u;   // 8191

// (priority << 32 | node) of the inserting order + the checkpoint id -> the stored value
__device__ __forceinline__ unsigned long long map_pack(unsigned long long val, uint32_t cur) {
  return ((val >> 32) << (32 + MAP_TREE_BITS)) | ((unsigned long long)(cur & MAP_TREE_PENDING) << 32) |
         (val & 0xffffffffull);
}
__device__ __forceinline__ uint32_t map_val_tree(unsigned long long v) {
  return (uint32_t)(v >> 32) & MAP_TREE_PENDING;
}

struct MapView {
  Key128* keys;               // the first slot's key (slot i's: map_key)
  unsigned long long* vals;   // the first slot's value (slot i's: map_val)
  uint64_t cap;               // any positive count (homes are mapped onto [0, cap) by a multiply)
  unsigned long long* size;   // device counter of occupied slots
};

// keys and values of a table of `cap` slots (+ the extra slot) at `mem`
__host__ __device__ __forceinline__ MapView map_at(void* mem, uint64_t cap, unsigned long long* size) {
  MapView m;
  m.keys = static_cast<Key128*>(mem);
  m.vals = B2D_MAP_SPLIT ? reinterpret_cast<unsigned long long*>(m.keys + cap + 1)
                         : reinterpret_cast<unsigned long long*>(m.keys) + 2;
  m.cap = cap;
  m.size = size;
  return m;
}
__host__ __device__ __forceinline__ Key128* map_key(const MapView& m, uint64_t i) { return m.keys + i * MAP_STRIDE; }
__host__ __device__ __forceinline__ unsigned long long* map_val(const MapView& m, uint64_t i) {
  return m.vals + (B2D_MAP_SPLIT ? i : 4 * i);
}

struct MapRef {
  uint64_t slot;       // valid when found
  bool found;
  bool inserted;
  unsigned long long prev;   // value before this insert's atomicMin (inserted only)
};

__device__ __forceinline__ Key128 digest_key(const Digest& d) {
  Key128 k;
  k.lo = (unsigned long long)d.w[0] | ((unsigned long long)d.w[1] << 32);
  k.hi = (unsigned long long)d.w[2] | ((unsigned long long)d.w[3] << 32);
  return k;
}
__device__ __forceinline__ bool key_is_empty_pattern(const Key128& k) {
  return k.lo == MAP_EMPTY && k.hi == MAP_EMPTY;
}
__device__ __forceinline__ uint64_t map_home(const Key128& k, uint64_t cap) {
  // digests are uniformly distributed; fold both halves, then scale the 64-bit value onto
  // [0, cap) (high half of the product), which needs no power-of-two capacity
  unsigned long long h = k.lo ^ (k.hi * 0x9E3779B97F4A7C15ull);
  h ^= h >> 31;
  return (uint64_t)__umul64hi(h, (unsigned long long)cap);
}
__device__ __forceinline__ uint64_t map_next(uint64_t i, uint64_t cap) { return i + 1 == cap ? 0 : i + 1; }

// Find without concurrent inserters on the probed path (all lookups in this library happen
// either in a later kernel than the inserts, or for keys whose probe path was complete
// before the launch).  Returns cap+1 when absent.
__device__ __forceinline__ uint64_t map_find(const MapView& m, const Digest& d) {
  const Key128 k = digest_key(d);
  if (key_is_empty_pattern(k)) return *map_val(m, m.cap) != MAP_EMPTY ? m.cap : m.cap + 1;
  uint64_t i = map_home(k, m.cap);
  for (uint64_t probe = 0; probe < m.cap; probe++) {
    const Key128 s = *map_key(m, i);
    if (s.lo == k.lo && s.hi == k.hi) return i;
    if (s.lo == MAP_EMPTY && s.hi == MAP_EMPTY) return m.cap + 1;
    i = map_next(i, m.cap);
  }
  return m.cap + 1;
}

// occupied-slot counter: one atomic per group of lanes that insert together (a single counter
// takes every insert of a launch, so per-lane atomics would serialise on it)
__device__ __forceinline__ void count_insert(unsigned long long* size) {
  const unsigned am = __activemask();
  const unsigned lane = threadIdx.x & 31u;
  if (lane == (unsigned)(__ffs(am) - 1)) atomicAdd(size, (unsigned long long)__popc(am));
}

__device__ __forceinline__ MapRef map_probe_from(const MapView& m, const Key128& k, unsigned long long val,
                                                 uint64_t i, uint64_t probe, DevStatus* st);

// Insert-if-absent of an already packed value (map_pack).  On success the value is merged
// with atomicMin.  On an existing key nothing is written here; the caller decides (through
// map_merge_current) whether the entry belongs to the current checkpoint.
__device__ __forceinline__ MapRef map_insert_key(const MapView& m, const Key128& k, unsigned long long val,
                                                 DevStatus* st) {
  MapRef r{0, false, false, ~0ull};
  if (key_is_empty_pattern(k)) {
    // the extra slot: the first value merged into it inserts the key
    r.prev = atomicMin(map_val(m, m.cap), val);
    r.slot = m.cap;
    r.found = true;
    r.inserted = r.prev == MAP_EMPTY;
    if (r.inserted) atomicAdd(m.size, 1ull);   // one slot, rare: no aggregation needed
    return r;
  }
  // Each probe reads the slot and CASes only when it may be empty; a key with an all-ones half
  // could be confused with a half-written slot: always CAS.  B2D_MAP_CAS_FIRST 1 makes every
  // probe one 128-bit CAS instead (its old value tells empty, this key and another key apart
  // in one round trip): measured slower, the hashing kernel 0.861 against 0.829 ms and the
  // forest 0.238 against 0.210 ms per 4 GiB step, as atomics on slots that hold other keys or
  // this key cost more than the reads they replace.
  return map_probe_from(m, k, val, map_home(k, m.cap), 0, st);
}
__device__ __forceinline__ MapRef map_insert_packed(const MapView& m, const Digest& d, unsigned long long val,
                                                    DevStatus* st) {
  return map_insert_key(m, digest_key(d), val, st);
}

// The probe loop of an insert from slot i, `probe` slots after the key's home (those hold other
// keys).  The key is not the EMPTY pattern.
__device__ __forceinline__ MapRef map_probe_from(const MapView& m, const Key128& k, unsigned long long val,
                                                 uint64_t i, uint64_t probe, DevStatus* st) {
  MapRef r{0, false, false, ~0ull};
  const bool cas_only = B2D_MAP_CAS_FIRST || (k.lo == MAP_EMPTY) || (k.hi == MAP_EMPTY);
  const Key128 empty{MAP_EMPTY, MAP_EMPTY};
  for (; probe < m.cap; probe++) {
    Key128* s = map_key(m, i);
    bool try_cas = true;
    if (!cas_only) {
      const unsigned long long lo = *reinterpret_cast<volatile unsigned long long*>(&s->lo);
      const unsigned long long hi = *reinterpret_cast<volatile unsigned long long*>(&s->hi);
      if (lo == k.lo && hi == k.hi) {
        r.slot = i; r.found = true; r.inserted = false;
        return r;
      }
      // a slot holding a complete other key can be skipped; anything with an all-ones half
      // may be empty or mid-claim and is resolved by the CAS
      try_cas = (lo == MAP_EMPTY) || (hi == MAP_EMPTY);
    }
    if (try_cas) {
      const Key128 old = atomicCAS(s, empty, k);
      if (old.lo == MAP_EMPTY && old.hi == MAP_EMPTY) {
        r.prev = atomicMin(map_val(m, i), val);
        count_insert(m.size);
        r.slot = i; r.found = true; r.inserted = true;
        return r;
      }
      if (old.lo == k.lo && old.hi == k.hi) {
        r.slot = i; r.found = true; r.inserted = false;
        return r;
      }
    }
    i = map_next(i, m.cap);
  }
  set_error(st, DERR_MAP_FULL, 0);
  return r;
}

// Up to G inserts of one thread at once, with the results of G calls of map_insert_packed.  The
// home slots of all keys are read before any is examined and the claims of all empty homes are
// issued before any result is used, so the thread waits for about one DRAM read and one atomic
// round trip for the group instead of one of each per key.  Keys whose home holds another key
// (rare below the load limit) and keys with an all-ones half continue one at a time.
template <int G>
__device__ __forceinline__ void map_insert_group(const MapView& m, const Key128 (&k)[G],
                                                 const unsigned long long (&val)[G], uint32_t cnt, MapRef (&r)[G],
                                                 DevStatus* st) {
  const Key128 empty{MAP_EMPTY, MAP_EMPTY};
  uint64_t home[G];
  unsigned long long lo[G], hi[G];
#pragma unroll
  for (int j = 0; j < G; j++) {
    r[j] = MapRef{0, false, false, ~0ull};
    if ((uint32_t)j < cnt) {
      home[j] = map_home(k[j], m.cap);
      const Key128* s = map_key(m, home[j]);
      lo[j] = *reinterpret_cast<const volatile unsigned long long*>(&s->lo);
      hi[j] = *reinterpret_cast<const volatile unsigned long long*>(&s->hi);
    }
  }
  uint32_t cas = 0, slow = 0, ins = 0;
#pragma unroll
  for (int j = 0; j < G; j++) {
    if ((uint32_t)j >= cnt) continue;
    if (B2D_MAP_CAS_FIRST || k[j].lo == MAP_EMPTY || k[j].hi == MAP_EMPTY) {
      slow |= 1u << j;   // the one-at-a-time path from the home slot
      home[j] = ~0ull;
    } else if (lo[j] == k[j].lo && hi[j] == k[j].hi) {
      r[j].slot = home[j];
      r[j].found = true;
    } else if (lo[j] == MAP_EMPTY || hi[j] == MAP_EMPTY) {
      cas |= 1u << j;
    } else {
      slow |= 1u << j;
    }
  }
  Key128 old[G];
#pragma unroll
  for (int j = 0; j < G; j++)
    if ((cas >> j) & 1u) old[j] = atomicCAS(map_key(m, home[j]), empty, k[j]);
#pragma unroll
  for (int j = 0; j < G; j++) {
    if (!((cas >> j) & 1u)) continue;
    if (old[j].lo == MAP_EMPTY && old[j].hi == MAP_EMPTY) {
      ins |= 1u << j;
      r[j].slot = home[j];
      r[j].found = r[j].inserted = true;
    } else if (old[j].lo == k[j].lo && old[j].hi == k[j].hi) {
      r[j].slot = home[j];
      r[j].found = true;
    } else {
      slow |= 1u << j;
    }
  }
#pragma unroll
  for (int j = 0; j < G; j++)
    if ((ins >> j) & 1u) r[j].prev = atomicMin(map_val(m, home[j]), val[j]);
  if (ins) {
    const unsigned am = __activemask();
    const uint32_t c = __reduce_add_sync(am, (uint32_t)__popc(ins));
    if ((threadIdx.x & 31u) == (unsigned)(__ffs(am) - 1)) atomicAdd(m.size, (unsigned long long)c);
  }
#pragma unroll
  for (int j = 0; j < G; j++)
    if ((slow >> j) & 1u)
      r[j] = home[j] == ~0ull ? map_insert_key(m, k[j], val[j], st)
                              : map_probe_from(m, k[j], val[j], map_next(home[j], m.cap), 1, st);
}

// insert with `val` = priority << 32 | node, stored for checkpoint `cur`
__device__ __forceinline__ MapRef map_insert(const MapView& m, const Digest& d, unsigned long long val,
                                             uint32_t cur, DevStatus* st) {
  return map_insert_packed(m, d, map_pack(val, cur), st);
}

// An existing entry belongs to the current checkpoint when its id is `cur` or still
// pending (claimed by a concurrent inserter of this launch).  In that case the lower
// (priority, node) value wins, matching "first insert in sequential order".  An entry of an
// older checkpoint is never changed by this one, so its id cannot change under the test.
__device__ __forceinline__ bool map_merge_current(const MapView& m, uint64_t slot, unsigned long long val,
                                                  uint32_t cur, unsigned long long* prev = nullptr) {
  unsigned long long* v = map_val(m, slot);
  const uint32_t t = map_val_tree(*reinterpret_cast<volatile unsigned long long*>(v));
  if (t == (cur & MAP_TREE_PENDING) || t == MAP_TREE_PENDING) {
    const unsigned long long p = atomicMin(v, map_pack(val, cur));
    if (prev) *prev = p;
    return true;
  }
  return false;
}

__device__ __forceinline__ uint32_t map_node(const MapView& m, uint64_t slot) {
  return (uint32_t)(*map_val(m, slot) & 0xffffffffull);
}
__device__ __forceinline__ uint32_t map_tree(const MapView& m, uint64_t slot) {
  return map_val_tree(*map_val(m, slot));
}

}  // namespace b2d

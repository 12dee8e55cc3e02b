// Sequential stand-in for Kokkos::UnorderedMap (see Kokkos_Core.hpp in this directory): an exact
// insert-if-absent hash map whose copies share one table, so a map captured by value in a
// dispatched lambda is the same map.  insert never overwrites an existing key's value and never
// fails (the table grows when it passes 3/4 full); value_at returns a mutable reference for
// in-place updates such as atomic_min.  Slot indices stay valid until the next insert that
// grows the table, rehash or clear.
#ifndef B2D_KOKKOS_SHIM_UNORDERED_MAP_HPP
#define B2D_KOKKOS_SHIM_UNORDERED_MAP_HPP

#include <cstring>

#include "Kokkos_Core.hpp"

namespace Kokkos {

// default key hash and equality: the key's bytes
template <class K>
struct pod_hash {
  uint32_t operator()(const K& k) const {
    uint64_t h = 1469598103934665603ull;
    const unsigned char* p = reinterpret_cast<const unsigned char*>(&k);
    for (size_t i = 0; i < sizeof(K); i++) h = (h ^ p[i]) * 1099511628211ull;
    return (uint32_t)(h ^ (h >> 32));
  }
};
template <class K>
struct pod_equal_to {
  bool operator()(const K& a, const K& b) const { return std::memcmp(&a, &b, sizeof(K)) == 0; }
};

class UnorderedMapInsertResult {
 public:
  UnorderedMapInsertResult(bool ok, bool ex, uint32_t i) : ok_(ok), ex_(ex), idx_(i) {}
  bool success() const { return ok_; }
  bool existing() const { return ex_; }
  bool failed() const { return !ok_ && !ex_; }
  uint32_t index() const { return idx_; }

 private:
  bool ok_, ex_;
  uint32_t idx_;
};

template <class K, class V, class Space = DefaultExecutionSpace, class Hasher = pod_hash<K>,
          class Equal = pod_equal_to<K>>
class UnorderedMap {
  struct Table {
    std::vector<K> keys;
    std::vector<V> vals;
    std::vector<uint8_t> used;
    size_t size = 0;
  };

 public:
  static constexpr uint32_t invalid_index = 0xffffffffu;

  explicit UnorderedMap(size_t capacity_hint = 0) : t_(std::make_shared<Table>()) { init(*t_, capacity_hint); }

  UnorderedMapInsertResult insert(const K& k, const V& v = V()) const {
    Table& t = *t_;
    if (4 * (t.size + 1) > 3 * t.keys.size()) grow(2 * t.keys.size());
    size_t s = slot(t, k);
    while (t.used[s]) {
      if (Equal()(t.keys[s], k)) return UnorderedMapInsertResult(false, true, (uint32_t)s);
      s = (s + 1) & (t.keys.size() - 1);
    }
    t.used[s] = 1;
    t.keys[s] = k;
    t.vals[s] = v;
    t.size++;
    return UnorderedMapInsertResult(true, false, (uint32_t)s);
  }
  uint32_t find(const K& k) const {
    const Table& t = *t_;
    size_t s = slot(t, k);
    while (t.used[s]) {
      if (Equal()(t.keys[s], k)) return (uint32_t)s;
      s = (s + 1) & (t.keys.size() - 1);
    }
    return invalid_index;
  }
  bool exists(const K& k) const { return find(k) != invalid_index; }
  bool valid_at(uint32_t i) const { return i < t_->keys.size() && t_->used[i]; }
  K& key_at(uint32_t i) const { return t_->keys[i]; }
  V& value_at(uint32_t i) const { return t_->vals[i]; }
  size_t size() const { return t_->size; }
  size_t capacity() const { return t_->keys.size(); }
  bool rehash(size_t n) const {
    if (n > capacity()) grow(n);
    return true;
  }
  void clear() const {
    std::fill(t_->used.begin(), t_->used.end(), 0);
    t_->size = 0;
  }

 private:
  static size_t pow2_at_least(size_t n) {
    size_t c = 16;
    while (c < n) c <<= 1;
    return c;
  }
  static void init(Table& t, size_t hint) {
    const size_t c = pow2_at_least(hint + hint / 3 + 1);
    t.keys.assign(c, K());
    t.vals.assign(c, V());
    t.used.assign(c, 0);
    t.size = 0;
  }
  static size_t slot(const Table& t, const K& k) {
    uint64_t h = (uint64_t)Hasher()(k) * 0x9E3779B97F4A7C15ull;
    h ^= h >> 29;
    return (size_t)(h & (t.keys.size() - 1));
  }
  void grow(size_t want) const {
    Table old = *t_;
    init(*t_, want);
    for (size_t i = 0; i < old.keys.size(); i++)
      if (old.used[i]) insert(old.keys[i], old.vals[i]);
  }

  std::shared_ptr<Table> t_;

  template <class K2, class V2, class S2, class H2, class E2>
  friend class UnorderedMap;
  template <class K2, class V2, class S1, class H1, class E1, class S2, class H2, class E2>
  friend void deep_copy(UnorderedMap<K2, V2, S1, H1, E1>&, const UnorderedMap<K2, V2, S2, H2, E2>&);
};

// the destination becomes an independent copy of the source's entries
template <class K, class V, class S1, class H1, class E1, class S2, class H2, class E2>
void deep_copy(UnorderedMap<K, V, S1, H1, E1>& dst, const UnorderedMap<K, V, S2, H2, E2>& src) {
  *dst.t_ = *src.t_;
}

}  // namespace Kokkos

#endif  // B2D_KOKKOS_SHIM_UNORDERED_MAP_HPP

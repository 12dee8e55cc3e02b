// Sequential host stand-in for the part of the Kokkos API that the reference's tree and list
// deduplicators use (src/tree_approach.cpp, src/list_approach.cpp and their headers), so that the
// reference's own source compiles unmodified on the CPU as a second oracle.  TEST INFRASTRUCTURE
// ONLY: built into oracle/_ref/ by oracle/Makefile when the reference source tree is present.
//
// Written from the documented semantics of the API, executed the way the reference's sequential
// reading assumes:
//   * every parallel dispatch runs its indices in ascending order on one thread; a team of AUTO
//     size has one member, so team barriers and broadcasts do nothing and a TeamThreadRange is a
//     plain loop; an explicit team size runs its members one after another;
//     a parallel_scan calls its functor once per index with the final flag set;
//   * atomics are plain read-modify-writes;
//   * a View is a reference-counted 1-D array (zero-initialised when allocated with a label),
//     copies share storage, and a host mirror of a view shares its storage, so deep copies
//     between a view and its mirror copy nothing.
#ifndef B2D_KOKKOS_SHIM_CORE_HPP
#define B2D_KOKKOS_SHIM_CORE_HPP

#include <algorithm>
#include <chrono>
#include <cstddef>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <string>
#include <iostream>
#include <limits>
#include <map>
#include <type_traits>
#include <unordered_map>
#include <utility>
#include <vector>

#define KOKKOS_INLINE_FUNCTION inline
#define KOKKOS_FORCEINLINE_FUNCTION inline
#define KOKKOS_FUNCTION
#define KOKKOS_LAMBDA [=]
#define KOKKOS_CLASS_LAMBDA [=, *this]

namespace Kokkos {

inline void initialize(int&, char**) {}
inline void initialize() {}
inline void finalize() {}
inline void fence() {}
inline void fence(const std::string&) {}

namespace Profiling {
inline void pushRegion(const std::string&) {}
inline void popRegion() {}
}  // namespace Profiling

struct HostSpace {};
struct Serial {
  using memory_space = HostSpace;
};
using DefaultExecutionSpace = Serial;
using DefaultHostExecutionSpace = Serial;

enum MemoryTraitsFlags : unsigned { Unmanaged = 1u };
template <unsigned T>
struct MemoryTraits {};

// -------------------------------------------------------------------------------- View
template <class D>
struct ViewShape;
template <class T>
struct ViewShape<T*> {
  using value_type = T;
  static constexpr size_t fixed = 0;
};
template <class T, size_t N>
struct ViewShape<T[N]> {
  using value_type = T;
  static constexpr size_t fixed = N;
};

template <class DataType, class... Props>
class View {
 public:
  using shape = ViewShape<DataType>;
  using value_type = typename shape::value_type;
  using non_const_value_type = typename std::remove_const<value_type>::type;
  using HostMirror = View<DataType, HostSpace>;
  using data_type = DataType;

  View() = default;
  explicit View(const std::string& label, size_t n = shape::fixed) : label_(label) { allocate(n); }
  // a view of memory owned elsewhere (MemoryTraits<Unmanaged>); a template, so a string literal
  // (the label of View<char*>) never binds to it
  template <class Ptr, class = typename std::enable_if<std::is_same<Ptr, value_type*>::value>::type>
  View(Ptr p, size_t n) : ptr_(p), n_(n) {}
  // views of the same data type share storage whatever their other properties
  template <class... P2>
  View(const View<DataType, P2...>& o) : mem_(o.mem_), ptr_(o.ptr_), n_(o.n_), label_(o.label_) {}
  template <class... P2>
  View& operator=(const View<DataType, P2...>& o) {
    mem_ = o.mem_;
    ptr_ = o.ptr_;
    n_ = o.n_;
    label_ = o.label_;
    return *this;
  }

  value_type& operator()(size_t i) const { return ptr_[i]; }
  value_type& operator[](size_t i) const { return ptr_[i]; }
  value_type* data() const { return ptr_; }
  size_t size() const { return n_; }
  size_t span() const { return n_; }
  size_t extent(int) const { return n_; }
  const std::string& label() const { return label_; }
  bool is_allocated() const { return ptr_ != nullptr; }

  void allocate(size_t n) {
    n_ = n;
    mem_ = std::shared_ptr<non_const_value_type>(new non_const_value_type[n ? n : 1](),
                                                 std::default_delete<non_const_value_type[]>());
    ptr_ = mem_.get();
  }

  std::shared_ptr<non_const_value_type> mem_;
  value_type* ptr_ = nullptr;
  size_t n_ = 0;
  std::string label_;
};

template <class D, class... P>
typename View<D, P...>::HostMirror create_mirror_view(const View<D, P...>& v) {
  return typename View<D, P...>::HostMirror(v);
}
template <class Space, class D, class... P>
typename View<D, P...>::HostMirror create_mirror_view(const Space&, const View<D, P...>& v) {
  return typename View<D, P...>::HostMirror(v);
}
template <class D, class... P>
typename View<D, P...>::HostMirror create_mirror(const View<D, P...>& v) {
  return typename View<D, P...>::HostMirror(v.label(), v.size());
}

template <class D1, class... P1, class D2, class... P2>
void deep_copy(const View<D1, P1...>& dst, const View<D2, P2...>& src) {
  if (dst.data() == src.data()) return;
  const size_t n = std::min(dst.size(), src.size());
  for (size_t i = 0; i < n; i++) dst(i) = src(i);
}
template <class S>
struct is_view : std::false_type {};
template <class D, class... P>
struct is_view<View<D, P...>> : std::true_type {};
// every element set to one value
template <class D, class... P, class S, class = typename std::enable_if<!is_view<S>::value>::type>
void deep_copy(const View<D, P...>& dst, const S& value) {
  for (size_t i = 0; i < dst.size(); i++) dst(i) = static_cast<typename View<D, P...>::value_type>(value);
}

// keeps the first min(old, n) elements, zero-fills the rest; a view that already has n elements
// is left as it is (same storage)
template <class D, class... P>
void resize(View<D, P...>& v, size_t n) {
  if (v.is_allocated() && v.size() == n) return;
  View<D, P...> nv(v.label(), n);
  const size_t k = std::min(n, v.size());
  for (size_t i = 0; i < k; i++) nv(i) = v(i);
  v = nv;
}

struct ALL_t {};
constexpr ALL_t ALL = ALL_t();
template <class D, class... P>
View<D, P...> subview(const View<D, P...>& v, ALL_t) {
  return v;
}
template <class D, class... P, class I1, class I2>
View<D, P...> subview(const View<D, P...>& v, const std::pair<I1, I2>& r) {
  View<D, P...> s = v;
  s.ptr_ = v.ptr_ + r.first;
  s.n_ = (size_t)(r.second - r.first);
  return s;
}
template <class T1, class T2>
std::pair<T1, T2> make_pair(T1 a, T2 b) {
  return std::pair<T1, T2>(a, b);
}
template <class T1, class T2>
using pair = std::pair<T1, T2>;

// -------------------------------------------------------------------------------- atomics
template <class T, class V>
T atomic_fetch_add(T* p, V v) {
  const T old = *p;
  *p = static_cast<T>(old + v);
  return old;
}
template <class T, class V>
void atomic_add(T* p, V v) {
  *p = static_cast<T>(*p + v);
}
template <class T, class V>
void atomic_min(T* p, V v) {
  if (static_cast<T>(v) < *p) *p = static_cast<T>(v);
}
template <class T, class V>
T atomic_fetch_min(T* p, V v) {
  const T old = *p;
  if (static_cast<T>(v) < old) *p = static_cast<T>(v);
  return old;
}

// -------------------------------------------------------------------------------- policies
template <class... P>
struct RangePolicy {
  RangePolicy(size_t b, size_t e) : begin(b), end(e) {}
  size_t begin, end;
};

struct AUTO_t {
  constexpr const AUTO_t& operator()() const { return *this; }
};
constexpr AUTO_t AUTO = AUTO_t();

// Team members run one after another, each to the end of the functor: correct for functors whose
// members do not wait for one another (a team of one, or members without barriers, which is how
// the reference uses explicit team sizes).
struct TeamMember {
  size_t league;
  size_t leagues;
  int rank;
  int size;
  size_t league_rank() const { return league; }
  size_t league_size() const { return leagues; }
  int team_rank() const { return rank; }
  int team_size() const { return size; }
  void team_barrier() const {}
  template <class T>
  void team_broadcast(T&, int) const {}
};

template <class... P>
struct TeamPolicy {
  using member_type = TeamMember;
  TeamPolicy(size_t league, AUTO_t) : leagues(league), size(1) {}
  TeamPolicy(size_t league, int team_size) : leagues(league), size(team_size > 0 ? team_size : 1) {}
  size_t leagues;
  int size;
};

// the iterations of a team-level loop that one member runs
struct TeamRange {
  size_t begin, end, first, stride;
};
inline TeamRange TeamThreadRange(const TeamMember& m, size_t n) {
  return TeamRange{0, n, (size_t)m.rank, (size_t)m.size};
}
inline TeamRange TeamThreadRange(const TeamMember& m, size_t b, size_t e) {
  return TeamRange{b, e, (size_t)m.rank, (size_t)m.size};
}

// -------------------------------------------------------------------------------- dispatch
template <class I, class F, class = typename std::enable_if<std::is_integral<I>::value>::type>
void parallel_for(const std::string&, I n, const F& f) {
  for (I i = 0; i < n; i++) f(i);
}
template <class I, class F, class = typename std::enable_if<std::is_integral<I>::value>::type>
void parallel_for(I n, const F& f) {
  for (I i = 0; i < n; i++) f(i);
}
template <class... P, class F>
void parallel_for(const std::string&, const RangePolicy<P...>& r, const F& f) {
  for (size_t i = r.begin; i < r.end; i++) f(i);
}
template <class... P, class F>
void parallel_for(const RangePolicy<P...>& r, const F& f) {
  for (size_t i = r.begin; i < r.end; i++) f(i);
}
template <class... P, class F>
void parallel_for(const std::string&, const TeamPolicy<P...>& t, const F& f) {
  for (size_t l = 0; l < t.leagues; l++)
    for (int j = 0; j < t.size; j++) f(TeamMember{l, t.leagues, j, t.size});
}
template <class... P, class F>
void parallel_for(const TeamPolicy<P...>& t, const F& f) {
  for (size_t l = 0; l < t.leagues; l++)
    for (int j = 0; j < t.size; j++) f(TeamMember{l, t.leagues, j, t.size});
}
template <class F>
void parallel_for(const TeamRange& r, const F& f) {
  for (size_t i = r.begin + r.first; i < r.end; i += r.stride) f(i);
}

// the accumulator type of a scan functor: the type its second parameter refers to
template <class F>
struct ScanArg;
template <class C, class R, class I, class T>
struct ScanArg<R (C::*)(I, T&, bool) const> {
  using type = T;
};
template <class I, class F, class = typename std::enable_if<std::is_integral<I>::value>::type>
void parallel_scan(const std::string&, I n, const F& f) {
  typename ScanArg<decltype(&F::operator())>::type acc = 0;
  for (I i = 0; i < n; i++) f(i, acc, true);
}
template <class... P, class F>
void parallel_scan(const std::string&, const RangePolicy<P...>& r, const F& f) {
  typename ScanArg<decltype(&F::operator())>::type acc = 0;
  for (size_t i = r.begin; i < r.end; i++) f(i, acc, true);
}

// reductions: the functor folds each index into one accumulator, which the reducer starts and
// hands back
template <class T>
struct Max {
  T& result;
  explicit Max(T& r) : result(r) {}
  void init(T& v) const { v = std::numeric_limits<T>::lowest(); }
};
template <class T>
struct Min {
  T& result;
  explicit Min(T& r) : result(r) {}
  void init(T& v) const { v = std::numeric_limits<T>::max(); }
};
template <class T>
struct Sum {
  T& result;
  explicit Sum(T& r) : result(r) {}
  void init(T& v) const { v = T(0); }
};
template <class... P, class F, class R>
void parallel_reduce(const std::string&, const RangePolicy<P...>& r, const F& f, const R& red) {
  typename std::remove_reference<decltype(red.result)>::type acc;
  red.init(acc);
  for (size_t i = r.begin; i < r.end; i++) f(i, acc);
  red.result = acc;
}

// -------------------------------------------------------------------------------- Bitset
template <class Space = DefaultExecutionSpace>
class Bitset {
 public:
  explicit Bitset(size_t n) : bits_(std::make_shared<std::vector<uint8_t>>(n, 0)) {}
  void set(size_t i) const { (*bits_)[i] = 1; }
  void reset(size_t i) const { (*bits_)[i] = 0; }
  void reset() const { std::fill(bits_->begin(), bits_->end(), 0); }
  void clear() const { reset(); }
  bool test(size_t i) const { return (*bits_)[i] != 0; }
  size_t size() const { return bits_->size(); }
  size_t count() const {
    size_t c = 0;
    for (uint8_t b : *bits_) c += b;
    return c;
  }

 private:
  std::shared_ptr<std::vector<uint8_t>> bits_;
};

}  // namespace Kokkos

#endif  // B2D_KOKKOS_SHIM_CORE_HPP

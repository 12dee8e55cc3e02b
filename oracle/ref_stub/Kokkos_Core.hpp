// Minimal stand-in for the Kokkos headers, just enough to compile the reference's
// header-only hash functions (include/kokkos_murmur3.hpp, include/kokkos_md5.hpp) as
// plain host C++ for the golden-vector generator.  No Kokkos functionality is provided.
#pragma once
#include <cstdint>
#include <cstddef>
#include <climits>
#define KOKKOS_INLINE_FUNCTION inline
#define KOKKOS_FORCEINLINE_FUNCTION inline
namespace Kokkos {
struct DefaultExecutionSpace {};
struct DefaultHostExecutionSpace {};
template <class K, class V, class E = DefaultExecutionSpace, class H = void, class Q = void>
class UnorderedMap;
}  // namespace Kokkos

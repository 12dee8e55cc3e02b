// Exposes the reference's own chunk hash functions, compiled unmodified from the
// reference headers, as a C ABI for the golden-vector generator (tests/golden/).
// TEST INFRASTRUCTURE ONLY: built into oracle/_ref/ from the reference tree in place.
#include "kokkos_murmur3.hpp"   // reference include/kokkos_murmur3.hpp
#include "kokkos_md5.hpp"       // reference include/kokkos_md5.hpp

extern "C" void ref_murmur3(const void* data, uint64_t len, uint8_t* out) {
  kokkos_murmur3::hash(data, len, out);
}
extern "C" void ref_md5(const void* data, uint64_t len, uint8_t* out) {
  kokkos_md5::hash(data, len, out);
}

// Kokkos::Bitset lives in Kokkos_Core.hpp of this stand-in (see there); this header exists
// because some reference headers include it by name.
#ifndef B2D_KOKKOS_SHIM_BITSET_HPP
#define B2D_KOKKOS_SHIM_BITSET_HPP
#include "Kokkos_Core.hpp"
#endif

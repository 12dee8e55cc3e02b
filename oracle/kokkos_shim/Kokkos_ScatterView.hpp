// Sequential stand-in for Kokkos::Experimental::ScatterView (see Kokkos_Core.hpp in this
// directory): with one thread there is nothing to duplicate, so access() writes straight into the
// original view and contribute() / reset_except() have nothing left to do.
#ifndef B2D_KOKKOS_SHIM_SCATTER_VIEW_HPP
#define B2D_KOKKOS_SHIM_SCATTER_VIEW_HPP

#include "Kokkos_Core.hpp"

namespace Kokkos {
namespace Experimental {

template <class DataType, class... Props>
class ScatterView {
 public:
  ScatterView() = default;
  template <class... P2>
  explicit ScatterView(const View<DataType, P2...>& v) : v_(v) {}
  View<DataType> access() const { return v_; }
  template <class... P2>
  void reset_except(const View<DataType, P2...>&) const {}
  void reset() const { deep_copy(v_, 0); }

 private:
  View<DataType> v_;
};

template <class DataType, class... P1, class... P2>
void contribute(const View<DataType, P1...>&, const ScatterView<DataType, P2...>&) {}

}  // namespace Experimental
}  // namespace Kokkos

#endif  // B2D_KOKKOS_SHIM_SCATTER_VIEW_HPP

// Sequential stand-in for Kokkos::BinSort with Kokkos::BinOp1D (see Kokkos_Core.hpp in this
// directory): a counting sort of the keys in [begin, end) by bin, keeping equal bins in their
// original order (what one thread filling the bins in index order produces), then sort(v) applies
// that permutation to a view.  BinOp1D(max_bins, min, max) maps a key linearly onto bins
// 0..max_bins; when min == max every key falls in bin 0.
#ifndef B2D_KOKKOS_SHIM_SORT_HPP
#define B2D_KOKKOS_SHIM_SORT_HPP

#include "Kokkos_Core.hpp"

namespace Kokkos {

template <class KeyView>
struct BinOp1D {
  BinOp1D() = default;
  BinOp1D(int max_bins, double min, double max) : bins_(max_bins + 1), min_(min), max_(max) {}
  template <class V>
  int bin(const V& keys, size_t i) const {
    if (max_ == min_) return 0;
    const double x = ((double)keys(i) - min_) * (double)(bins_ - 1) / (max_ - min_);
    int b = (int)x;
    return b < 0 ? 0 : (b >= bins_ ? bins_ - 1 : b);
  }
  int max_bins() const { return bins_; }
  int bins_ = 1;
  double min_ = 0, max_ = 0;
};

template <class KeyView, class BinOp, class Space = DefaultExecutionSpace, class Size = size_t>
class BinSort {
 public:
  BinSort(const KeyView& keys, size_t begin, size_t end, BinOp op, bool /*sort_within_bins*/ = false)
      : keys_(keys), begin_(begin), end_(end), op_(op) {}
  BinSort(const KeyView& keys, BinOp op, bool sort_within_bins = false)
      : BinSort(keys, 0, keys.size(), op, sort_within_bins) {}
  void create_permute_vector() {
    const int nb = op_.max_bins();
    std::vector<size_t> count((size_t)nb + 1, 0);
    for (size_t i = begin_; i < end_; i++) count[(size_t)op_.bin(keys_, i) + 1]++;
    for (int b = 0; b < nb; b++) count[(size_t)b + 1] += count[(size_t)b];
    perm_.assign(end_ - begin_, 0);
    for (size_t i = begin_; i < end_; i++) perm_[count[(size_t)op_.bin(keys_, i)]++] = i;
  }
  template <class V>
  void sort(const V& v) const {
    std::vector<typename std::remove_const<typename V::value_type>::type> tmp(perm_.size());
    for (size_t j = 0; j < perm_.size(); j++) tmp[j] = v(perm_[j]);
    for (size_t j = 0; j < perm_.size(); j++) v(begin_ + j) = tmp[j];
  }

 private:
  KeyView keys_;
  size_t begin_, end_;
  BinOp op_;
  std::vector<size_t> perm_;
};

}  // namespace Kokkos

#endif  // B2D_KOKKOS_SHIM_SORT_HPP

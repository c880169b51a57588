// Stand-in for xtensor's masked view as DP3's AntennaConstraint uses it:
// xt::masked_view(t, mask).fill(v) sets the elements of t where mask is true.
// Only for building DP3's sources outside a DP3 tree.
#ifndef DP3B200_STANDIN_XTENSOR_VIEWS_XMASKED_VIEW_HPP
#define DP3B200_STANDIN_XTENSOR_VIEWS_XMASKED_VIEW_HPP

#include "../containers/xtensor.hpp"

namespace xt {

template <typename T, size_t N, typename M>
class masked_view_t {
 public:
  masked_view_t(xtensor<T, N>& t, const xtensor<M, N>& mask) : t_(t), mask_(mask) {}
  void fill(const T& v) {
    for (size_t i = 0; i != t_.size(); ++i)
      if (mask_.data()[i]) t_.data()[i] = v;
  }

 private:
  xtensor<T, N>& t_;
  xtensor<M, N> mask_;
};

template <typename T, size_t N, typename M>
masked_view_t<T, N, M> masked_view(xtensor<T, N>& t, const xtensor<M, N>& mask) {
  return masked_view_t<T, N, M>(t, mask);
}

}  // namespace xt

#endif

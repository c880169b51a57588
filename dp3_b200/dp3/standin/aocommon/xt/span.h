// Stand-in for aocommon's xt::Span: a non-owning N-dimensional row-major view
// of contiguous memory with xtensor's shape() / operator() interface, as
// DP3's SolutionSpan (ddecal/Solutions.h) uses it. Only for building DP3's
// sources and the SolverBase adapter outside a DP3 tree.
#ifndef DP3B200_STANDIN_AOCOMMON_XT_SPAN_H
#define DP3B200_STANDIN_AOCOMMON_XT_SPAN_H

#include <array>
#include <cassert>
#include <cstddef>

#include <xtensor/containers/xtensor.hpp>

namespace aocommon::xt {

template <typename T, size_t N>
class Span {
 public:
  using value_type = T;
  using shape_type = std::array<size_t, N>;
  Span(T* data, const shape_type& shape) : data_(data), shape_(shape) {}

  const shape_type& shape() const { return shape_; }
  size_t shape(size_t i) const { return shape_[i]; }
  size_t size() const { return ::xt::detail::Product(shape_); }
  size_t dimension() const { return N; }
  T* data() const { return data_; }
  T* begin() const { return data_; }
  T* end() const { return data_ + size(); }

  template <typename... I>
  T& operator()(I... idx) const {
    static_assert(sizeof...(I) == N, "index count must equal the rank");
    const std::array<size_t, N> ix{size_t(idx)...};
    size_t off = 0;
    for (size_t d = 0; d != N; ++d) {
      assert(ix[d] < shape_[d]);
      off = off * shape_[d] + ix[d];
    }
    return data_[off];
  }

 private:
  T* data_;
  shape_type shape_;
};

template <typename T, size_t N>
Span<T, N> CreateSpan(::xt::xtensor<T, N>& t) {
  return Span<T, N>(t.data(), t.shape());
}

template <typename T, size_t N>
Span<T, N> CreateSpan(T* data, const std::array<size_t, N>& shape) {
  return Span<T, N>(data, shape);
}

}  // namespace aocommon::xt

#endif

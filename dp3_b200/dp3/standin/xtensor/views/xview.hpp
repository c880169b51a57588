// Stand-in for xtensor's views as DP3's DDECal sources use them:
// xt::view(e, i, j, xt::all(), ...) (integer indices fix a dimension,
// xt::all() keeps it) and xt::reshape_view(e, {shape...}) over contiguous
// row-major storage. Both are strided references (no copy); they can be read
// element-wise, copied into an xt::xtensor, assigned from one, filled and
// divided element-wise. Only for building DP3's sources outside a DP3 tree.
#ifndef DP3B200_STANDIN_XTENSOR_VIEWS_XVIEW_HPP
#define DP3B200_STANDIN_XTENSOR_VIEWS_XVIEW_HPP

#include <array>
#include <cassert>
#include <cstddef>
#include <type_traits>

#include "../containers/xtensor.hpp"

namespace xt {

struct all_tag {};
inline all_tag all() { return {}; }

template <typename T, size_t M>
class strided_view {
 public:
  using value_type = std::remove_const_t<T>;
  strided_view(T* base, const std::array<size_t, M>& shape,
               const std::array<size_t, M>& strides)
      : base_(base), shape_(shape), strides_(strides) {}

  bool is_xt_view() const { return true; }
  const std::array<size_t, M>& shape() const { return shape_; }
  size_t shape(size_t i) const { return shape_[i]; }
  size_t size() const { return detail::Product(shape_); }

  template <typename... I>
  T& operator()(I... idx) const {
    static_assert(sizeof...(I) == M, "index count must equal the view's rank");
    const std::array<size_t, M> ix{size_t(idx)...};
    size_t off = 0;
    for (size_t d = 0; d != M; ++d) {
      assert(ix[d] < shape_[d]);
      off += ix[d] * strides_[d];
    }
    return base_[off];
  }

  // Row-major traversal: f(element reference, flat index).
  template <typename F>
  void for_each(F&& f) const {
    const size_t n = size();
    std::array<size_t, M> ix{};
    for (size_t flat = 0; flat != n; ++flat) {
      size_t off = 0;
      for (size_t d = 0; d != M; ++d) off += ix[d] * strides_[d];
      f(base_[off], flat);
      for (size_t d = M; d-- > 0;) {
        if (++ix[d] < shape_[d]) break;
        ix[d] = 0;
      }
    }
  }
  void copy_to(value_type* out) const {
    for_each([&](T& v, size_t i) { out[i] = v; });
  }
  template <typename U>
  const strided_view& operator=(const xtensor<U, M>& src) const {
    assert(src.size() == size());
    for_each([&](T& v, size_t i) { v = src.data()[i]; });
    return *this;
  }
  template <typename U, size_t K>
  const strided_view& operator/=(const strided_view<U, K>& other) const {
    static_assert(K == M, "ranks must agree");
    std::vector<value_type> tmp(other.size());
    other.copy_to(tmp.data());
    for_each([&](T& v, size_t i) { v /= tmp[i]; });
    return *this;
  }
  void fill(const value_type& value) const {
    for_each([&](T& v, size_t) { v = value; });
  }

 private:
  T* base_;
  std::array<size_t, M> shape_;
  std::array<size_t, M> strides_;
};

namespace detail {
template <typename E>
auto* DataOf(E& e) {
  return e.data();
}
template <size_t N>
std::array<size_t, N> RowMajorStrides(const std::array<size_t, N>& shape) {
  std::array<size_t, N> s{};
  size_t acc = 1;
  for (size_t d = N; d-- > 0;) {
    s[d] = acc;
    acc *= shape[d];
  }
  return s;
}
template <typename A>
constexpr size_t KeptDims() {
  return std::is_same_v<std::decay_t<A>, all_tag> ? 1 : 0;
}
}  // namespace detail

// xt::view(e, args...): one argument per dimension of e (integers or all()).
template <typename E, typename... Args>
auto view(E& e, Args... args) {
  constexpr size_t N = std::decay_t<decltype(e.shape())>{}.size();
  static_assert(sizeof...(Args) == N, "one argument per dimension");
  constexpr size_t M = (detail::KeptDims<Args>() + ...);
  using T = std::remove_pointer_t<decltype(detail::DataOf(e))>;
  const auto& shape = e.shape();
  const std::array<size_t, N> strides = detail::RowMajorStrides<N>(shape);
  std::array<size_t, M> vs{}, vst{};
  size_t offset = 0, d = 0, k = 0;
  auto one = [&](auto a) {
    if constexpr (std::is_same_v<std::decay_t<decltype(a)>, all_tag>) {
      vs[k] = shape[d];
      vst[k] = strides[d];
      ++k;
    } else {
      assert(size_t(a) < shape[d]);
      offset += size_t(a) * strides[d];
    }
    ++d;
  };
  (one(args), ...);
  return strided_view<T, M>(detail::DataOf(e) + offset, vs, vst);
}

// xt::reshape_view(e, {shape...}): the same contiguous data with a new shape.
template <typename E, size_t M>
auto reshape_view(E& e, const size_t (&shape)[M]) {
  using T = std::remove_pointer_t<decltype(detail::DataOf(e))>;
  std::array<size_t, M> s;
  for (size_t i = 0; i != M; ++i) s[i] = shape[i];
  assert(detail::Product(s) == e.size());
  return strided_view<T, M>(detail::DataOf(e), s, detail::RowMajorStrides<M>(s));
}

// xt::isfinite over a view: an owning boolean tensor of the view's shape.
template <typename T, size_t M>
xtensor<bool, M> isfinite(const strided_view<T, M>& v) {
  xtensor<bool, M> out(v.shape());
  v.for_each([&](T& x, size_t i) { out.data()[i] = detail::IsFiniteValue(x); });
  return out;
}

// xt::sum(e)(): the sum of all elements (booleans count as 0 / 1), evaluated
// when called, as DP3 uses the reducer.
template <typename T>
struct sum_result {
  T value;
  T operator()() const { return value; }
};
template <typename T, size_t N>
auto sum(const xtensor<T, N>& t) {
  using R = std::conditional_t<std::is_same_v<T, bool>, size_t, T>;
  R s = R(0);
  for (size_t i = 0; i != t.size(); ++i) s += R(t.data()[i]);
  return sum_result<R>{s};
}

}  // namespace xt

#endif

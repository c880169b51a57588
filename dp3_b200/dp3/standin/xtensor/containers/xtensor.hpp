// Stand-in for the subset of xtensor that DP3's DDECal solver, SolveData and
// constraint sources use (xtensor is fetched by DP3's build, absent here).
// Eager and row-major only: xt::xtensor<T, N> owns a contiguous buffer; the
// views (xview.hpp) are strided references into contiguous storage; the
// elementwise functions DP3 calls (zeros, isfinite, cast, !, +=, /=) return
// or update whole tensors at once. Only for building DP3's sources and the
// SolverBase adapter outside a DP3 tree; a DP3 build uses the real xtensor.
#ifndef DP3B200_STANDIN_XTENSOR_CONTAINERS_XTENSOR_HPP
#define DP3B200_STANDIN_XTENSOR_CONTAINERS_XTENSOR_HPP

#include <array>
#include <cassert>
#include <cmath>
#include <complex>
#include <cstddef>
#include <cstdint>
#include <initializer_list>
#include <type_traits>
#include <vector>

namespace xt {

namespace detail {
template <size_t N>
size_t Product(const std::array<size_t, N>& s) {
  size_t p = 1;
  for (size_t v : s) p *= v;
  return p;
}
template <typename T>
bool IsFiniteValue(const T& v) {
  return std::isfinite(v);
}
template <typename T>
bool IsFiniteValue(const std::complex<T>& v) {
  return std::isfinite(v.real()) && std::isfinite(v.imag());
}
}  // namespace detail

template <typename T, size_t N>
class xtensor {
 public:
  using value_type = T;
  // bool elements are stored as bytes (std::vector<bool> has no data())
  using storage_type = std::conditional_t<std::is_same_v<T, bool>, unsigned char, T>;
  using shape_type = std::array<size_t, N>;
  using iterator = typename std::vector<storage_type>::iterator;
  using const_iterator = typename std::vector<storage_type>::const_iterator;
  static constexpr size_t rank = N;

  xtensor() { shape_.fill(0); }
  explicit xtensor(const shape_type& shape) : shape_(shape), data_(detail::Product(shape)) {}
  xtensor(const shape_type& shape, const T& value)
      : shape_(shape), data_(detail::Product(shape), value) {}
  xtensor(const xtensor&) = default;
  xtensor(xtensor&&) noexcept = default;
  xtensor& operator=(const xtensor&) = default;
  xtensor& operator=(xtensor&&) noexcept = default;

  // Converting assignment (e.g. xtensor<size_t, N> = isfinite(...)).
  template <typename U, typename = std::enable_if_t<!std::is_same_v<U, T>>>
  xtensor& operator=(const xtensor<U, N>& other) {
    shape_ = other.shape();
    data_.resize(other.size());
    for (size_t i = 0; i != data_.size(); ++i)
      data_[i] = static_cast<storage_type>(static_cast<T>(other.data()[i]));
    return *this;
  }
  // Assignment from any view with rank N (xview.hpp).
  template <typename View, typename = decltype(std::declval<const View&>().is_xt_view())>
  xtensor& operator=(const View& v) {
    shape_ = v.shape();
    data_.resize(detail::Product(shape_));
    v.copy_to(data_.data());
    return *this;
  }

  void resize(const shape_type& shape) {
    shape_ = shape;
    data_.resize(detail::Product(shape));
  }

  const shape_type& shape() const { return shape_; }
  size_t shape(size_t i) const { return shape_[i]; }
  size_t size() const { return data_.size(); }
  size_t dimension() const { return N; }
  storage_type* data() { return data_.data(); }
  const storage_type* data() const { return data_.data(); }
  iterator begin() { return data_.begin(); }
  iterator end() { return data_.end(); }
  const_iterator begin() const { return data_.begin(); }
  const_iterator end() const { return data_.end(); }

  template <typename... I>
  storage_type& operator()(I... idx) {
    static_assert(sizeof...(I) == N, "index count must equal the rank");
    return data_[Offset({size_t(idx)...})];
  }
  template <typename... I>
  const storage_type& operator()(I... idx) const {
    static_assert(sizeof...(I) == N, "index count must equal the rank");
    return data_[Offset({size_t(idx)...})];
  }

  void fill(const T& v) { std::fill(data_.begin(), data_.end(), v); }

  template <typename U>
  xtensor& operator+=(const xtensor<U, N>& o) {
    assert(o.size() == size());
    for (size_t i = 0; i != data_.size(); ++i) data_[i] += o.data()[i];
    return *this;
  }
  template <typename U>
  xtensor& operator/=(const xtensor<U, N>& o) {
    assert(o.size() == size());
    for (size_t i = 0; i != data_.size(); ++i) data_[i] /= o.data()[i];
    return *this;
  }

 private:
  size_t Offset(const std::array<size_t, N>& idx) const {
    size_t off = 0;
    for (size_t d = 0; d != N; ++d) {
      assert(idx[d] < shape_[d]);
      off = off * shape_[d] + idx[d];
    }
    return off;
  }

  shape_type shape_;
  std::vector<storage_type> data_;
};

template <typename T, size_t N>
xtensor<T, N> zeros(const size_t (&shape)[N]) {
  std::array<size_t, N> s;
  for (size_t i = 0; i != N; ++i) s[i] = shape[i];
  return xtensor<T, N>(s, T(0));
}

template <typename T, size_t N>
xtensor<bool, N> isfinite(const xtensor<T, N>& t) {
  xtensor<bool, N> out(t.shape());
  for (size_t i = 0; i != t.size(); ++i) out.data()[i] = detail::IsFiniteValue(t.data()[i]);
  return out;
}

template <typename T, size_t N>
xtensor<bool, N> operator!(const xtensor<T, N>& t) {
  xtensor<bool, N> out(t.shape());
  for (size_t i = 0; i != t.size(); ++i) out.data()[i] = !t.data()[i];
  return out;
}

template <typename To, typename T, size_t N>
xtensor<To, N> cast(const xtensor<T, N>& t) {
  xtensor<To, N> out(t.shape());
  for (size_t i = 0; i != t.size(); ++i) out.data()[i] = static_cast<To>(t.data()[i]);
  return out;
}

}  // namespace xt

// DP3's sources call xt::reshape_view after including only this header.
#include "../views/xview.hpp"

#endif

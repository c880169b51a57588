// Stand-in for the subset of xsimd that DP3's SolverBase::Step uses in its
// phase-only branch (ddecal/gain_solvers/SolverBase.cc:117-155): batches of
// width 1, so every operation is the scalar std:: function it vectorises
// (arg = std::arg, polar = std::polar). Only for building DP3's sources
// outside a DP3 tree; a DP3 build uses the real xsimd.
#ifndef DP3B200_STANDIN_XSIMD_XSIMD_HPP
#define DP3B200_STANDIN_XSIMD_XSIMD_HPP

#include <complex>
#include <cstddef>

namespace xsimd {

template <typename T>
struct batch_bool {
  bool v;
};

template <typename T>
struct batch {
  static constexpr size_t size = 1;
  T v;
  batch() = default;
  batch(T x) : v(x) {}
  static batch load_unaligned(const T* p) { return batch(*p); }
  void store_unaligned(T* p) const { *p = v; }
  batch& operator+=(const batch& o) {
    v += o.v;
    return *this;
  }
  batch& operator-=(const batch& o) {
    v -= o.v;
    return *this;
  }
};

template <typename T>
batch<T> operator-(const batch<T>& a) {
  return batch<T>(-a.v);
}
template <typename T>
batch<T> operator+(const batch<T>& a, const batch<T>& b) {
  return batch<T>(a.v + b.v);
}
template <typename T>
batch<T> operator-(const batch<T>& a, const batch<T>& b) {
  return batch<T>(a.v - b.v);
}
template <typename T>
batch<T> operator*(const batch<T>& a, const batch<T>& b) {
  return batch<T>(a.v * b.v);
}
template <typename T>
batch<T> operator*(T s, const batch<T>& b) {
  return batch<T>(s * b.v);
}
template <typename T>
batch<T> operator*(const batch<T>& b, T s) {
  return batch<T>(b.v * s);
}

inline batch<double> broadcast(double x) { return batch<double>(x); }
inline batch<float> broadcast(float x) { return batch<float>(x); }

template <typename T>
batch_bool<T> gt(const batch<T>& a, const batch<T>& b) {
  return {a.v > b.v};
}
template <typename T>
batch_bool<T> lt(const batch<T>& a, const batch<T>& b) {
  return {a.v < b.v};
}
template <typename T>
batch<T> select(const batch_bool<T>& c, const batch<T>& a, const batch<T>& b) {
  return c.v ? a : b;
}

template <typename T>
batch<T> arg(const batch<std::complex<T>>& z) {
  return batch<T>(std::arg(z.v));
}
template <typename T>
batch<std::complex<T>> polar(const batch<T>& r, const batch<T>& theta) {
  return batch<std::complex<T>>(std::polar(r.v, theta.v));
}

}  // namespace xsimd

#endif

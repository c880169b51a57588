// Stand-in for the subset of aocommon's diagonal 2x2 matrix header that
// DP3's DDECal solver sources use: diag(a, b), with the products that mix it
// with a full row-major 2x2 matrix (a diagonal on the left scales the rows,
// on the right the columns). Only for building DP3's sources outside a DP3
// tree; a DP3 build uses the real aocommon.
#ifndef DP3B200_STANDIN_AOCOMMON_MATRIX2X2DIAG_H
#define DP3B200_STANDIN_AOCOMMON_MATRIX2X2DIAG_H

#include <complex>

#include "matrix2x2.h"

namespace aocommon {

template <typename T>
class MC2x2DiagBase {
 public:
  using value_type = std::complex<T>;

  MC2x2DiagBase() = default;
  MC2x2DiagBase(value_type a, value_type b) : v_{a, b} {}
  template <typename U>
  explicit MC2x2DiagBase(const MC2x2DiagBase<U>& other)
      : v_{value_type(other.Get(0)), value_type(other.Get(1))} {}

  static MC2x2DiagBase Zero() { return MC2x2DiagBase(0, 0); }
  static MC2x2DiagBase Unity() { return MC2x2DiagBase(1, 1); }

  const value_type& Get(size_t i) const { return v_[i]; }
  void Set(size_t i, value_type value) { v_[i] = value; }
  value_type& operator[](size_t i) { return v_[i]; }
  const value_type& operator[](size_t i) const { return v_[i]; }

  MC2x2DiagBase& operator+=(const MC2x2DiagBase& r) {
    v_[0] += r.v_[0];
    v_[1] += r.v_[1];
    return *this;
  }
  MC2x2DiagBase& operator-=(const MC2x2DiagBase& r) {
    v_[0] -= r.v_[0];
    v_[1] -= r.v_[1];
    return *this;
  }
  MC2x2DiagBase operator+(const MC2x2DiagBase& r) const {
    return MC2x2DiagBase(v_[0] + r.v_[0], v_[1] + r.v_[1]);
  }
  MC2x2DiagBase operator-(const MC2x2DiagBase& r) const {
    return MC2x2DiagBase(v_[0] - r.v_[0], v_[1] - r.v_[1]);
  }
  MC2x2DiagBase operator*(const MC2x2DiagBase& r) const {
    return MC2x2DiagBase(v_[0] * r.v_[0], v_[1] * r.v_[1]);
  }
  MC2x2DiagBase operator*(value_type s) const { return MC2x2DiagBase(v_[0] * s, v_[1] * s); }
  // diag * full: row r scaled by v_[r]
  MC2x2Base<T> operator*(const MC2x2Base<T>& m) const {
    return MC2x2Base<T>(v_[0] * m.Get(0), v_[0] * m.Get(1), v_[1] * m.Get(2), v_[1] * m.Get(3));
  }

 private:
  value_type v_[2];
};

// full * diag: column c scaled by d[c]
template <typename T>
MC2x2Base<T> operator*(const MC2x2Base<T>& m, const MC2x2DiagBase<T>& d) {
  return MC2x2Base<T>(m.Get(0) * d.Get(0), m.Get(1) * d.Get(1), m.Get(2) * d.Get(0),
                      m.Get(3) * d.Get(1));
}

template <typename T>
MC2x2DiagBase<T> HermTranspose(const MC2x2DiagBase<T>& d) {
  return MC2x2DiagBase<T>(std::conj(d.Get(0)), std::conj(d.Get(1)));
}

template <typename T>
MC2x2DiagBase<T> Diagonal(const MC2x2Base<T>& m) {
  return MC2x2DiagBase<T>(m.Get(0), m.Get(3));
}

template <typename T>
MC2x2DiagBase<T> Diagonal(const MC2x2DiagBase<T>& d) {
  return d;
}

template <typename T>
std::complex<T> Trace(const MC2x2DiagBase<T>& d) {
  return d.Get(0) + d.Get(1);
}

template <typename T>
T Norm(const MC2x2DiagBase<T>& d) {
  return std::norm(d.Get(0)) + std::norm(d.Get(1));
}

using MC2x2FDiag = MC2x2DiagBase<float>;
using MC2x2Diag = MC2x2DiagBase<double>;

}  // namespace aocommon

#endif

// Stand-in for the subset of aocommon's 2x2 matrix header that DP3's DDECal
// solver sources use (aocommon is a git submodule of DP3, absent from its
// source tree here). Written from the documented semantics: a row-major 2x2
// complex matrix [XX XY; YX YY], element i = row * 2 + column (comment at
// ddecal/gain_solvers/IterativeDiagonalSolver.cc:21-23), HermTranspose the
// conjugate transpose, Diagonal the diagonal part, Trace the sum of the
// diagonal, Norm the squared Frobenius norm (the CUDA restatement in
// ddecal/gain_solvers/kernels/MatrixComplex2x2.h:9-116 follows the same
// conventions). Only for building DP3's sources and the SolverBase adapter
// outside a DP3 tree; a DP3 build uses the real aocommon.
#ifndef DP3B200_STANDIN_AOCOMMON_MATRIX2X2_H
#define DP3B200_STANDIN_AOCOMMON_MATRIX2X2_H

#include <cmath>
#include <complex>
#include <limits>

namespace aocommon {

template <typename T>
class MC2x2Base {
 public:
  using value_type = std::complex<T>;

  MC2x2Base() = default;
  MC2x2Base(value_type a, value_type b, value_type c, value_type d) : v_{a, b, c, d} {}
  template <typename U>
  explicit MC2x2Base(const std::complex<U>* values)
      : v_{value_type(values[0]), value_type(values[1]), value_type(values[2]),
           value_type(values[3])} {}
  template <typename U>
  explicit MC2x2Base(const MC2x2Base<U>& other)
      : v_{value_type(other.Get(0)), value_type(other.Get(1)), value_type(other.Get(2)),
           value_type(other.Get(3))} {}

  static MC2x2Base Zero() { return MC2x2Base(0, 0, 0, 0); }
  static MC2x2Base Unity() { return MC2x2Base(1, 0, 0, 1); }
  static MC2x2Base NaN() {
    const T n = std::numeric_limits<T>::quiet_NaN();
    return MC2x2Base(value_type(n, n), value_type(n, n), value_type(n, n), value_type(n, n));
  }

  // this * rhs^H
  MC2x2Base MultiplyHerm(const MC2x2Base& r) const {
    return MC2x2Base(v_[0] * std::conj(r.v_[0]) + v_[1] * std::conj(r.v_[1]),
                     v_[0] * std::conj(r.v_[2]) + v_[1] * std::conj(r.v_[3]),
                     v_[2] * std::conj(r.v_[0]) + v_[3] * std::conj(r.v_[1]),
                     v_[2] * std::conj(r.v_[2]) + v_[3] * std::conj(r.v_[3]));
  }
  // The four elements, converted, into dest[0..3].
  template <typename U>
  void AssignTo(std::complex<U>* dest) const {
    for (int i = 0; i != 4; ++i) dest[i] = std::complex<U>(v_[i]);
  }

  const value_type& Get(size_t i) const { return v_[i]; }
  void Set(size_t i, value_type value) { v_[i] = value; }
  value_type& operator[](size_t i) { return v_[i]; }
  const value_type& operator[](size_t i) const { return v_[i]; }
  const value_type* Data() const { return v_; }

  MC2x2Base& operator+=(const MC2x2Base& r) {
    for (int i = 0; i != 4; ++i) v_[i] += r.v_[i];
    return *this;
  }
  MC2x2Base& operator-=(const MC2x2Base& r) {
    for (int i = 0; i != 4; ++i) v_[i] -= r.v_[i];
    return *this;
  }
  MC2x2Base& operator*=(const MC2x2Base& r) {
    *this = *this * r;
    return *this;
  }
  MC2x2Base& operator*=(value_type s) {
    for (int i = 0; i != 4; ++i) v_[i] *= s;
    return *this;
  }
  MC2x2Base operator+(const MC2x2Base& r) const {
    MC2x2Base m(*this);
    return m += r;
  }
  MC2x2Base operator-(const MC2x2Base& r) const {
    MC2x2Base m(*this);
    return m -= r;
  }
  MC2x2Base operator*(const MC2x2Base& r) const {
    return MC2x2Base(v_[0] * r.v_[0] + v_[1] * r.v_[2], v_[0] * r.v_[1] + v_[1] * r.v_[3],
                     v_[2] * r.v_[0] + v_[3] * r.v_[2], v_[2] * r.v_[1] + v_[3] * r.v_[3]);
  }
  MC2x2Base operator*(value_type s) const {
    return MC2x2Base(v_[0] * s, v_[1] * s, v_[2] * s, v_[3] * s);
  }

  // In-place inverse; false (and unchanged) when the determinant is zero.
  bool Invert() {
    const value_type det = v_[0] * v_[3] - v_[1] * v_[2];
    if (det == value_type(0)) return false;
    const value_type inv = value_type(1) / det;
    const value_type a = v_[0];
    v_[0] = v_[3] * inv;
    v_[1] = -v_[1] * inv;
    v_[2] = -v_[2] * inv;
    v_[3] = a * inv;
    return true;
  }

 private:
  value_type v_[4];
};

template <typename T>
MC2x2Base<T> operator*(std::complex<T> s, const MC2x2Base<T>& m) {
  return m * s;
}

template <typename T>
MC2x2Base<T> HermTranspose(const MC2x2Base<T>& m) {
  return MC2x2Base<T>(std::conj(m.Get(0)), std::conj(m.Get(2)), std::conj(m.Get(1)),
                      std::conj(m.Get(3)));
}

template <typename T>
std::complex<T> Trace(const MC2x2Base<T>& m) {
  return m.Get(0) + m.Get(3);
}

template <typename T>
T Norm(const MC2x2Base<T>& m) {
  return std::norm(m.Get(0)) + std::norm(m.Get(1)) + std::norm(m.Get(2)) +
         std::norm(m.Get(3));
}

using MC2x2F = MC2x2Base<float>;
using MC2x2 = MC2x2Base<double>;

struct Matrix2x2 {
  template <typename T>
  static bool IsFinite(const std::complex<T>* m) {
    for (int i = 0; i != 4; ++i)
      if (!std::isfinite(m[i].real()) || !std::isfinite(m[i].imag())) return false;
    return true;
  }
};

}  // namespace aocommon

// DP3's sources use MC2x2FDiag after including only this header.
#include "matrix2x2diag.h"

#endif

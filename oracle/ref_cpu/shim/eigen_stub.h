// Stand-in for the Eigen 3 matrix types named by the reference's headers
// (see eigen3/Eigen/Core in this directory), used ONLY to compile and run
// the reference's sources on the CPU (test infrastructure).  Column-major
// fixed-size storage as Eigen's, with the element access, comma
// initialisation and the few element-wise operations that
// include/solver/gnSolver/gnSolver.cu names.  The two numerical routines
// the reference takes from Eigen -- the 6x6 LDLT solve and the exponential
// of an se(3) twist matrix (gnSolver.cu:439-445) -- are the oracle's own
// (../../gn_algebra.h), so a reference solve driven through this header
// and the oracle share that algebra and differ only where the reference's
// own code does.  exp() accepts only twist matrices (bottom row zero).
#pragma once
#include <cmath>
#include <cstdio>
#include <cstdlib>

#include "../../gn_algebra.h"

namespace Eigen {

template <class S, int R, int C>
struct Matrix {
  S v[R * C];

  S& operator()(int r, int c) { return v[c * R + r]; }
  const S& operator()(int r, int c) const { return v[c * R + r]; }
  S& operator()(int i) { return v[i]; }
  const S& operator()(int i) const { return v[i]; }
  S* data() { return v; }
  const S* data() const { return v; }

  // m << a, b, c, ...: row by row
  struct CommaInit {
    Matrix* m;
    int k;
    template <class T>
    CommaInit& operator,(T x) {
      (*m)(k / C, k % C) = (S)x;
      ++k;
      return *this;
    }
  };
  template <class T>
  CommaInit operator<<(T x) {
    (*this)(0, 0) = (S)x;
    return CommaInit{this, 1};
  }

  S sum() const {
    S s = 0;
    for (int i = 0; i < R * C; ++i) s += v[i];
    return s;
  }
  S norm() const {
    S s = 0;
    for (int i = 0; i < R * C; ++i) s += v[i] * v[i];
    return std::sqrt(s);
  }
  S maxCoeff() const {
    S s = v[0];
    for (int i = 1; i < R * C; ++i) s = v[i] > s ? v[i] : s;
    return s;
  }
  Matrix& operator*=(S x) {
    for (int i = 0; i < R * C; ++i) v[i] *= x;
    return *this;
  }
  Matrix operator+(const Matrix& o) const {
    Matrix r;
    for (int i = 0; i < R * C; ++i) r.v[i] = v[i] + o.v[i];
    return r;
  }
  Matrix operator-(const Matrix& o) const {
    Matrix r;
    for (int i = 0; i < R * C; ++i) r.v[i] = v[i] - o.v[i];
    return r;
  }
  friend Matrix operator*(S x, const Matrix& m) {
    Matrix r;
    for (int i = 0; i < R * C; ++i) r.v[i] = x * m.v[i];
    return r;
  }
  template <int K>
  Matrix<S, R, K> operator*(const Matrix<S, C, K>& o) const {
    Matrix<S, R, K> r;
    for (int i = 0; i < R; ++i)
      for (int j = 0; j < K; ++j) {
        S s = 0;
        for (int k = 0; k < C; ++k) s += (*this)(i, k) * o(k, j);
        r(i, j) = s;
      }
    return r;
  }
  template <class T>
  Matrix<T, R, C> cast() const {
    Matrix<T, R, C> r;
    for (int i = 0; i < R * C; ++i) r.v[i] = (T)v[i];
    return r;
  }

  // A.ldlt().solve(b) for the 6x6 systems of gnSolver.cu:439-442 (a zero
  // pivot gives NaN, which the reference's NaN guard then zeroes)
  struct LDLT {
    const Matrix* a;
    Matrix<S, C, 1> solve(const Matrix<S, C, 1>& b) const {
      static_assert(R == 6 && C == 6, "the shim solves 6x6 systems only");
      double A[36], bb[6], x[6] = {0, 0, 0, 0, 0, 0};
      for (int i = 0; i < 6; ++i) {
        for (int j = 0; j < 6; ++j) A[i * 6 + j] = (double)(*a)(i, j);
        bb[i] = (double)b(i);
      }
      Matrix<S, C, 1> r;
      if (!dyo_gn::ldlt6(A, bb, x))
        for (int i = 0; i < 6; ++i) x[i] = NAN;
      for (int i = 0; i < 6; ++i) r(i) = (S)x[i];
      return r;
    }
  };
  LDLT ldlt() const { return LDLT{this}; }
  // exp() of v2t(xi) (gnSolver.cu:443-455): xi read back from the twist
  Matrix exp() const {
    static_assert(R == 4 && C == 4, "the shim exponentiates 4x4 twists only");
    if ((*this)(3, 0) != 0 || (*this)(3, 1) != 0 || (*this)(3, 2) != 0 || (*this)(3, 3) != 0) {
      std::fprintf(stderr, "eigen shim: exp() of a matrix that is not a twist\n");
      std::abort();
    }
    const double xi[6] = {(double)(*this)(2, 1), (double)(*this)(0, 2), (double)(*this)(1, 0),
                          (double)(*this)(0, 3), (double)(*this)(1, 3), (double)(*this)(2, 3)};
    double T[16];
    dyo_gn::se3_exp(xi, T);
    Matrix r;
    for (int i = 0; i < 4; ++i)
      for (int j = 0; j < 4; ++j) r(i, j) = (S)T[i * 4 + j];
    return r;
  }
};

typedef Matrix<float, 4, 4> Matrix4f;
typedef Matrix<double, 4, 4> Matrix4d;
typedef Matrix<float, 3, 3> Matrix3f;
typedef Matrix<double, 3, 3> Matrix3d;
typedef Matrix<float, 3, 1> Vector3f;
typedef Matrix<double, 3, 1> Vector3d;
typedef Matrix<double, 6, 1> Vector6d;

// gnSolver.cu adds a 6x6 identity written as MatrixXd::Identity(6, 6).
struct MatrixXd {
  static Matrix<double, 6, 6> Identity(int r, int c) {
    if (r != 6 || c != 6) std::abort();
    Matrix<double, 6, 6> m;
    for (int i = 0; i < 36; ++i) m.v[i] = (i % 7 == 0) ? 1.0 : 0.0;
    return m;
  }
};

}  // namespace Eigen

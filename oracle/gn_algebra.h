// gn_algebra.h -- the FP64 6x6 LDL^T solve and the closed-form SE(3)
// exponential of the oracle (test infrastructure), header-only so that the
// Eigen stand-in used to build the reference's gnSolver.cu for the CPU
// (ref_cpu/shim/eigen_stub.h) runs exactly the same arithmetic.  The
// reference calls Eigen for both (gnSolver.cu:439-445); Eigen is absent, so
// these are the published methods it computes, not Eigen's code.
#pragma once
#include <cmath>

namespace dyo_gn {

// Solve A x = b, A symmetric positive definite (6x6): LDL^T without
// pivoting.  Stands in for Eigen's A.ldlt().solve(b) (gnSolver.cu:439-442).
inline int ldlt6(const double* A, const double* b, double* x) {
  double L[36] = {0}, D[6];
  for (int j = 0; j < 6; ++j) {
    double s = A[j * 6 + j];
    for (int k = 0; k < j; ++k) s -= L[j * 6 + k] * L[j * 6 + k] * D[k];
    D[j] = s;
    if (!(std::fabs(s) > 0)) return 0;
    L[j * 6 + j] = 1;
    for (int i = j + 1; i < 6; ++i) {
      double t = A[i * 6 + j];
      for (int k = 0; k < j; ++k) t -= L[i * 6 + k] * L[j * 6 + k] * D[k];
      L[i * 6 + j] = t / D[j];
    }
  }
  double y[6];
  for (int i = 0; i < 6; ++i) {
    double t = b[i];
    for (int k = 0; k < i; ++k) t -= L[i * 6 + k] * y[k];
    y[i] = t;
  }
  for (int i = 0; i < 6; ++i) y[i] /= D[i];
  for (int i = 5; i >= 0; --i) {
    double t = y[i];
    for (int k = i + 1; k < 6; ++k) t -= L[k * 6 + i] * x[k];
    x[i] = t;
  }
  return 1;
}

// exp of the twist matrix v2t(xi) (gnSolver.cu:446-455, Eigen exp at :443):
// closed form R = I + a W + b W^2, t = (I + b W + c W^2) v with
// a = sin(th)/th, b = (1-cos th)/th^2, c = (th - sin th)/th^3 (Rodrigues
// and the SE(3) left Jacobian); Taylor series below th = 1e-4.
inline void se3_exp(const double* xi, double* T) {
  double w0 = xi[0], w1 = xi[1], w2 = xi[2];
  double th2 = w0 * w0 + w1 * w1 + w2 * w2, th = std::sqrt(th2);
  double a, b, c;
  if (th < 1e-4) {
    a = 1.0 - th2 / 6.0;
    b = 0.5 - th2 / 24.0;
    c = 1.0 / 6.0 - th2 / 120.0;
  } else {
    a = std::sin(th) / th;
    b = (1.0 - std::cos(th)) / th2;
    c = (th - std::sin(th)) / (th2 * th);
  }
  double W[9] = {0, -w2, w1, w2, 0, -w0, -w1, w0, 0};
  double W2[9];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      double s = 0;
      for (int k = 0; k < 3; ++k) s += W[i * 3 + k] * W[k * 3 + j];
      W2[i * 3 + j] = s;
    }
  double Rm[9], Vm[9];
  for (int i = 0; i < 9; ++i) {
    double I = (i % 4 == 0) ? 1.0 : 0.0;
    Rm[i] = I + a * W[i] + b * W2[i];
    Vm[i] = I + b * W[i] + c * W2[i];
  }
  for (int i = 0; i < 3; ++i) {
    for (int j = 0; j < 3; ++j) T[i * 4 + j] = Rm[i * 3 + j];
    T[i * 4 + 3] = Vm[i * 3 + 0] * xi[3] + Vm[i * 3 + 1] * xi[4] + Vm[i * 3 + 2] * xi[5];
  }
  T[12] = T[13] = T[14] = 0;
  T[15] = 1;
}

}  // namespace dyo_gn

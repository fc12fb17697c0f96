// Type-only stand-in for the Eigen 3 matrix types named by the reference's
// headers (see eigen3/Eigen/Core in this directory).
#pragma once
namespace Eigen {
template <class S, int R, int C>
struct Matrix {
  S v[R * C];
};
typedef Matrix<float, 4, 4> Matrix4f;
typedef Matrix<double, 4, 4> Matrix4d;
typedef Matrix<float, 3, 3> Matrix3f;
typedef Matrix<double, 3, 3> Matrix3d;
typedef Matrix<float, 3, 1> Vector3f;
typedef Matrix<double, 3, 1> Vector3d;
typedef Matrix<double, 6, 1> Vector6d;
}  // namespace Eigen

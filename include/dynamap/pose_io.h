// dynamap/pose_io.h -- TUM-format trajectory lines and the quaternion <->
// rotation conversions behind them (header-only, no dependencies).
//
// The reference writes one line per frame with builder::writePoseToTxt
// (include/builder/builder.cu:243-257): "stamp tx ty tz qx qy qz qw" in
// fixed notation with 4 decimals, the quaternion taken from the pose's
// rotation by Eigen; it reads ground-truth lines with builder::v2tRef
// (builder.cu:222-241) and dataSet::getCurrentPose (utils_Dataset.cpp:69-88):
// the quaternion normalised, turned into a rotation in double and rounded to
// float.  Eigen is not available here; the conversions below are the
// published methods those calls implement, in double:
//   rotation -> quaternion: Shoemake, "Animating rotation with quaternion
//     curves" (SIGGRAPH 1985) -- from the trace when it is positive, else
//     from the largest diagonal element;
//   quaternion -> rotation: the standard homogeneous form of a unit
//     quaternion's rotation.
#pragma once

#include <cmath>
#include <cstdio>
#include <string>

namespace DynaMap {
namespace pose_io {

// q = {x, y, z, w}
struct Quat {
  double x = 0.0, y = 0.0, z = 0.0, w = 1.0;
};

// m[r][c] of a rotation matrix (double) -> unit quaternion.
inline Quat quat_from_rotation(const double m[3][3]) {
  Quat q;
  double t = m[0][0] + m[1][1] + m[2][2];
  if (t > 0.0) {
    double s = std::sqrt(t + 1.0);
    q.w = 0.5 * s;
    s = 0.5 / s;
    q.x = (m[2][1] - m[1][2]) * s;
    q.y = (m[0][2] - m[2][0]) * s;
    q.z = (m[1][0] - m[0][1]) * s;
  } else {
    int i = 0;
    if (m[1][1] > m[0][0]) i = 1;
    if (m[2][2] > m[i][i]) i = 2;
    const int j = (i + 1) % 3, k = (j + 1) % 3;
    double v[3];
    double s = std::sqrt(m[i][i] - m[j][j] - m[k][k] + 1.0);
    v[i] = 0.5 * s;
    s = 0.5 / s;
    q.w = (m[k][j] - m[j][k]) * s;
    v[j] = (m[j][i] + m[i][j]) * s;
    v[k] = (m[k][i] + m[i][k]) * s;
    q.x = v[0];
    q.y = v[1];
    q.z = v[2];
  }
  return q;
}

// Quaternion (normalised first) -> rotation matrix r[r][c], in double.
inline void rotation_from_quat(Quat q, double r[3][3]) {
  const double n = std::sqrt(q.x * q.x + q.y * q.y + q.z * q.z + q.w * q.w);
  q.x /= n;
  q.y /= n;
  q.z /= n;
  q.w /= n;
  const double tx = 2.0 * q.x, ty = 2.0 * q.y, tz = 2.0 * q.z;
  const double twx = tx * q.w, twy = ty * q.w, twz = tz * q.w;
  const double txx = tx * q.x, txy = ty * q.x, txz = tz * q.x;
  const double tyy = ty * q.y, tyz = tz * q.y, tzz = tz * q.z;
  r[0][0] = 1.0 - (tyy + tzz);
  r[0][1] = txy - twz;
  r[0][2] = txz + twy;
  r[1][0] = txy + twz;
  r[1][1] = 1.0 - (txx + tzz);
  r[1][2] = tyz - twx;
  r[2][0] = txz - twy;
  r[2][1] = tyz + twx;
  r[2][2] = 1.0 - (txx + tyy);
}

// A TUM line {stamp, tx, ty, tz, qx, qy, qz, qw} -> row-major float 4x4
// camera-to-world pose (v2tRef: translation and rotation rounded to float).
inline void pose_from_tum(const double v[8], float pose[16]) {
  Quat q;
  q.x = v[4];
  q.y = v[5];
  q.z = v[6];
  q.w = v[7];
  double r[3][3];
  rotation_from_quat(q, r);
  for (int i = 0; i < 3; ++i) {
    for (int j = 0; j < 3; ++j) pose[i * 4 + j] = (float)r[i][j];
    pose[i * 4 + 3] = (float)v[1 + i];
  }
  pose[12] = pose[13] = pose[14] = 0.0f;
  pose[15] = 1.0f;
}

// The line writePoseToTxt appends for a row-major float 4x4 pose (no
// newline): stamp, translation, quaternion x y z w, "%.4f" each.
inline std::string tum_line(double stamp, const float pose[16]) {
  double m[3][3];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) m[i][j] = (double)pose[i * 4 + j];
  const Quat q = quat_from_rotation(m);
  char buf[256];
  std::snprintf(buf, sizeof buf, "%.4f %.4f %.4f %.4f %.4f %.4f %.4f %.4f", stamp,
                (double)pose[3], (double)pose[7], (double)pose[11], q.x, q.y, q.z, q.w);
  return std::string(buf);
}

}  // namespace pose_io
}  // namespace DynaMap

// dynamap/types.h -- the reference's small value types, for the C++ drop-in
// classes (header-only, over the C ABI of dynamap.h).
//
//   rgbdSensor      include/image/sensor/rgbdSensor.h:13-19
//   float4x4        include/math/utils_matrix.h:816-1177 (row-major m11..m44)
//   gaussianKernal  include/image/kernel2D/kernel2D.h:20-43
//   Matrix4f        stands in for Eigen::Matrix4f (column-major storage, as
//                   Eigen stores it), which the reference's builder and
//                   gnSolver use for poses (builder.h, gnSolver.h:72)
#pragma once

#include <cmath>
#include <cstdint>
#include <ostream>
#include <stdexcept>
#include <string>

#include "../dynamap.h"

// The CUDA vector types the reference's interfaces name (float3, int3,
// uchar3): CUDA's own when its headers are on the include path, else
// layout-compatible host structs (the library needs no CUDA headers).
#if defined(__has_include)
#if __has_include(<vector_types.h>) && __has_include(<vector_functions.h>)
#include <vector_types.h>
#include <vector_functions.h>
#define DYNAMAP_CUDA_VECTOR_TYPES 1
#endif
#endif
#ifndef DYNAMAP_CUDA_VECTOR_TYPES
struct float3 {
  float x, y, z;
};
struct int3 {
  int x, y, z;
};
struct uchar3 {
  unsigned char x, y, z;
};
inline float3 make_float3(float x, float y, float z) { return float3{x, y, z}; }
inline int3 make_int3(int x, int y, int z) { return int3{x, y, z}; }
inline uchar3 make_uchar3(unsigned char x, unsigned char y, unsigned char z) {
  return uchar3{x, y, z};
}
#endif

namespace DynaMap {

struct float2_ {
  float x, y;
};

struct rgbdSensor {
  unsigned int rows = 480;
  unsigned int cols = 640;
  float2_ f{525.0f, 525.0f};
  float2_ c{319.5f, 239.5f};
  float depthScaler = 5000.0f;

  dyn_sensor to_c() const {
    dyn_sensor s;
    s.rows = rows;
    s.cols = cols;
    s.fx = f.x;
    s.fy = f.y;
    s.cx = c.x;
    s.cy = c.y;
    s.depth_scaler = depthScaler;
    return s;
  }
};

struct gaussianKernal {
  int diameter = 8;
  float sigmaI = 10.0f;
  float sigmaS = 1.0f;
  float* kernel = nullptr;  // unused: the weights are computed on the fly
};

// Row-major 4x4, the reference's device matrix layout.
struct float4x4 {
  float entries[16];
  float4x4() {
    for (int i = 0; i < 16; ++i) entries[i] = (i % 5 == 0) ? 1.0f : 0.0f;
  }
  explicit float4x4(const float v[16]) {
    for (int i = 0; i < 16; ++i) entries[i] = v[i];
  }
  float& operator()(int r, int c) { return entries[r * 4 + c]; }
  float operator()(int r, int c) const { return entries[r * 4 + c]; }
  float4x4 getTranspose() const {
    float4x4 t;
    for (int r = 0; r < 4; ++r)
      for (int c = 0; c < 4; ++c) t.entries[c * 4 + r] = entries[r * 4 + c];
    return t;
  }
};

// Column-major 4x4 standing in for Eigen::Matrix4f.
struct Matrix4f {
  float data_[16];
  Matrix4f() {
    for (int i = 0; i < 16; ++i) data_[i] = (i % 5 == 0) ? 1.0f : 0.0f;
  }
  static Matrix4f Identity() { return Matrix4f(); }
  void setIdentity() { *this = Matrix4f(); }
  float& operator()(int r, int c) { return data_[c * 4 + r]; }
  float operator()(int r, int c) const { return data_[c * 4 + r]; }
  float* data() { return data_; }
  const float* data() const { return data_; }
  // builder.cu:102: float4x4(pose.data()).getTranspose()
  float4x4 to_row_major() const { return float4x4(data_).getTranspose(); }
  static Matrix4f from_row_major(const float* rm) {
    Matrix4f m;
    for (int r = 0; r < 4; ++r)
      for (int c = 0; c < 4; ++c) m(r, c) = rm[r * 4 + c];
    return m;
  }
};

// Eigen's stream form: four rows, entries separated by spaces
inline std::ostream& operator<<(std::ostream& os, const Matrix4f& m) {
  for (int r = 0; r < 4; ++r) {
    for (int c = 0; c < 4; ++c) os << (c ? " " : "") << m(r, c);
    if (r < 3) os << "\n";
  }
  return os;
}

typedef double Vector6d[6];

inline void dyn_throw(const char* what, dyn_status s) {
  if (s != DYN_OK)
    throw std::runtime_error(std::string(what) + ": " + dyn_status_string(s));
}

}  // namespace DynaMap

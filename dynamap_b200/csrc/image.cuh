// image.cuh -- depth ingest, bilateral filter, pyramid and normal maps.
#pragma once
#include "common.cuh"

namespace dyn {

struct LevelMaps {
  const float* depth;  // level depth (metres, 0 invalid)
  float4* normal;      // level normals (0 = invalid)
  float4* vertex;      // optional vertex map (may be null)
  DSensor s;
  int offset;          // first flattened thread index of this level
};
struct MapsArgs {
  LevelMaps lv[kLevels];
  int nlev;
  int total;
};

// Bilateral filter constants: spatial weights per tap offset (row-major
// 2r x 2r, r <= 16) and the range-weight constants.
struct BilateralTable {
  float gs[32 * 32];
  int radius;
  float inv2s2;  // 1 / (2 sigma_i^2)
  float norm;    // 1 / (2 pi sigma_i^2)
};
BilateralTable make_bilateral_table(int radius, float sigma_i, float sigma_s);

// Launchers (all asynchronous on 'st').
void launch_ingest(const uint16_t* raw, const uint8_t* rgb, int n, float scaler,
                   float* depth_out, float* intensity_out, cudaStream_t st);
void launch_bilateral(const float* src, float* dst, int rows, int cols,
                      const BilateralTable& tb, cudaStream_t st);
void launch_downsample_depth(const float* src, int rows, int cols, float* dst,
                             cudaStream_t st);
void launch_downsample_intensity(const float* src, int rows, int cols, float* dst,
                                 cudaStream_t st);
void launch_maps(const MapsArgs& a, cudaStream_t st);
// raycast output -> target level 0: misses (>= dmax) become 0; optional rgb ->
// intensity
void launch_target_prepare(const float* ray_depth, float* depth0, float dmax,
                           const uint8_t* rgb, float* intensity0, int n,
                           cudaStream_t st);
void launch_copy_f(const float* src, float* dst, size_t n, cudaStream_t st);

}  // namespace dyn

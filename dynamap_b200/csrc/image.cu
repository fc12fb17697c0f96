// image.cu -- depth ingest, bilateral filter, 2x pyramid and normal maps.
//
// Reference: include/image/pyramid/pyramid.cu (bilateral :208-252, pyramid
// :49-143), include/image/sensor/rgbdImage.cu (vertex map :23-38, normals
// :126-157), include/solver/gnSolver/gnSolver.cu:457-465 (intensity).
//
// Each stage's arithmetic is one __device__ function, used by a by-value
// kernel (stage entry points) and by a fused kernel that runs the stage for
// every session of a frame in one launch (blockIdx.z = session).
#include "image.cuh"

#include <cmath>
#include <cstring>

#include "dyn_exp.h"
#include "sessdev.cuh"

namespace dyn {

namespace {

// gnSolver::Intensity(ColorToFloat(c)), gnSolver.cu:457-459 + utils.h:98-102:
// channel/255 in float, weighted sum in double, result rounded to float.
__device__ inline float intensity_u8(const uint8_t* c) {
  float r = (float)c[0] / 255.0f, g = (float)c[1] / 255.0f, b = (float)c[2] / 255.0f;
  return (float)(0.2126 * (double)r + 0.7152 * (double)g + 0.0722 * (double)b);
}

// u16 sensor units -> metres (builder.cu:111, utils_Dataset.cpp:233-235)
__device__ inline void ingest_px(const uint16_t* __restrict__ raw, const uint8_t* __restrict__ rgb,
                                 float scaler, float* __restrict__ depth,
                                 float* __restrict__ inten, int i) {
  depth[i] = (float)raw[i] / scaler;
  if (inten) inten[i] = rgb ? intensity_u8(rgb + 3 * (size_t)i) : 0.0f;
}

__global__ void ingest_kernel(const uint16_t* __restrict__ raw,
                              const uint8_t* __restrict__ rgb, int n, float scaler,
                              float* __restrict__ depth, float* __restrict__ inten) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  ingest_px(raw, rgb, scaler, depth, inten, i);
}

constexpr int BTX = 32, BTY = 8;

// pyramid::applyBilateralFilter, pyramid.cu:213-233, one thread per pixel,
// window rows x-r..x+r-1, cols y-r..y+r-1, summed row-major.  The depth tile
// plus halo is staged in shared memory; the spatial weights, a pure function
// of the tap offset, come precomputed on the host in double and rounded to
// float exactly as the reference rounds them per tap (read as warp-uniform
// values).  The range weight uses dyn_expf, the same operation sequence the
// oracle runs, so the filtered depth is bit-identical to the oracle's.  Taps
// outside the image or with depth <= 0 are skipped; invalid centres stay 0.
// FAST (mixed-precision sessions): each tap's weight in one hardware
// base-2 exponential, gs * exp(-dn^2 / (2 s^2)) = 2^(log2 gs - dn^2 c) with
// c = log2(e) / (2 s^2), the spatial weights staged as their logarithms;
// the range normalisation 1/(2 pi s^2), common to every weight, cancels in
// acc / wp and is left out.
template <bool FAST>
__device__ inline void bilateral_tile(const float* __restrict__ src, float* __restrict__ dst,
                                      int rows, int cols, const BilateralTable& tb, int bx,
                                      int by, float* tile) {
  const int D = 2 * tb.radius, half = tb.radius;
  const int TW = BTX + D - 1, TH = BTY + D - 1;
  float* gs = tile + TW * TH;  // the spatial weights, staged once per CTA
  const int tid = threadIdx.y * BTX + threadIdx.x;
  const int row0 = by * BTY - half, col0 = bx * BTX - half;
  for (int k = tid; k < TW * TH; k += BTX * BTY) {
    int tr = k / TW, tc = k - (k / TW) * TW;
    int gr = row0 + tr, gc = col0 + tc;
    tile[k] = (gr >= 0 && gr < rows && gc >= 0 && gc < cols) ? src[gr * cols + gc] : 0.0f;
  }
  for (int k = tid; k < D * D; k += BTX * BTY) gs[k] = FAST ? __log2f(tb.gs[k]) : tb.gs[k];
  __syncthreads();
  const int x = by * BTY + threadIdx.y;  // row (the reference's x)
  const int y = bx * BTX + threadIdx.x;  // column
  if (x >= rows || y >= cols) return;
  const float c = tile[(threadIdx.y + half) * TW + threadIdx.x + half];
  if (!(c > 0.0f)) {
    dst[x * cols + y] = 0.0f;
    return;
  }
  const float inv2s2 = tb.inv2s2, norm = tb.norm;
  const float c2 = inv2s2 * 1.4426950408889634f;  // FAST: log2(e) / (2 s^2)
  float acc = 0.0f, wp = 0.0f;
  // the taps inside the image: row x - half + i in [0, rows), column
  // y - half + j in [0, cols); summed in the reference's order
  const int i0 = max(0, half - x), i1 = min(D, rows - x + half);
  const int j0 = max(0, half - y), j1 = min(D, cols - y + half);
  for (int i = i0; i < i1; ++i) {
    const float* trow = tile + (threadIdx.y + i) * TW + threadIdx.x;
    const float* grow = gs + i * D;
    for (int j = j0; j < j1; ++j) {
      float nv = trow[j];
      if (!(nv > 0.0f)) continue;
      const float dn = nv - c;
      if (FAST) {
        float w;
        asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(w) : "f"(__fmaf_rn(-(dn * dn), c2, grow[j])));
        acc = __fmaf_rn(nv, w, acc);
        wp += w;
      } else {
        float w = range_weight(dn, inv2s2, norm) * grow[j];
        acc += nv * w;
        wp += w;
      }
    }
  }
  dst[x * cols + y] = acc / wp;
}

__global__ void bilateral_kernel(const float* __restrict__ src, float* __restrict__ dst,
                                 int rows, int cols, const __grid_constant__ BilateralTable tb) {
  extern __shared__ float tile[];
  bilateral_tile<false>(src, dst, rows, cols, tb, blockIdx.x, blockIdx.y, tile);
}

// One 2x pyramid step: mean of the valid depths of each 2x2 cell (fix of
// pyramid.cu:49-82, which scatters into a fixed 640x480 window).
__device__ inline void downsample_depth_px(const float* __restrict__ src, int cols, int c2,
                                           float* __restrict__ dst, int i) {
  int y = i / c2, x = i - (i / c2) * c2;
  const float* a = src + (2 * y) * cols + 2 * x;
  float v[4] = {a[0], a[1], a[cols], a[cols + 1]};
  float s = 0.0f;
  int n = 0;
#pragma unroll
  for (int k = 0; k < 4; ++k)
    if (v[k] > 0.0f) {
      s += v[k];
      n++;
    }
  dst[i] = n ? s / (float)n : 0.0f;
}
__device__ inline void downsample_intensity_px(const float* __restrict__ src, int cols, int c2,
                                               float* __restrict__ dst, int i) {
  int y = i / c2, x = i - (i / c2) * c2;
  const float* a = src + (2 * y) * cols + 2 * x;
  dst[i] = (((a[0] + a[1]) + a[cols]) + a[cols + 1]) * 0.25f;
}

__global__ void downsample_depth_kernel(const float* __restrict__ src, int rows, int cols,
                                        float* __restrict__ dst) {
  int c2 = cols / 2, r2 = rows / 2;
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= r2 * c2) return;
  downsample_depth_px(src, cols, c2, dst, i);
}

__global__ void downsample_intensity_kernel(const float* __restrict__ src, int rows, int cols,
                                            float* __restrict__ dst) {
  int c2 = cols / 2, r2 = rows / 2;
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= r2 * c2) return;
  downsample_intensity_px(src, cols, c2, dst, i);
}

// creatPointCloudKernel (rgbdImage.cu:23-38) and vertextoNormal
// (rgbdImage.cu:126-145): n = normalize(cross(V(u+2)-V(u-2), V(v+1)-V(v-1))).
// Vertices are recomputed from depth, so neighbours need no vertex map.  A
// normal is 0 when the centre or a neighbour is invalid or outside the
// row/image.
__device__ inline void maps_px(const float* __restrict__ depth, float4* __restrict__ normal,
                               float4* __restrict__ vertex, const DSensor& s, int i) {
  const int y = i / s.cols, x = i - y * s.cols;
  float d = depth[i];
  float4 nrm = make_float4(0.f, 0.f, 0.f, 0.f);
  if (!(d > 0.0f)) {
    normal[i] = nrm;
    if (vertex) vertex[i] = nrm;
    return;
  }
  F3 p = point3d_uv(x, y, d, s);
  if (vertex) vertex[i] = make_float4(p.x, p.y, p.z, 1.0f);
  if (x - 2 >= 0 && x + 2 < s.cols && y - 1 >= 0 && y + 1 < s.rows) {
    int il = i - 2, ir = i + 2, iu = i - s.cols, id = i + s.cols;
    float dl = depth[il], dr = depth[ir], du = depth[iu], dd = depth[id];
    if (dl > 0.0f && dr > 0.0f && du > 0.0f && dd > 0.0f) {
      F3 left = point3d_uv(x - 2, y, dl, s), right = point3d_uv(x + 2, y, dr, s);
      F3 up = point3d_uv(x, y - 1, du, s), down = point3d_uv(x, y + 1, dd, s);
      F3 c = cross3(right - left, down - up);
      float dd2 = dot3(c, c);
      if (dd2 > 0.0f) {
        F3 n = c * (1.0f / sqrtf(dd2));
        nrm = make_float4(n.x, n.y, n.z, 0.0f);
      }
    }
  }
  normal[i] = nrm;
}

// all pyramid levels of one image in one launch
__global__ void maps_kernel(MapsArgs a) {
  int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= a.total) return;
  int l = 0;
#pragma unroll
  for (int k = 1; k < kLevels; ++k)
    if (k < a.nlev && g >= a.lv[k].offset) l = k;
  const LevelMaps& L = a.lv[l];
  maps_px(L.depth, L.normal, L.vertex, L.s, g - L.offset);
}

__device__ inline void target_prepare_px(const float* __restrict__ ray, float* __restrict__ d0,
                                         float dmax, const uint8_t* __restrict__ rgb,
                                         float* __restrict__ inten, int i) {
  float d = ray[i];
  d0[i] = (d < dmax) ? d : 0.0f;
  if (inten) inten[i] = rgb ? intensity_u8(rgb + 3 * (size_t)i) : 0.0f;
}

__global__ void target_prepare_kernel(const float* __restrict__ ray, float* __restrict__ d0,
                                      float dmax, const uint8_t* __restrict__ rgb,
                                      float* __restrict__ inten, int n) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  target_prepare_px(ray, d0, dmax, rgb, inten, i);
}

// ---------------------------------------------------------------- fused
// ingest (+ the unfiltered copy when the bilateral filter is off), and the
// distance from the camera centre to each pixel's back-projected point
// (IntegrateScanKernel's per-voxel |getPoint3d(pixel, depth)|,
// tsdf.cu:316-317): it depends only on the pixel, so integration reads it
// instead of recomputing it (two divisions and a square root) for every
// voxel that projects there -- the same operations, so the same bits
__global__ void fused_ingest_kernel(const SessDev* __restrict__ tab) {
  const SessDev& S = tab[blockIdx.z];
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= S.npx) return;
  ingest_px(S.u16, *S.rgb_flag ? S.rgb : nullptr, S.depth_scaler, S.raw,
            S.use_color ? S.sint[0] : nullptr, i);
  const float d = S.raw[i];
  if (!S.bil_enabled) S.filt[i] = d;
  const DSensor& s0 = S.ls[0];
  const int y = i / s0.cols;
  S.sdist[i] = norm3(point3d_uv(i - y * s0.cols, y, d, s0));
}

// The free-space tile map of a depth-only frame of a carving session (one
// thread per fine tile; its value also enters its coarse tile's minimum).
__global__ void fused_free_tiles_kernel(const SessDev* __restrict__ tab) {
  const SessDev& S = tab[blockIdx.z];
  if (!S.ftile || S.vol.t.band || *S.rgb_flag) return;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= S.rb_tx * S.rb_ty) return;
  const DSensor& s = S.ls[0];
  const DTsdf& t = S.vol.t;
  const int tx = i % S.rb_tx, ty = i / S.rb_tx;
  const int x0 = tx * kRbTile, y0 = ty * kRbTile;
  const int x1 = min(x0 + kRbTile, s.cols), y1 = min(y0 + kRbTile, s.rows);
  float mn = 3.0e38f;
  bool ok = true;
  for (int y = y0; y < y1; ++y)
    for (int x = x0; x < x1; ++x) {
      const float d = S.raw[y * s.cols + x];
      if (!(d >= t.dmin && d <= t.dmax)) ok = false;
      else mn = fminf(mn, S.sdist[y * s.cols + x] - t.trunc);
    }
  const unsigned v = __float_as_uint(ok ? fmaxf(mn, 0.0f) : 0.0f);
  S.ftile[i] = v;
  const int cx = (S.rb_tx + kRbCoarse - 1) / kRbCoarse;
  atomicMin(S.ftile + S.rb_tx * S.rb_ty + (ty / kRbCoarse) * cx + tx / kRbCoarse, v);
}

__global__ void fused_bilateral_kernel(const SessDev* __restrict__ tab) {
  extern __shared__ float tile[];
  const SessDev& S = tab[blockIdx.z];
  if (!S.bil_enabled) return;
  const int rows = S.ls[0].rows, cols = S.ls[0].cols;
  if ((int)blockIdx.x * BTX >= cols || (int)blockIdx.y * BTY >= rows) return;
  if (S.vol.fp16)  // mixed-precision session
    bilateral_tile<true>(S.raw, S.filt, rows, cols, *S.btab, blockIdx.x, blockIdx.y, tile);
  else
    bilateral_tile<false>(S.raw, S.filt, rows, cols, *S.btab, blockIdx.x, blockIdx.y, tile);
}

// level l of the source (target == 0) or target pyramid from level l-1
__global__ void fused_downsample_kernel(const SessDev* __restrict__ tab, int l, int target) {
  const SessDev& S = tab[blockIdx.z];
  if (l >= S.nlev) return;
  const DSensor& sp = S.ls[l - 1];
  const int c2 = sp.cols / 2, n = (sp.rows / 2) * c2;
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  downsample_depth_px(target ? S.tdep[l - 1] : S.sdep[l - 1], sp.cols, c2,
                      target ? S.tdep[l] : S.sdep[l], i);
  if (S.use_color)
    downsample_intensity_px(target ? S.tint[l - 1] : S.sint[l - 1], sp.cols, c2,
                            target ? S.tint[l] : S.sint[l], i);
}

__global__ void fused_maps_kernel(const SessDev* __restrict__ tab, int target) {
  const SessDev& S = tab[blockIdx.z];
  int g = blockIdx.x * blockDim.x + threadIdx.x;
  for (int l = 0; l < S.nlev; ++l) {
    const int n = S.ls[l].rows * S.ls[l].cols;
    if (g < n) {
      float4* vtx = S.debug_maps ? (target ? S.tvtx[l] : S.svtx[l]) : nullptr;
      maps_px(target ? S.tdep[l] : S.sdep[l], target ? S.tnrm[l] : S.snrm[l], vtx, S.ls[l], g);
      return;
    }
    g -= n;
  }
}

// next frame's target level 0: the raycast (mode 1, misses -> 0) or the
// source itself (mode 0); flags the target as present
__global__ void fused_target_prepare_kernel(const SessDev* __restrict__ tab) {
  const SessDev& S = tab[blockIdx.z];
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i == 0) S.icp->have_target = 1;
  if (i >= S.npx) return;
  if (S.mode == 1) {
    target_prepare_px(S.ray, S.tdep[0], S.vol.t.dmax, S.use_color ? S.trgb : nullptr,
                      S.use_color ? S.tint[0] : nullptr, i);
  } else {
    S.tdep[0][i] = S.sdep[0][i];
    if (S.use_color) S.tint[0][i] = S.sint[0][i];
  }
}

inline int nblk(long long n, int t) { return (int)((n + t - 1) / t); }

}  // namespace

void launch_ingest(const uint16_t* raw, const uint8_t* rgb, int n, float scaler,
                   float* depth_out, float* intensity_out, cudaStream_t st) {
  ingest_kernel<<<nblk(n, 256), 256, 0, st>>>(raw, rgb, n, scaler, depth_out, intensity_out);
}

// pyramid::gaussian, pyramid.cu:208-211, in double.
static double gaussian_d(double x, double sigma) {
  return std::exp(-(std::pow(x, 2)) / (2 * std::pow(sigma, 2))) /
         (2 * 3.14159265358979323846 * std::pow(sigma, 2));
}

BilateralTable make_bilateral_table(int radius, float sigma_i, float sigma_s) {
  BilateralTable tb;
  std::memset(&tb, 0, sizeof(tb));
  tb.radius = radius;
  const int D = 2 * radius, half = radius;
  for (int i = 0; i < D; ++i)
    for (int j = 0; j < D; ++j) {
      // vertexDistance (pyramid.cu:201-206) in float, gaussian in double
      float dx = (float)(half - i), dy = (float)(half - j);
      float dd = std::sqrt(dx * dx + dy * dy + 0.0f * 0.0f);
      tb.gs[i * D + j] = (float)gaussian_d((double)dd, (double)sigma_s);
    }
  double si = (double)sigma_i;
  tb.inv2s2 = (float)(1.0 / (2.0 * si * si));
  tb.norm = (float)(1.0 / (2.0 * 3.14159265358979323846 * si * si));
  return tb;
}

// depth tile with its halo, then the D x D spatial weights
static size_t bilateral_smem(int radius) {
  int D = 2 * radius;
  return sizeof(float) * ((size_t)(BTX + D - 1) * (BTY + D - 1) + (size_t)D * D);
}

void launch_bilateral(const float* src, float* dst, int rows, int cols, const BilateralTable& tb,
                      cudaStream_t st) {
  dim3 grid(nblk(cols, BTX), nblk(rows, BTY));
  bilateral_kernel<<<grid, dim3(BTX, BTY), bilateral_smem(tb.radius), st>>>(src, dst, rows, cols,
                                                                            tb);
}

void launch_downsample_depth(const float* src, int rows, int cols, float* dst, cudaStream_t st) {
  int n = (rows / 2) * (cols / 2);
  if (n > 0) downsample_depth_kernel<<<nblk(n, 256), 256, 0, st>>>(src, rows, cols, dst);
}
void launch_downsample_intensity(const float* src, int rows, int cols, float* dst,
                                 cudaStream_t st) {
  int n = (rows / 2) * (cols / 2);
  if (n > 0) downsample_intensity_kernel<<<nblk(n, 256), 256, 0, st>>>(src, rows, cols, dst);
}
void launch_maps(const MapsArgs& a, cudaStream_t st) {
  if (a.total > 0) maps_kernel<<<nblk(a.total, 256), 256, 0, st>>>(a);
}
void launch_target_prepare(const float* ray_depth, float* depth0, float dmax, const uint8_t* rgb,
                           float* intensity0, int n, cudaStream_t st) {
  target_prepare_kernel<<<nblk(n, 256), 256, 0, st>>>(ray_depth, depth0, dmax, rgb, intensity0,
                                                      n);
}
void launch_copy_f(const float* src, float* dst, size_t n, cudaStream_t st) {
  if (n) cudaMemcpyAsync(dst, src, n * sizeof(float), cudaMemcpyDeviceToDevice, st);
}

// ---- fused stages
void fused_ingest(const SessDev* tab, const BatchShape& b, cudaStream_t st) {
  fused_ingest_kernel<<<dim3(nblk(b.max_npx, 256), 1, b.n), 256, 0, st>>>(tab);
  fused_free_tiles_kernel<<<dim3(nblk(b.max_rb_tiles, 128), 1, b.n), 128, 0, st>>>(tab);
}

void fused_bilateral(const SessDev* tab, const BatchShape& b, cudaStream_t st) {
  if (b.max_bil_radius > 0)
    fused_bilateral_kernel<<<dim3(nblk(b.max_cols, BTX), nblk(b.max_rows, BTY), b.n),
                             dim3(BTX, BTY), bilateral_smem(b.max_bil_radius), st>>>(tab);
}

void fused_pyramid(const SessDev* tab, const BatchShape& b, int target, cudaStream_t st) {
  for (int l = 1; l < b.max_nlev; ++l)
    if (b.max_level_px[l] > 0)
      fused_downsample_kernel<<<dim3(nblk(b.max_level_px[l], 256), 1, b.n), 256, 0, st>>>(
          tab, l, target);
  int tot = 0;
  for (int l = 0; l < b.max_nlev; ++l) tot += b.max_level_px[l];
  fused_maps_kernel<<<dim3(nblk(tot, 256), 1, b.n), 256, 0, st>>>(tab, target);
}

void fused_target_prepare(const SessDev* tab, const BatchShape& b, cudaStream_t st) {
  fused_target_prepare_kernel<<<dim3(nblk(b.max_npx, 256), 1, b.n), 256, 0, st>>>(tab);
}

}  // namespace dyn

// sessdev.cuh -- the per-session device descriptor used by the fused
// per-frame kernels.
//
// Every session owns one SessDev in device memory (written once at creation:
// its buffers, sensor levels and parameters).  A frame of N sessions runs
// each stage as ONE launch whose blockIdx.z selects the session from a table
// of descriptors; a single session is a table of one.  Inside its z-slice a
// session partitions its work exactly as it would alone (CTAs beyond its own
// grid return at once), so its results do not depend on the other sessions.
#pragma once
#include "common.cuh"
#include "icp.cuh"
#include "image.cuh"
#include "tsdf.cuh"

namespace dyn {

// Ray depth bounds of the frame raycast: 8x8-pixel fine tiles, and coarse
// tiles of kRbCoarse x kRbCoarse fine ones; near and far bound per tile.
constexpr int kRbTile = 8;
constexpr int kRbCoarse = 8;
inline __host__ __device__ int ray_bounds_words(int tiles_x, int tiles_y) {
  const int cx = (tiles_x + kRbCoarse - 1) / kRbCoarse, cy = (tiles_y + kRbCoarse - 1) / kRbCoarse;
  return 2 * tiles_x * tiles_y + 2 * cx * cy;
}

// The visible list's session index carries this bit for free-space blocks
// (every voxel takes the free-space update; see fused_visible_kernel).
constexpr int kVisFree = 1 << 30;
// Free-space tile map of a depth-only frame: per fine 8x8-pixel tile, then
// per coarse tile, the least (sdist - truncation) over its pixels as float
// bits, 0 where a pixel's depth is outside the sensor range (negative
// values count as 0).
inline __host__ __device__ int free_tile_words(int tiles_x, int tiles_y) {
  return ray_bounds_words(tiles_x, tiles_y) / 2;
}

struct SessDev {
  DSensor ls[kLevels];  // level sensors (scale 1, 2, 4, 8)
  int nlev;             // levels in use
  int npx;              // level-0 pixels
  float depth_scaler;
  const int* rgb_flag;  // nonzero: the current frame carries RGB (device, set per frame)
  int use_color;        // photometric term on (intensity / colour images kept)
  int bil_enabled;
  int mode;             // 0 frame-to-frame, 1 frame-to-model
  int debug_maps;       // also write vertex maps
  // frame input (device copies)
  const uint16_t* u16;
  const uint8_t* rgb;
  // images
  float* raw;
  float* sdist;         // |point3d_uv(x, y, raw)| per pixel (integration)
  float* filt;
  float* sdep[kLevels];
  float4* snrm[kLevels];
  float4* svtx[kLevels];
  float* sint[kLevels];
  float* tdep[kLevels];
  float4* tnrm[kLevels];
  float4* tvtx[kLevels];
  float* tint[kLevels];
  float* ray;
  uint8_t* trgb;
  unsigned* ftile;      // free-space tile map, free_tile_words(rb_tx, rb_ty) words
  unsigned* rbound;     // ray depth bounds (float bits), ray_bounds_words(rb_tx,
  int rb_tx, rb_ty;     // rb_ty) words; rb_tx x rb_ty fine tiles
  const BilateralTable* btab;  // device copy
  // solver
  IcpState* icp;
  PoseState* pose;
  double* partials;
  IcpParams icpp;
  int slot_level[3];  // pyramid level of each ICP level slot
  int slot_iters[3];  // lvl_iteration_num of each slot (runs N-1 iterations)
  // map
  VolumeDev vol;
};

// Launch helpers of the fused stages (image.cu, icp.cu, tsdf.cu).  'tab' is
// a device array of n descriptors; the grid of each launch is sized for the
// largest session of the table (BatchShape).
struct BatchShape {
  int n;
  int max_rows, max_cols;  // largest level-0 image
  int max_npx;
  int max_nlev;
  int max_blocks;          // largest num_blocks
  int max_level_px[kLevels];
  int max_slot_px[3];      // largest pixel count of each ICP level slot
  int max_slot_iters[3];   // largest lvl_iteration_num of each slot
  int max_bil_radius;      // 0: no session filters
  int max_rb_tiles;        // largest ray-start bound (tiles; at least 1)
  int kahan_mask;          // bit 0: some session sums plainly, bit 1: some use Kahan sums
  int fp16_mask;           // bit 0: some session keeps FP32 voxels, bit 1: some mixed
  // launch shapes that leave every result unchanged (chosen by a batch's
  // autotuner): CTAs of the integration grid (0: 148 x 8) and the raycast
  // tile (0: 16x16, 1: 32x8, 2: 8x8 pixels)
  int integrate_ctas;
  int ray_tile;
  int2* gvis;              // batch-wide visible list (session, heap index)
  int* gcount;             // its length (device)
  int gvis_cap;
  // the persistent ICP: blocks of its cooperative launches (0: the chained
  // kernels instead) in all and per summation kind (plain, compensated),
  // the budget each launch's shares are taken from, and the barrier's
  // counters, flags and abort word (kIcpBarWords, device)
  int icp_grid;
  int icp_grid_k[2];
  int icp_budget;
  unsigned* icp_bar;
};

// image.cu
void fused_ingest(const SessDev* tab, const BatchShape& b, cudaStream_t st);
void fused_bilateral(const SessDev* tab, const BatchShape& b, cudaStream_t st);
void fused_pyramid(const SessDev* tab, const BatchShape& b, int target, cudaStream_t st);
void fused_target_prepare(const SessDev* tab, const BatchShape& b, cudaStream_t st);
// icp.cu
void fused_icp_iteration(const SessDev* tab, const BatchShape& b, int slot, int it, bool chained,
                         cudaStream_t st);
void fused_pose_finalize(const SessDev* tab, const BatchShape& b, int bump, cudaStream_t st);
void fused_icp_persistent(const SessDev* tab, const BatchShape& b, cudaStream_t st);
// tsdf.cu
void fused_reset_counters(const SessDev* tab, const BatchShape& b, cudaStream_t st);
void fused_allocate(const SessDev* tab, const BatchShape& b, cudaStream_t st);
void fused_visible(const SessDev* tab, const BatchShape& b, cudaStream_t st);
void fused_integrate(const SessDev* tab, const BatchShape& b, cudaStream_t st);
void fused_free_cells(const SessDev* tab, const BatchShape& b, cudaStream_t st);
void fused_raycast(const SessDev* tab, const BatchShape& b, cudaStream_t st);

}  // namespace dyn

// icp.cuh -- projective point-to-plane (+photometric) ICP normal equations
// and the on-device Gauss-Newton step.
#pragma once
#include "common.cuh"

namespace dyn {

// Per-session solver state, device resident.
struct IcpState {
  double inc[6];      // xi accumulated over the frame's levels (gnSolver.cu:345)
  double prev[6];     // prev_increment (gnSolver.cu:347,415)
  float T[16];        // float exp(v2t(inc)) used by the next reduction
  int converged;      // current level stopped (|delta| <= minIncrement)
  int have_target;    // 0 until a target exists (first frame: no tracking)
  unsigned int ticket;  // last-block-done counter
  int iters[3];
  int inliers[3];
  float rms[3];
};

// Pose of the session, device resident.
struct PoseState {
  double pose[16];    // camera-to-world (row-major, double)
  float posef[16];    // float copy used by the kernels
  float invf[16];     // float4x4::getInverse of posef (utils_matrix.h:970-1086)
  double last_inc[6];
  int reset;          // NaN / maxIncrement guard fired this frame
  int frame;
};

struct IcpLevel {
  const float* sd;     // source depth
  const float4* sn;    // source normals
  const float* si;     // source intensity (may be null if cw == 0)
  const float* td;     // target depth
  const float4* tn;    // target normals
  const float* ti;     // target intensity (may be null if cw == 0)
  DSensor s;
};

struct IcpParams {
  float dmin, dmax;    // icp depth window
  float cos_thr;
  float cw;            // color weight
  float min_inc, max_inc, reg;
  int compose_left;
  int kahan;           // compensated FP32 per-thread sums (mixed precision)
};

constexpr int kIcpThreads = 256;
constexpr int kIcpMaxBlocks = 148 * 8;
constexpr int kIcpVals = 29;
// The per-frame ICP sums its normal equations per pixel tile: tile j holds
// pixels [j * t, (j + 1) * t) of a level of n pixels, t = icp_tile_px(n)
// (256, 512 or 1024 pixels: one, two or four per thread, smaller tiles on
// the coarse levels so that more blocks share their short work), and its
// partial sums are the same whichever block computes them; the level's
// total adds the tiles in index order.  So the result does not depend on
// how many blocks work on a level, nor on the sessions that share the
// launch.  A level never has more tiles than the session's finest one.
inline __host__ __device__ int icp_tile_px(int npx) {
  return npx <= 8192 ? kIcpThreads : (npx <= 65536 ? 2 * kIcpThreads : 4 * kIcpThreads);
}
inline __host__ __device__ int icp_tiles(int npx) {
  const int t = icp_tile_px(npx);
  return (npx + t - 1) / t;
}

// Scratch a reduction needs: per-block partial sums (kIcpMaxBlocks*29 doubles).
size_t icp_scratch_bytes();
// Scratch of the per-frame ICP of a session whose largest level has npx
// pixels: two rows of per-tile partial sums (iterations alternate rows) and
// at least icp_scratch_bytes().
size_t icp_frame_scratch_bytes(size_t npx);

// The persistent ICP (one cooperative launch per frame and summation kind):
// the blocks that can be resident at once on 'device' (0: cooperative
// launches unavailable), and the grids of a table whose sessions' largest
// levels have npx[j] pixels and sum plainly (kahan[j] == 0) or with
// compensation: grid_k[kind] blocks within 'budget' each (0: no session of
// that kind).  Returns their total, or 0 when a kind does not fit (the
// chained kernels run the table, with the same results).
int icp_persistent_capacity(int device);
int icp_persistent_grid(const int* npx, const int* kahan, int n, int budget, int* grid_k);
// The persistent ICP's grid barrier words (a launch's arrival counters,
// release flags and abort word, each on its own 128-byte line): a launch's
// barrier buffer holds kIcpBarWords unsigned words.
constexpr int kIcpBarSpread = 8;
constexpr int kIcpBarWords = (2 * kIcpBarSpread + 1) * 32;
// A bounded grid barrier run alone: 'blocks' blocks wait for blocks +
// missing arrivals (bar_dev: kIcpBarWords words).  DYN_OK when it completes,
// DYN_ERR_TIMEOUT when the bounded wait ran out, DYN_ERR_INVALID_ARG when
// the blocks cannot all be resident.
dyn_status icp_barrier_selftest(int blocks, int missing, unsigned* bar_dev, cudaStream_t st);
// After the last level: guards, pose composition, float pose + inverse, reset
// of the solver state.  Runs with one thread.
void launch_pose_finalize(const IcpParams& P, IcpState* st, PoseState* ps,
                          cudaStream_t stream);
// Tracking of the next frame starts from the motion from the current pose
// to 'hint' (double[16], camera-to-world): the solver's increment becomes
// its SE(3) logarithm (before the first target, the hint becomes the pose).
void launch_pose_hint(PoseState* ps, IcpState* st, const double* hint_dev, int compose_left,
                      cudaStream_t stream);
// Set the pose from the host (double[16]); recomputes posef/invf.
void launch_pose_set(PoseState* ps, const double* pose_dev, cudaStream_t stream);
// Normal equations only (no solve): out[29] doubles on the device.
void launch_icp_reduce_only(const IcpLevel& L, const IcpParams& P, const float* T_dev,
                            double* partials, unsigned int* ticket, double* out_dev,
                            cudaStream_t stream);
// The same reduction on an explicit grid ('partials' holds grid * 29
// doubles; pixels beyond grid * kIcpThreads are covered by the grid-stride
// loop).
void launch_icp_reduce_grid(const IcpLevel& L, const IcpParams& P, const float* T_dev,
                            double* partials, unsigned int* ticket, double* out_dev, int grid,
                            cudaStream_t stream);

}  // namespace dyn

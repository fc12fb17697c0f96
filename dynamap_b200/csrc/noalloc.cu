// noalloc.cu -- dyn_icp_normal_equations_noalloc: the ICP normal-equation
// reduction for callers that cannot allocate device memory.
//
// Some callers cannot call cudaMalloc: a host process that reserves a fixed
// device-memory budget up front and forbids later allocations (a real-time
// robotics executor running the tracker inside its control loop, a plugin
// host that owns all GPU memory), or code that must not risk the implicit
// device synchronisation and failure modes of an allocation in the middle of
// a frame.  dyn_icp_normal_equations allocates its scratch (per-block partial
// sums, a completion counter, the transform and the result) on first use;
// this variant keeps all of that in one file-scope __device__ array of fixed
// size instead, so it calls no cudaMalloc, cudaFree or allocating library
// routine.  The caller still passes the input images and receives the sums.
//
// Limits: the array holds kNoAllocSlots per-block partial sums; one block of
// 256 threads covers up to 4 pixels per thread, so a level may have at most
// kNoAllocSlots * 256 * 4 = 2,097,152 pixels (1920x1080 fits); larger levels
// are rejected with DYN_ERR_INVALID_ARG.  The array (about 465 KiB) lives on
// every GPU that loads the library until the process exits.
//
// Every call on a device shares the array and it keeps the last call's
// contents: the completion counter is cleared at the start of each call.
// Calls whose GPU work overlaps (two host threads, or two streams, on the
// same device at once) race on the array and must be serialised by the
// caller.  The first call on a device looks up the array's device address
// (cudaGetSymbolAddress) with that device current; make that first call
// before any stream capture on the device.  The address is kept for the
// life of the process, so the library must not be used across a
// cudaDeviceReset of that device (the allocating entry point keeps its
// buffers the same way).
//
// Inputs are checked exactly as dyn_icp_normal_equations checks them
// (valid_sensor: sides 1..8192, positive focal lengths and depth scaler),
// so both entry points accept and reject the same levels.
#include <cuda_runtime.h>

#include <mutex>

#include "icp.cuh"
#include "session_impl.cuh"

using namespace dyn;

namespace {

constexpr int kNoAllocSlots = 2048;
constexpr int kNoAllocPixPerThread = 4;
constexpr long long kNoAllocMaxPixels =
    (long long)kNoAllocSlots * kIcpThreads * kNoAllocPixPerThread;

// byte offsets inside the array (each piece 256-byte aligned)
constexpr size_t kOffPartials = 0;
constexpr size_t kPartialBytes = sizeof(double) * (size_t)kNoAllocSlots * kIcpVals;
constexpr size_t kOffOut = kPartialBytes;
constexpr size_t kOffT = kOffOut + 256;
constexpr size_t kOffTicket = kOffT + 256;
constexpr size_t kScratchBytes = kOffTicket + 256;

static __device__ __align__(256) unsigned char g_icp_noalloc_scratch[kScratchBytes];

std::mutex g_setup_mu;
void* g_scratch_addr[64] = {};

// Device address of the array on the current device (set-up on first use).
dyn_status scratch_base(int dev, unsigned char** out) {
  if (dev < 0 || dev >= 64) return DYN_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> lk(g_setup_mu);
  if (!g_scratch_addr[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_icp_noalloc_scratch);
    if (e != cudaSuccess || p == nullptr) {
      cudaGetLastError();
      return DYN_ERR_CUDA;
    }
    g_scratch_addr[dev] = p;
  }
  *out = static_cast<unsigned char*>(g_scratch_addr[dev]);
  return DYN_OK;
}

}  // namespace

extern "C" dyn_status dyn_icp_normal_equations_noalloc(
    const float* src_depth_dev, const float* src_normal4_dev, const float* src_intensity_dev,
    const float* tgt_depth_dev, const float* tgt_normal4_dev, const float* tgt_intensity_dev,
    const dyn_sensor* level, const dyn_gn_params* gn, const float T[16], double out_host[29],
    void* stream) {
  if (!src_depth_dev || !src_normal4_dev || !tgt_depth_dev || !tgt_normal4_dev ||
      !dyn::host::valid_sensor(level) || !gn || !T || !out_host)
    return DYN_ERR_INVALID_ARG;
  if (gn->color_weight != 0.0f && (!src_intensity_dev || !tgt_intensity_dev))
    return DYN_ERR_INVALID_ARG;
  const long long n = (long long)level->rows * level->cols;
  if (n > kNoAllocMaxPixels) return DYN_ERR_INVALID_ARG;  // beyond the array's capacity
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return DYN_ERR_NO_DEVICE;
  unsigned char* base = nullptr;
  dyn_status r = scratch_base(dev, &base);
  if (r != DYN_OK) return r;
  double* partials = reinterpret_cast<double*>(base + kOffPartials);
  double* out_dev = reinterpret_cast<double*>(base + kOffOut);
  float* T_dev = reinterpret_cast<float*>(base + kOffT);
  unsigned int* ticket = reinterpret_cast<unsigned int*>(base + kOffTicket);
  cudaStream_t st = (cudaStream_t)stream;

  IcpLevel L;
  L.sd = src_depth_dev;
  L.sn = reinterpret_cast<const float4*>(src_normal4_dev);
  L.si = src_intensity_dev;
  L.td = tgt_depth_dev;
  L.tn = reinterpret_cast<const float4*>(tgt_normal4_dev);
  L.ti = tgt_intensity_dev;
  L.s.rows = (int)level->rows;
  L.s.cols = (int)level->cols;
  L.s.fx = level->fx;
  L.s.fy = level->fy;
  L.s.cx = level->cx;
  L.s.cy = level->cy;
  IcpParams P;
  P.dmin = gn->icp_min_depth;
  P.dmax = gn->icp_max_depth;
  P.cos_thr = gn->normal_cos_thresh;
  P.cw = gn->color_weight;
  P.min_inc = gn->min_increment;
  P.max_inc = gn->max_increment;
  P.reg = gn->regularization;
  P.compose_left = gn->compose_left;
  P.kahan = 0;
  const long long per_block = (long long)kIcpThreads * kNoAllocPixPerThread;
  const int grid = (int)((n + per_block - 1) / per_block);

  // the counter must start at zero; the array keeps the previous call's data
  if (cudaMemsetAsync(ticket, 0, sizeof(unsigned int), st) != cudaSuccess ||
      cudaMemcpyAsync(T_dev, T, 16 * sizeof(float), cudaMemcpyHostToDevice, st) != cudaSuccess)
    return DYN_ERR_CUDA;
  launch_icp_reduce_grid(L, P, T_dev, partials, ticket, out_dev, grid, st);
  if (cudaGetLastError() != cudaSuccess) return DYN_ERR_CUDA;
  if (cudaMemcpyAsync(out_host, out_dev, sizeof(double) * kIcpVals, cudaMemcpyDeviceToHost,
                      st) != cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess)
    return DYN_ERR_CUDA;
  return DYN_OK;
}

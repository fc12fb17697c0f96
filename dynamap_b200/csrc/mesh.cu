// mesh.cu -- triangle mesh of a session's TSDF over a box
// (tsdfVolume::ExtractMesh, tsdf.cu:551-560; MeshExtractor::ExtractMesh,
// meshExtractor.cu:364-407), the reference's dense cell walk driven by the
// allocated blocks instead.
//
// Which cells mesh: a cell yields triangles only when all 64 voxels its
// eight corner samples read are observed, so the block of its key voxel
// (mesh_cell.h: key_index) is allocated.  key_index is monotone per axis,
// so the cells keyed to one block form a box of about 8x8x8, found by
// binary search.  One CTA takes one allocated block at a time:
//   1. the block ranges per axis and the heap indices of the 2x2x2 blocks
//      a cell of it can read (its samples lie 0..3 voxels above the key);
//   2. the 11x11x11 voxels from the block's origin staged in shared memory
//      (10.6 KB; FP32 and mixed voxels both as the 8-byte form);
//   3. per cell the corner samples from that tile (the global volume for a
//      sample outside it), the cube index and the triangles.
// Two passes make the output deterministic: the first counts triangles per
// block, a scan gives each block its offset, the second writes them --
// block by block in heap order, cells in x-fastest order inside a block,
// triangles in table order.  Pass 2 repeats pass 1's arithmetic on the
// same voxels, so its counts are the same.
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <mutex>

#include "mesh_kernels.cuh"
#include "session_impl.cuh"


using namespace dyn::host;

namespace {

// The marching-cubes triangle table (d_mc_tri) is written once per device,
// synchronously, before the first mesh kernel on that device runs; later
// calls (from any session's stream) only read it.
std::mutex g_mc_mu;
bool g_mc_ready[64] = {};

dyn_status mc_table_ready(int dev) {
  if (dev < 0 || dev >= 64) return DYN_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> lk(g_mc_mu);
  if (!g_mc_ready[dev]) {
    DYN_CUDA(cudaMemcpyToSymbol(dyn::d_mc_tri, dyn::kMcTriangles, sizeof(dyn::kMcTriangles)));
    g_mc_ready[dev] = true;
  }
  return DYN_OK;
}

}  // namespace

dyn_status dyn_extract_mesh(dyn_session* s, const float lower[3], const float upper[3],
                            float* triangles_host, int64_t capacity, int64_t* n_out) {
  if (!s || !lower || !upper || !n_out || capacity < 0) return DYN_ERR_INVALID_ARG;
  dyn::mesh::Grid g;
  if (!dyn::mesh::make_grid(lower, upper, s->tp.voxel_size, &g)) return DYN_ERR_INVALID_ARG;
  *n_out = 0;
  int64_t nb = 0;
  DYN_TRY(dyn_num_blocks(s, &nb));  // waits for the session's frames
  if (nb == 0 || g.n[0] == 0 || g.n[1] == 0 || g.n[2] == 0) return DYN_OK;
  DeviceGuard dg(s->device);
  cudaStream_t st = s->stream;
  DYN_TRY(mc_table_ready(s->device));
  const int n = (int)nb;
  long long* counts = nullptr;
  long long* offsets = nullptr;  // n offsets, then the total
  float* tri = nullptr;
  dyn_status r = DYN_OK;
  long long total = 0;
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, s->device);
  const int grid = std::min(n, sms * 8);
  do {
    if (cudaMallocAsync(&counts, sizeof(long long) * (size_t)n, st) != cudaSuccess ||
        cudaMallocAsync(&offsets, sizeof(long long) * ((size_t)n + 1), st) != cudaSuccess) {
      r = DYN_ERR_OOM;
      break;
    }
    dyn::mesh_blocks_kernel<false><<<grid, dyn::kMeshThreads, 0, st>>>(s->vol, g, n, counts,
                                                                          nullptr, nullptr, 0);
    dyn::mesh_scan_kernel<<<1, 1024, 0, st>>>(counts, n, offsets, offsets + n);
    if (cudaMemcpyAsync(&total, offsets + n, sizeof(long long), cudaMemcpyDeviceToHost, st) !=
            cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess) {
      r = DYN_ERR_CUDA;
      break;
    }
    *n_out = total;
    const long long m = std::min<long long>(total, capacity);
    if (!triangles_host || m == 0) break;
    const size_t bytes = sizeof(float) * dyn::kTriFloats * (size_t)m;
    if (cudaMallocAsync(&tri, bytes, st) != cudaSuccess) {
      r = DYN_ERR_OOM;
      break;
    }
    dyn::mesh_blocks_kernel<true><<<grid, dyn::kMeshThreads, 0, st>>>(s->vol, g, n, counts,
                                                                         offsets, tri, m);
    if (cudaMemcpyAsync(triangles_host, tri, bytes, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
      r = DYN_ERR_CUDA;
  } while (false);
  if (r != DYN_OK) cudaGetLastError();
  if (tri) cudaFreeAsync(tri, st);
  if (offsets) cudaFreeAsync(offsets, st);
  if (counts) cudaFreeAsync(counts, st);
  if (cudaStreamSynchronize(st) != cudaSuccess && r == DYN_OK) r = DYN_ERR_CUDA;
  return r;
}

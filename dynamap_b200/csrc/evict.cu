// evict.cu -- block eviction and streaming for a session's volume
// (HashTable::DeleteBlock, hashTable.cu:112-134, which the reference never
// calls; here the way a session stays inside an HBM budget).
//
// dyn_evict_blocks removes the blocks the allocation has not touched for a
// number of frames, dyn_delete_blocks those at given coordinates; both can
// hand the removed blocks to the host first, and dyn_upload_blocks puts
// blocks (from the host) back.  Removal compacts the heap (evict_ops.h):
//   mark      keep flag per allocated block (by entry stamp, or by lookup)
//   scan      survivors before each block -> L survivors, dead blocks listed
//   gather    (optional) the dead blocks' coordinates and voxels
//   move      survivors at L and above into the holes below L
//   rewrite   every bucket front-packed with the new heap indices
//   clear     heap [L, n) zeroed, heap top = L
// All on the session's stream between frames; nothing here runs inside
// the per-frame graph, and the per-frame allocation is unchanged (its bump
// pointer resumes at L).
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <algorithm>

#include "evict_kernels.cuh"
#include "session_impl.cuh"

namespace dyn {
namespace {

int grid_for(long long n, int threads) {
  const long long g = (n + threads - 1) / threads;
  return (int)std::max<long long>(1, std::min<long long>(g, 148LL * 16));
}

}  // namespace
}  // namespace dyn

using namespace dyn::host;

namespace {

// The removal shared by dyn_evict_blocks and dyn_delete_blocks: 'mark'
// fills keep[0..n) on the stream; the rest as the file header says.
template <class Mark>
dyn_status remove_blocks(dyn_session* s, Mark mark, int32_t* coords_out, dyn_voxel* voxels_out,
                         int64_t capacity, int64_t* n_out) {
  if (!s || !n_out || capacity < 0) return DYN_ERR_INVALID_ARG;
  *n_out = 0;
  int64_t nb = 0;
  DYN_TRY(dyn_num_blocks(s, &nb));  // waits for the session's frames
  if (nb == 0) return DYN_OK;
  DeviceGuard dg(s->device);
  cudaStream_t st = s->stream;
  const int n = (int)nb;
  int *keep = nullptr, *pos = nullptr, *dead_at = nullptr, *dest = nullptr, *gcoords = nullptr;
  dyn_voxel* gvox = nullptr;
  dyn_status r = DYN_OK;
  do {
    if (cudaMallocAsync(&keep, sizeof(int) * (size_t)n, st) != cudaSuccess ||
        cudaMallocAsync(&pos, sizeof(int) * ((size_t)n + 1), st) != cudaSuccess ||
        cudaMallocAsync(&dead_at, sizeof(int) * (size_t)n, st) != cudaSuccess ||
        cudaMallocAsync(&dest, sizeof(int) * (size_t)n, st) != cudaSuccess) {
      r = DYN_ERR_OOM;
      break;
    }
    r = mark(st, n, keep);
    if (r != DYN_OK) break;
    dyn::scan_flags_kernel<<<1, 1024, 0, st>>>(keep, n, pos);
    int L = 0;
    if (cudaMemcpyAsync(&L, pos + n, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess) {
      r = DYN_ERR_CUDA;
      break;
    }
    const int dead = n - L;
    *n_out = dead;
    if (dead == 0) break;
    dyn::dead_list_kernel<<<dyn::grid_for(n, dyn::kEvT), dyn::kEvT, 0, st>>>(keep, pos, n, dead_at);
    const int m = (int)std::min<int64_t>(dead, capacity);
    if (m > 0 && (coords_out || voxels_out)) {
      if (cudaMallocAsync(&gcoords, sizeof(int) * 3 * (size_t)m, st) != cudaSuccess ||
          cudaMallocAsync(&gvox, sizeof(dyn_voxel) * dyn::kBlockVox * (size_t)m, st) !=
              cudaSuccess) {
        r = DYN_ERR_OOM;
        break;
      }
      dyn::gather_kernel<<<std::min(m, 148 * 8), dyn::kEvT, 0, st>>>(s->vol, dead_at, m, gcoords,
                                                                     gvox);
      if ((coords_out && cudaMemcpyAsync(coords_out, gcoords, sizeof(int) * 3 * (size_t)m,
                                         cudaMemcpyDeviceToHost, st) != cudaSuccess) ||
          (voxels_out &&
           cudaMemcpyAsync(voxels_out, gvox, sizeof(dyn_voxel) * dyn::kBlockVox * (size_t)m,
                           cudaMemcpyDeviceToHost, st) != cudaSuccess)) {
        r = DYN_ERR_CUDA;
        break;
      }
    }
    dyn::dest_kernel<<<dyn::grid_for(n, dyn::kEvT), dyn::kEvT, 0, st>>>(keep, pos, n, L, dead_at,
                                                                      dest);
    if (n > L)
      dyn::move_kernel<<<std::min(n - L, 148 * 8), dyn::kEvT, 0, st>>>(s->vol, n, L, dest);
    const int nbk = s->tp.num_buckets;
    dyn::rewrite_kernel<<<dyn::grid_for(nbk, dyn::kEvT), dyn::kEvT, 0, st>>>(
        s->vol.entries, nbk, s->tp.bucket_size, n, keep, dest);
    const size_t tail = (size_t)(n - L) * dyn::kBlockVox, from = (size_t)L * dyn::kBlockVox;
    cudaError_t e = cudaSuccess;
    if (s->vol.voxels)
      e = cudaMemsetAsync(s->vol.voxels + from, 0, sizeof(dyn_voxel) * tail, st);
    if (e == cudaSuccess && s->vol.vox16)
      e = cudaMemsetAsync(s->vol.vox16 + from, 0, sizeof(unsigned) * tail, st);
    if (e == cudaSuccess && s->vol.colors)
      e = cudaMemsetAsync(s->vol.colors + from, 0, sizeof(uchar4) * tail, st);
    if (e == cudaSuccess && s->vol.nonsat)
      e = cudaMemsetAsync(s->vol.nonsat + L, 0, sizeof(int) * (size_t)(n - L), st);
    if (e == cudaSuccess && s->vol.freecell)
      e = cudaMemsetAsync(s->vol.freecell + L, 0, (size_t)(n - L), st);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(&s->vol.cnt->nalloc, &L, sizeof(int), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);  // the copy reads L from this stack
    if (e != cudaSuccess) r = DYN_ERR_CUDA;
  } while (false);
  if (r != DYN_OK) cudaGetLastError();
  for (void* p : {(void*)keep, (void*)pos, (void*)dead_at, (void*)dest, (void*)gcoords,
                  (void*)gvox})
    if (p) cudaFreeAsync(p, st);
  if (cudaStreamSynchronize(st) != cudaSuccess && r == DYN_OK) r = DYN_ERR_CUDA;
  return r;
}

}  // namespace

dyn_status dyn_evict_blocks(dyn_session* s, int32_t max_age_frames, int32_t* coords_out,
                            dyn_voxel* voxels_out, int64_t capacity, int64_t* n_out) {
  if (max_age_frames < 0) return DYN_ERR_INVALID_ARG;
  auto mark = [s, max_age_frames](cudaStream_t st, int n, int* keep) -> dyn_status {
    DYN_CUDA(cudaMemsetAsync(keep, 0, sizeof(int) * (size_t)n, st));
    const long long ne = (long long)s->tp.num_buckets * s->tp.bucket_size;
    dyn::mark_age_kernel<<<dyn::grid_for(ne, dyn::kEvT), dyn::kEvT, 0, st>>>(
        s->vol.entries, ne, n, s->d_pose, max_age_frames, keep);
    return DYN_OK;
  };
  return remove_blocks(s, mark, coords_out, voxels_out, capacity, n_out);
}

dyn_status dyn_delete_blocks(dyn_session* s, const int32_t* coords, int64_t n_coords,
                             int32_t* coords_out, dyn_voxel* voxels_out, int64_t capacity,
                             int64_t* n_out) {
  if (n_coords < 0 || (n_coords > 0 && !coords)) return DYN_ERR_INVALID_ARG;
  int* dcoords = nullptr;
  int* removed = nullptr;
  auto mark = [&](cudaStream_t st, int n, int* keep) -> dyn_status {
    dyn::fill_kernel<<<dyn::grid_for(n, dyn::kEvT), dyn::kEvT, 0, st>>>(keep, n, 1);
    if (n_coords == 0) return DYN_OK;
    if (cudaMallocAsync(&dcoords, sizeof(int) * 3 * (size_t)n_coords, st) != cudaSuccess ||
        cudaMallocAsync(&removed, sizeof(int), st) != cudaSuccess)
      return DYN_ERR_OOM;
    DYN_CUDA(cudaMemcpyAsync(dcoords, coords, sizeof(int) * 3 * (size_t)n_coords,
                             cudaMemcpyHostToDevice, st));
    DYN_CUDA(cudaMemsetAsync(removed, 0, sizeof(int), st));
    dyn::mark_coords_kernel<<<dyn::grid_for(n_coords, dyn::kEvT), dyn::kEvT, 0, st>>>(
        s->vol, dcoords, n_coords, n, keep, removed);
    return DYN_OK;
  };
  dyn_status r = remove_blocks(s, mark, coords_out, voxels_out, capacity, n_out);
  if (s) {
    DeviceGuard dg(s->device);
    if (dcoords) cudaFreeAsync(dcoords, s->stream);
    if (removed) cudaFreeAsync(removed, s->stream);
    if (cudaStreamSynchronize(s->stream) != cudaSuccess && r == DYN_OK) r = DYN_ERR_CUDA;
  }
  return r;
}

dyn_status dyn_upload_blocks(dyn_session* s, const int32_t* coords, const dyn_voxel* voxels,
                             int64_t n, int64_t counts_out[4]) {
  if (!s || n < 0 || (n > 0 && (!coords || !voxels)) || !counts_out) return DYN_ERR_INVALID_ARG;
  for (int k = 0; k < 4; ++k) counts_out[k] = 0;
  if (n == 0) return DYN_OK;
  if (n > s->tp.num_blocks) return DYN_ERR_INVALID_ARG;
  DYN_TRY(quiesce(s));
  DeviceGuard dg(s->device);
  cudaStream_t st = s->stream;
  int* dcoords = nullptr;
  int* dcounts = nullptr;
  dyn_voxel* dvox = nullptr;
  dyn_status r = DYN_OK;
  int hc[4] = {0, 0, 0, 0};
  do {
    if (cudaMallocAsync(&dcoords, sizeof(int) * 3 * (size_t)n, st) != cudaSuccess ||
        cudaMallocAsync(&dvox, sizeof(dyn_voxel) * dyn::kBlockVox * (size_t)n, st) !=
            cudaSuccess ||
        cudaMallocAsync(&dcounts, sizeof(int) * 4, st) != cudaSuccess) {
      r = DYN_ERR_OOM;
      break;
    }
    if (cudaMemcpyAsync(dcoords, coords, sizeof(int) * 3 * (size_t)n, cudaMemcpyHostToDevice,
                        st) != cudaSuccess ||
        cudaMemcpyAsync(dvox, voxels, sizeof(dyn_voxel) * dyn::kBlockVox * (size_t)n,
                        cudaMemcpyHostToDevice, st) != cudaSuccess ||
        cudaMemsetAsync(dcounts, 0, sizeof(int) * 4, st) != cudaSuccess) {
      r = DYN_ERR_CUDA;
      break;
    }
    dyn::upload_kernel<<<(int)std::min<int64_t>(n, 148 * 8), dyn::kEvT, 0, st>>>(
        s->vol, s->d_pose, dcoords, dvox, (int)n, dcounts);
    if (cudaMemcpyAsync(hc, dcounts, sizeof(int) * 4, cudaMemcpyDeviceToHost, st) !=
            cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
      r = DYN_ERR_CUDA;
  } while (false);
  if (r != DYN_OK) cudaGetLastError();
  for (void* p : {(void*)dcoords, (void*)dvox, (void*)dcounts})
    if (p) cudaFreeAsync(p, st);
  if (cudaStreamSynchronize(st) != cudaSuccess && r == DYN_OK) r = DYN_ERR_CUDA;
  for (int k = 0; k < 4; ++k) counts_out[k] = hc[k];
  return r;
}

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

#include "evict_ops.h"
#include "session_impl.cuh"

namespace dyn {
namespace {

constexpr int kEvT = 256;

__global__ void fill_kernel(int* a, int n, int v) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) a[i] = v;
}

// keep[p] = 1 for the blocks touched within max_age frames of the last one.
__global__ void mark_age_kernel(const Entry* __restrict__ entries, long long ne, int n,
                                const PoseState* __restrict__ ps, int max_age,
                                int* __restrict__ keep) {
  // the frame counter advances before the allocation runs, so the last
  // frame's allocation stamped its blocks with the counter's value now
  const int last = ps->frame;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < ne;
       i += (long long)gridDim.x * blockDim.x) {
    const Entry e = entries[i];
    const int p = evict::entry_block(e, n);
    if (p >= 0 && evict::young(e, last, max_age)) keep[p] = 1;
  }
}

// keep[p] = 0 for the blocks at the m coordinates; *removed counts them once.
__global__ void mark_coords_kernel(VolumeDev v, const int* __restrict__ coords, long long m, int n,
                                   int* __restrict__ keep, int* __restrict__ removed) {
  for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < m;
       j += (long long)gridDim.x * blockDim.x) {
    const int p = find_block(v.entries, v.t, coords[3 * j], coords[3 * j + 1], coords[3 * j + 2]);
    if (p >= 0 && p < n && atomicExch(&keep[p], 0) == 1) atomicAdd(removed, 1);
  }
}

// Exclusive prefix sums of n flags into pos[0..n] (pos[n] = the total); one
// CTA of 1024 threads, each a contiguous chunk.
__global__ void __launch_bounds__(1024) scan_flags_kernel(const int* __restrict__ keep, int n,
                                                          int* __restrict__ pos) {
  __shared__ int sums[1024];
  const int t = threadIdx.x;
  const int chunk = (n + 1023) / 1024;
  const long long lo = (long long)t * chunk;
  const long long hi = lo + chunk < n ? lo + chunk : (long long)n;
  int s = 0;
  for (long long i = lo; i < hi; ++i) s += keep[i];
  sums[t] = s;
  __syncthreads();
  for (int o = 1; o < 1024; o <<= 1) {
    const int y = t >= o ? sums[t - o] : 0;
    __syncthreads();
    sums[t] += y;
    __syncthreads();
  }
  int run = sums[t] - s;
  for (long long i = lo; i < hi; ++i) {
    pos[i] = run;
    run += keep[i];
  }
  if (t == 1023) pos[n] = sums[1023];
}

// dead_at[k] = the k-th removed block (index order); the first ones are the
// holes below L.
__global__ void dead_list_kernel(const int* __restrict__ keep, const int* __restrict__ pos, int n,
                                 int* __restrict__ dead_at) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    if (!keep[i]) dead_at[evict::hole_rank(i, pos)] = i;
}

__global__ void dest_kernel(const int* __restrict__ keep, const int* __restrict__ pos, int n, int L,
                            const int* __restrict__ dead_at, int* __restrict__ dest) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    dest[i] = evict::destination(i, L, keep, pos, dead_at);
}

// One voxel of either form in the 8-byte layout (weights above 255 clamp).
__device__ inline dyn_voxel voxel8(const VolumeDev& v, size_t i) {
  dyn_voxel o;
  if (!v.fp16) {
    o = v.voxels[i];
    return o;
  }
  const unsigned raw = v.vox16[i];
  __half_raw hr;
  hr.x = (unsigned short)(raw & 0xffffu);
  o.sdf = __half2float(__half(hr)) * v.t.trunc;  // stored as sdf / trunc
  const unsigned w = raw >> 16;
  o.weight = (uint8_t)(w > 255u ? 255u : w);
  if (v.colors) {
    const uchar4 c = v.colors[i];
    o.r = c.x;
    o.g = c.y;
    o.b = c.z;
  } else {
    o.r = o.g = o.b = 0;
  }
  return o;
}

// The k-th removed block's coordinate and voxels into the staging output
// (one CTA per block, k < m).
__global__ void gather_kernel(VolumeDev v, const int* __restrict__ dead_at, int m,
                              int* __restrict__ coords, dyn_voxel* __restrict__ vox) {
  for (int k = blockIdx.x; k < m; k += gridDim.x) {
    const int i = dead_at[k];
    if (threadIdx.x == 0) {
      const unsigned long long key = v.block_keys[i];
      coords[3 * k] = key_x(key);
      coords[3 * k + 1] = key_y(key);
      coords[3 * k + 2] = key_z(key);
    }
    for (int j = threadIdx.x; j < kBlockVox; j += blockDim.x)
      vox[(size_t)k * kBlockVox + j] = voxel8(v, (size_t)i * kBlockVox + j);
  }
}

// Survivor j (L <= j < n) into its hole: voxels and key (one CTA per block).
__global__ void move_kernel(VolumeDev v, int n, int L, const int* __restrict__ dest) {
  for (int j = L + blockIdx.x; j < n; j += gridDim.x) {
    const int d = dest[j];
    if (d < 0) continue;  // removed
    const size_t src = (size_t)j * kBlockVox, dst = (size_t)d * kBlockVox;
    if (!v.fp16) {
      const uint4* s4 = reinterpret_cast<const uint4*>(v.voxels + src);
      uint4* d4 = reinterpret_cast<uint4*>(v.voxels + dst);
      for (int q = threadIdx.x; q < kBlockVox * (int)sizeof(dyn_voxel) / 16; q += blockDim.x)
        d4[q] = s4[q];
    } else {
      const uint4* s4 = reinterpret_cast<const uint4*>(v.vox16 + src);
      uint4* d4 = reinterpret_cast<uint4*>(v.vox16 + dst);
      for (int q = threadIdx.x; q < kBlockVox * 4 / 16; q += blockDim.x) d4[q] = s4[q];
      if (v.colors) {
        const uint4* c4 = reinterpret_cast<const uint4*>(v.colors + src);
        uint4* e4 = reinterpret_cast<uint4*>(v.colors + dst);
        for (int q = threadIdx.x; q < kBlockVox * 4 / 16; q += blockDim.x) e4[q] = c4[q];
      }
    }
    if (threadIdx.x == 0) v.block_keys[d] = v.block_keys[j];
  }
}

__global__ void rewrite_kernel(Entry* entries, int nbuckets, int bsz, int n,
                               const int* __restrict__ keep, const int* __restrict__ dest) {
  for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < nbuckets; b += gridDim.x * blockDim.x)
    evict::rewrite_bucket(entries + (size_t)b * bsz, bsz, n, keep, dest);
}

// Blocks from the host into the volume: each key inserted (stamped with the
// last frame), a heap index taken for a new one, its voxels written in the
// volume's form.  Keys already present are left as they are.  counts:
// [placed, present, bucket full, heap exhausted].
__global__ void upload_kernel(VolumeDev v, const PoseState* __restrict__ ps,
                              const int* __restrict__ coords, const dyn_voxel* __restrict__ vox,
                              int m, int* __restrict__ counts) {
  __shared__ int ptr_s;
  __shared__ int unique_s;  // bucket_insert's probe count (unused here)
  for (int k = blockIdx.x; k < m; k += gridDim.x) {
    if (threadIdx.x == 0) {
      const unsigned long long key = pack_key(coords[3 * k], coords[3 * k + 1], coords[3 * k + 2]);
      const int r = bucket_insert(v.entries, v.t, key, ps->frame, &unique_s);
      int ptr = -1;
      if (r >= 0) {
        ptr = atomicAdd(&v.cnt->nalloc, 1);
        if (ptr < v.t.num_blocks) {
          v.entries[r].ptr = ptr;
          v.block_keys[ptr] = key;
          atomicAdd(&counts[0], 1);
        } else {
          ptr = -1;
          atomicAdd(&counts[3], 1);
        }
      } else {
        atomicAdd(&counts[r == -1 ? 1 : 2], 1);
      }
      ptr_s = ptr;
    }
    __syncthreads();
    const int ptr = ptr_s;
    if (ptr >= 0) {
      for (int j = threadIdx.x; j < kBlockVox; j += blockDim.x) {
        const dyn_voxel o = vox[(size_t)k * kBlockVox + j];
        const size_t i = (size_t)ptr * kBlockVox + j;
        if (!v.fp16) {
          v.voxels[i] = o;
        } else {
          const __half h = __float2half_rn(o.sdf / v.t.trunc);
          v.vox16[i] = (unsigned)__half_as_ushort(h) | ((unsigned)o.weight << 16);
          if (v.colors) v.colors[i] = make_uchar4(o.r, o.g, o.b, 0);
        }
      }
    }
    __syncthreads();  // ptr_s is rewritten for the next block
  }
}

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

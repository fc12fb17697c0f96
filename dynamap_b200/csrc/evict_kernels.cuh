// evict_kernels.cuh -- the kernels of block eviction (evict.cu, which
// describes the method): included by evict.cu, and by the host emulation of
// CUDA thread blocks the tests run the same kernels on.
#pragma once
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include "evict_ops.h"
#include "tsdf.cuh"

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
    if (threadIdx.x == 0) {
      v.block_keys[d] = v.block_keys[j];
      if (v.nonsat) {  // the free-space summaries move with the block
        v.nonsat[d] = v.nonsat[j];
        v.freecell[d] = v.freecell[j];
      }
    }
  }
}

__global__ void rewrite_kernel(Entry* entries, int nbuckets, int bsz, int n,
                               const int* __restrict__ keep, const int* __restrict__ dest) {
  for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < nbuckets; b += gridDim.x * blockDim.x)
    evict::rewrite_bucket(entries + (size_t)b * bsz, bsz, n, keep, dest);
}

// Blocks from the host into the volume: each key inserted (stamped with the
// last frame), a heap index taken for a new one, its voxels written in the
// volume's form.  Keys already present with a block are left as they are.
// A key whose entry has no block (an earlier insert found the heap full)
// takes a heap index now if there is one, so a retry after a heap-exhausted
// result places the block or reports the heap exhausted again, never
// "present".  Whichever CTA moves the entry's ptr from -1 to the claim mark
// -3 gives it its heap index, so a key that occurs twice is placed once.
// counts: [placed, present, bucket full, heap exhausted].
// A placed block's free-space summaries: its count of observed,
// non-saturated voxels, its own free-cell flag cleared (set again by the
// next frame that sees it), and, when it holds such voxels, the flags of
// its seven lower neighbours cleared (their cells read it).
__global__ void upload_kernel(VolumeDev v, const PoseState* __restrict__ ps,
                              const int* __restrict__ coords, const dyn_voxel* __restrict__ vox,
                              int m, int* __restrict__ counts) {
  __shared__ int ptr_s;
  __shared__ int unique_s;  // bucket_insert's probe count (unused here)
  __shared__ int nonsat_s;
  for (int k = blockIdx.x; k < m; k += gridDim.x) {
    if (threadIdx.x == 0) {
      const unsigned long long key = pack_key(coords[3 * k], coords[3 * k + 1], coords[3 * k + 2]);
      const int r = bucket_insert(v.entries, v.t, key, ps->frame, &unique_s);
      const int e = r >= 0 ? r : (r == -1 ? find_entry(v.entries, v.t, key) : -1);
      int ptr = -1;
      if (e < 0) {
        atomicAdd(&counts[2], 1);  // bucket full
      } else if (atomicCAS(&v.entries[e].ptr, -1, -3) == -1) {
        ptr = atomicAdd(&v.cnt->nalloc, 1);
        if (ptr < v.t.num_blocks) {
          atomicExch(&v.entries[e].ptr, ptr);
          v.block_keys[ptr] = key;
          atomicAdd(&counts[0], 1);
        } else {
          ptr = -1;
          atomicExch(&v.entries[e].ptr, -1);
          atomicAdd(&counts[3], 1);
        }
      } else {
        atomicAdd(&counts[1], 1);  // present with a block (or placed by another CTA)
      }
      ptr_s = ptr;
      nonsat_s = 0;
    }
    __syncthreads();
    const int ptr = ptr_s;
    if (ptr >= 0) {
      int ns = 0;
      for (int j = threadIdx.x; j < kBlockVox; j += blockDim.x) {
        const dyn_voxel o = vox[(size_t)k * kBlockVox + j];
        const size_t i = (size_t)ptr * kBlockVox + j;
        if (!v.fp16) {
          v.voxels[i] = o;
          ns += o.weight != 0 && !(o.sdf >= v.sat_lo);
        } else {
          const __half h = __float2half_rn(o.sdf / v.t.trunc);
          v.vox16[i] = (unsigned)__half_as_ushort(h) | ((unsigned)o.weight << 16);
          if (v.colors) v.colors[i] = make_uchar4(o.r, o.g, o.b, 0);
          ns += o.weight != 0 && __half_as_ushort(h) != 0x3C00u;
        }
      }
      if (ns) atomicAdd(&nonsat_s, ns);
    }
    __syncthreads();
    if (ptr >= 0 && threadIdx.x == 0 && v.nonsat) {
      v.nonsat[ptr] = nonsat_s;
      v.freecell[ptr] = 0;
      if (nonsat_s) {
        const int x = coords[3 * k], y = coords[3 * k + 1], z = coords[3 * k + 2];
        for (int q = 1; q < 8; ++q) {
          const int lo = find_block(v.entries, v.t, x - (q & 1), y - ((q >> 1) & 1),
                                    z - ((q >> 2) & 1));
          if (lo >= 0) v.freecell[lo] = 0;
        }
      }
    }
    __syncthreads();  // ptr_s and nonsat_s are rewritten for the next block
  }
}

}  // namespace
}  // namespace dyn

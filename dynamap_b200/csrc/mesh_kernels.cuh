// mesh_kernels.cuh -- the kernels of the mesh extraction (mesh.cu, which
// describes the method): included by mesh.cu, and by the host emulation of
// CUDA thread blocks the tests run the same kernels on.
#pragma once
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include "mc_tables.h"
#include "mesh_cell.h"
#include "tsdf.cuh"

namespace dyn {
namespace {

// Voxels per tile edge: a block plus the 3 above it that its cells' samples
// reach.  Samples outside the tile read the volume, so any edge of at least
// 8 gives the same mesh; the tests build a smaller tile to exercise that
// path.
#ifndef DYN_MESH_TILE
#define DYN_MESH_TILE 11
#endif
constexpr int kTile = DYN_MESH_TILE;
static_assert(kTile >= 8 && kTile <= 16, "the tile spans the block and at most one more");
constexpr int kTileVox = kTile * kTile * kTile;
constexpr int kMeshThreads = 256;
constexpr int kMeshWarps = kMeshThreads / 32;
constexpr int kTriFloats = 18;  // three vertices of {x, y, z, r, g, b}

__device__ signed char d_mc_tri[256][kMcMaxTriIdx];

// One voxel of either form in the 8-byte layout (weights above 255 clamp:
// only zero / non-zero is read).
__device__ inline uint2 voxel_bits(const VolumeDev& v, int ptr, int lin) {
  if (ptr < 0) return make_uint2(0u, 0u);
  const size_t i = (size_t)ptr * kBlockVox + lin;
  if (!v.fp16) return __ldg(reinterpret_cast<const uint2*>(v.voxels) + i);
  const unsigned raw = __ldg(v.vox16 + i);
  __half_raw hr;
  hr.x = (unsigned short)(raw & 0xffffu);
  const float sdf = __half2float(__half(hr)) * v.t.trunc;  // stored as sdf / trunc
  const unsigned w = raw >> 16;
  unsigned rgb = 0u;
  if (v.colors) {
    const uchar4 c = v.colors[i];
    rgb = (unsigned)c.x | ((unsigned)c.y << 8) | ((unsigned)c.z << 16);
  }
  return make_uint2(rgb | ((w > 255u ? 255u : w) << 24), __float_as_uint(sdf));
}

// The Sampler of mesh_cell.h over a staged tile (global fallback).
struct TileSampler {
  const VolumeDev* v;
  const uint2* tile;  // shared: kTile^3 voxels from (ox, oy, oz)
  int ox, oy, oz;
  float inv_vs;
  __device__ int index(float p) const { return voxel_index(p, v->t.vs, inv_vs); }
  __device__ mesh::VoxelBits fetch(int gx, int gy, int gz) const {
    const unsigned tx = (unsigned)(gx - ox), ty = (unsigned)(gy - oy), tz = (unsigned)(gz - oz);
    uint2 r;
    if (tx < (unsigned)kTile && ty < (unsigned)kTile && tz < (unsigned)kTile) {
      r = tile[(tx * kTile + ty) * kTile + tz];
    } else {
      const int ptr = find_block(v->entries, v->t, blk_of(gx), blk_of(gy), blk_of(gz));
      r = voxel_bits(*v, ptr, (loc_of(gx) << 6) | (loc_of(gy) << 3) | loc_of(gz));
    }
    mesh::VoxelBits b;
    b.rgbw = r.x;
    b.sdf = __uint_as_float(r.y);
    return b;
  }
};

// Exclusive prefix of x over the CTA; *total gets the sum.  Every thread of
// the CTA calls it.
__device__ inline int cta_exclusive_scan(int x, int* warp_sums, int* total) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  int inc = x;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= o) inc += y;
  }
  if (lane == 31) warp_sums[w] = inc;
  __syncthreads();
  int before = 0, all = 0;
#pragma unroll
  for (int k = 0; k < kMeshWarps; ++k) {
    const int s = warp_sums[k];
    before += k < w ? s : 0;
    all += s;
  }
  __syncthreads();  // warp_sums is reused by the next call
  *total = all;
  return before + inc - x;
}

// Pass 1 (WRITE false): triangles per allocated block into counts.  Pass 2
// (WRITE true): the triangles of block i from offsets[i] on, those below cap.
template <bool WRITE>
__global__ void __launch_bounds__(kMeshThreads) mesh_blocks_kernel(
    const __grid_constant__ VolumeDev v, const mesh::Grid g, int nblocks,
    long long* __restrict__ counts,
    const long long* __restrict__ offsets, float* __restrict__ out, long long cap) {
  __shared__ uint2 tile[kTileVox];
  __shared__ int ptrs[8];
  __shared__ int range[3][2];
  __shared__ int warp_sums[kMeshWarps];
  const float inv_vs = 1.0f / v.t.vs;
  for (int blk = blockIdx.x; blk < nblocks; blk += gridDim.x) {
    const unsigned long long key = v.block_keys[blk];
    const int b[3] = {key_x(key), key_y(key), key_z(key)};
    TileSampler S{&v, tile, 8 * b[0], 8 * b[1], 8 * b[2], inv_vs};
    const int t = threadIdx.x;
    if (t < 6) {
      const int axis = t >> 1;
      range[axis][t & 1] = mesh::key_lower_bound(g, S, axis, 8 * b[axis] + 8 * (t & 1));
    } else if (t >= 32 && t < 40) {  // another warp: the eight heap indices
      const int k = t - 32;
      ptrs[k] = find_block(v.entries, v.t, b[0] + (k >> 2), b[1] + ((k >> 1) & 1), b[2] + (k & 1));
    }
    __syncthreads();
    const int nx = range[0][1] - range[0][0], ny = range[1][1] - range[1][0],
              nz = range[2][1] - range[2][0];
    const long long ncell = (nx > 0 && ny > 0 && nz > 0) ? (long long)nx * ny * nz : 0;
    if (ncell > 0) {
      for (int i = t; i < kTileVox; i += kMeshThreads) {
        const int tx = i / (kTile * kTile), ty = (i / kTile) % kTile, tz = i % kTile;
        const int ptr = ptrs[((tx >> 3) << 2) | ((ty >> 3) << 1) | (tz >> 3)];
        tile[i] = voxel_bits(v, ptr, ((tx & 7) << 6) | ((ty & 7) << 3) | (tz & 7));
      }
    }
    __syncthreads();
    long long base = 0;
    for (long long c0 = 0; c0 < ncell; c0 += kMeshThreads) {  // uniform over the CTA
      const long long c = c0 + t;
      int ntri = 0, cube = -1;
      int ix = 0, iy = 0, iz = 0;
      float pos[3], d[8];
      if (c < ncell) {
        ix = range[0][0] + (int)(c % nx);
        iy = range[1][0] + (int)((c / nx) % ny);
        iz = range[2][0] + (int)(c / ((long long)nx * ny));
        cube = mesh::cell_cube(g, S, ix, iy, iz, pos, d);
        if (cube > 0 && cube < 255) ntri = mesh::cube_triangles(d_mc_tri[cube], kMcMaxTriIdx);
      }
      int total = 0;
      const int before = cta_exclusive_scan(ntri, warp_sums, &total);
      if (WRITE && ntri > 0) {
        const mesh::VoxelBits centre =
            S.fetch(S.index(pos[0]), S.index(pos[1]), S.index(pos[2]));
        const signed char* row = d_mc_tri[cube];
        long long o = offsets[blk] + base + before;
        for (int j = 0; j < ntri; ++j, ++o) {
          if (o >= cap) break;
          float* dst = out + (size_t)o * kTriFloats;
          for (int k = 0; k < 3; ++k)
            mesh::edge_vertex(g, pos, d, centre.rgbw & 0xffffffu, row[3 * j + k], dst + 6 * k);
        }
      }
      base += total;
    }
    if (!WRITE && t == 0) counts[blk] = base;
    __syncthreads();  // tile and ranges are rewritten for the next block
  }
}

// Exclusive scan of n counts into offsets (one CTA of 1024 threads, each a
// contiguous chunk); *total gets the sum.
__global__ void __launch_bounds__(1024) mesh_scan_kernel(const long long* __restrict__ counts, int n,
                                                         long long* __restrict__ offsets,
                                                         long long* __restrict__ total) {
  __shared__ long long sums[1024];
  const int t = threadIdx.x;
  const int chunk = (n + 1023) / 1024;
  const long long lo = (long long)t * chunk;
  const long long hi = lo + chunk < n ? lo + chunk : (long long)n;
  long long s = 0;
  for (long long i = lo; i < hi; ++i) s += counts[i];
  sums[t] = s;
  __syncthreads();
  for (int o = 1; o < 1024; o <<= 1) {  // Hillis-Steele inclusive scan
    const long long y = t >= o ? sums[t - o] : 0;
    __syncthreads();
    sums[t] += y;
    __syncthreads();
  }
  long long run = sums[t] - s;
  for (long long i = lo; i < hi; ++i) {
    offsets[i] = run;
    run += counts[i];
  }
  if (t == 1023) *total = sums[1023];
}

}  // namespace
}  // namespace dyn

// tsdf.cu -- voxel-hashed TSDF kernels.
//
// Reference: include/geometry/tsdf/tsdf.cu (integration :268-344, allocation
// :346-453, raycast :471-526, voxel addressing :47-239),
// include/dataStructure/hashTable/hashTable.cu (:80-163),
// include/geometry/geom_Types.h (Voxel merge :79-103).
//
// Layout in HBM (per session): a bucketed hash of 16-byte entries
// {u64 packed block key, i32 heap index, i32 frame stamp}; a heap-index ->
// key array; voxels as 8-byte {r,g,b,w,f32 sdf} (the reference's Voxel),
// 512 per block in x-major order, so one block is 4 KB contiguous.  The
// mixed form keeps {f16 sdf / truncation, u16 weight} per voxel (2 KB per
// block) and an optional uchar4 colour array.
//
// Each stage is a __device__ body used by a by-value kernel (one session)
// and by a fused kernel over every session of a frame (blockIdx.z).
#include "tsdf.cuh"

#include <cuda_fp16.h>

#include "sessdev.cuh"

namespace dyn {

namespace {

// ------------------------------------------------------------ allocation
constexpr int kAllocT = 16;          // 16x16 pixel tile per CTA
constexpr int kSetSlots = 2048;      // CTA-local dedup set (16 KB)
constexpr int kSetProbes = 32;

__device__ inline unsigned set_hash(unsigned long long k) {
  return (unsigned)((k * 0x9E3779B97F4A7C15ull) >> 53) & (kSetSlots - 1);
}

struct AllocSmem {
  unsigned long long set[kSetSlots];
  int claim_entry[kSetSlots];
  int nclaims;
  int base;
  int new_blocks, bucket_full, heap_exhausted, unique, overruns;
};

// bucket_insert (the lock-free unique insert) is in common.cuh.

// AllocateFromDepthKernel (tsdf.cu:346-453) for one pixel: the reference's
// DDA over blocks, exact FP32 (this file is built with -fmad=false), with
// the 'diff' pre-step for negative directions and the step cap.
template <class F>
__device__ inline bool dda_ray(F3 start_pt, F3 point, float trunc, float block_size, int cap,
                               F&& visit) {
  F3 dir = normalize3(point - start_pt);
  float surface_distance = norm3(start_pt - point);
  F3 ray_start = start_pt;
  F3 ray_end = start_pt + dir * (surface_distance + trunc);
  int bpx = (int)floorf(ray_start.x / block_size);
  int bpy = (int)floorf(ray_start.y / block_size);
  int bpz = (int)floorf(ray_start.z / block_size);
  int ebx = (int)floorf(ray_end.x / block_size);
  int eby = (int)floorf(ray_end.y / block_size);
  int ebz = (int)floorf(ray_end.z / block_size);
  int sx = (dir.x > 0) - (dir.x < 0), sy = (dir.y > 0) - (dir.y < 0),
      sz = (dir.z > 0) - (dir.z < 0);
  const float FMAX = 3.402823466e+38f;
  float dtx = dir.x != 0 ? fabsf(block_size / dir.x) : FMAX;
  float dty = dir.y != 0 ? fabsf(block_size / dir.y) : FMAX;
  float dtz = dir.z != 0 ? fabsf(block_size / dir.z) : FMAX;
  float bdx = ((float)bpx + (float)sx) * block_size;
  float bdy = ((float)bpy + (float)sy) * block_size;
  float bdz = ((float)bpz + (float)sz) * block_size;
  float mx = dir.x != 0 ? (bdx - ray_start.x) / dir.x : FMAX;
  float my = dir.y != 0 ? (bdy - ray_start.y) / dir.y : FMAX;
  float mz = dir.z != 0 ? (bdz - ray_start.z) / dir.z : FMAX;
  int dx = 0, dy = 0, dz = 0;
  bool neg = false;
  if (bpx != ebx && dir.x < 0) { dx--; neg = true; }
  if (bpy != eby && dir.y < 0) { dy--; neg = true; }
  if (bpz != ebz && dir.z < 0) { dz--; neg = true; }
  visit(bpx, bpy, bpz);
  if (neg) {
    bpx += dx;
    bpy += dy;
    bpz += dz;
    visit(bpx, bpy, bpz);
  }
  int steps = 0;
  while (bpx != ebx || bpy != eby || bpz != ebz) {
    if (steps++ >= cap) return false;
    if (mx < my) {
      if (mx < mz) { bpx += sx; mx += dtx; }
      else { bpz += sz; mz += dtz; }
    } else {
      if (my < mz) { bpy += sy; my += dty; }
      else { bpz += sz; mz += dtz; }
    }
    visit(bpx, bpy, bpz);
  }
  return true;
}

// One 16x16 pixel tile (tx, ty) of AllocateFromDepthKernel.
__device__ inline void allocate_tile(const float* __restrict__ depth, const DSensor& s,
                                     const VolumeDev& v, const PoseState* __restrict__ ps,
                                     int tx, int ty) {
  __shared__ AllocSmem sm;
  __shared__ M4f T;
  __shared__ int stamp_s;
  const int tid = threadIdx.y * kAllocT + threadIdx.x;
  for (int k = tid; k < kSetSlots; k += kAllocT * kAllocT) sm.set[k] = kEmptyKey;
  if (tid < 16) T.m[tid] = ps->posef[tid];
  if (tid == 0) {
    sm.nclaims = 0;
    sm.new_blocks = sm.bucket_full = sm.heap_exhausted = sm.unique = sm.overruns = 0;
    stamp_s = ps->frame;
  }
  __syncthreads();
  const int stamp = stamp_s;
  const DTsdf& t = v.t;
  const int x = tx * kAllocT + threadIdx.x;
  const int y = ty * kAllocT + threadIdx.y;
  if (x < s.cols && y < s.rows) {
    const int i = y * s.cols + x;
    const float d = depth[i];
    if (!(d < t.dmin || d > t.dmax)) {  // tsdf.cu:442-444
      F3 point = xform(T, point3d_uv(x, y, d, s));
      if (!(point.x == 0 && point.y == 0 && point.z == 0)) {
        F3 start_pt = f3(T.m[3], T.m[7], T.m[11]);
        // band allocation: the ray starts a truncation distance before the
        // surface point instead of at the camera
        if (t.band) start_pt = point - normalize3(point - start_pt) * t.trunc;
        bool ok = dda_ray(start_pt, point, t.trunc, t.bsm, t.dda_cap, [&](int bx, int by, int bz) {
          unsigned long long key = pack_key(bx, by, bz);
          unsigned h = set_hash(key);
          for (int p = 0; p < kSetProbes; ++p) {
            unsigned slot = (h + p) & (kSetSlots - 1);
            // neighbouring rays visit the same blocks: most visits find
            // their key already in the set with a plain read
            unsigned long long old = *(volatile unsigned long long*)&sm.set[slot];
            if (old == key) return;
            if (old == kEmptyKey) {
              old = atomicCAS(&sm.set[slot], kEmptyKey, key);
              if (old == kEmptyKey || old == key) return;
            }
          }
          // set saturated: insert directly
          int r = bucket_insert(v.entries, t, key, stamp, &sm.unique);
          if (r >= 0) {
            int ptr = atomicAdd(&v.cnt->nalloc, 1);
            if (ptr < t.num_blocks) {
              v.entries[r].ptr = ptr;
              v.block_keys[ptr] = key;
              atomicAdd(&sm.new_blocks, 1);
            } else {
              atomicAdd(&sm.heap_exhausted, 1);
            }
          } else if (r == -2) {
            atomicAdd(&sm.bucket_full, 1);
          }
        });
        if (!ok) atomicAdd(&sm.overruns, 1);
      }
    }
  }
  __syncthreads();
  // drain the set into the global table
  for (int k = tid; k < kSetSlots; k += kAllocT * kAllocT) {
    unsigned long long key = sm.set[k];
    if (key == kEmptyKey) continue;
    int r = bucket_insert(v.entries, t, key, stamp, &sm.unique);
    if (r >= 0) {
      int c = atomicAdd(&sm.nclaims, 1);
      sm.claim_entry[c] = r;
    } else if (r == -2) {
      atomicAdd(&sm.bucket_full, 1);
    }
  }
  __syncthreads();
  if (tid == 0 && sm.nclaims > 0) sm.base = atomicAdd(&v.cnt->nalloc, sm.nclaims);
  __syncthreads();
  for (int c = tid; c < sm.nclaims; c += kAllocT * kAllocT) {
    int ptr = sm.base + c;
    int e = sm.claim_entry[c];
    if (ptr < t.num_blocks) {
      v.entries[e].ptr = ptr;
      v.block_keys[ptr] = v.entries[e].key;
      atomicAdd(&sm.new_blocks, 1);
    } else {
      atomicAdd(&sm.heap_exhausted, 1);
    }
  }
  __syncthreads();
  if (tid == 0) {
    if (sm.new_blocks) atomicAdd(&v.cnt->new_blocks, sm.new_blocks);
    if (sm.bucket_full) atomicAdd(&v.cnt->bucket_full, sm.bucket_full);
    if (sm.heap_exhausted) atomicAdd(&v.cnt->heap_exhausted, sm.heap_exhausted);
    if (sm.unique) atomicAdd(&v.cnt->unique_probed, sm.unique);
    if (sm.overruns) atomicAdd(&v.cnt->dda_overruns, sm.overruns);
  }
}

// (8 CTAs per SM -- at most 32 registers, 24.7 KB of shared memory each --
// so that a 640x480 frame's 1,200 tiles run in one wave instead of 1.35)
__global__ void __launch_bounds__(kAllocT* kAllocT, 8)
    fused_allocate_kernel(const SessDev* __restrict__ tab) {
  const SessDev& S = tab[blockIdx.z];
  const DSensor& s = S.ls[0];
  if ((int)blockIdx.x * kAllocT >= s.cols || (int)blockIdx.y * kAllocT >= s.rows) return;
  allocate_tile(S.raw, s, S.vol, S.pose, blockIdx.x, blockIdx.y);
}

// ------------------------------------------------------------ visibility
// IntegrateScanKernel's block test (tsdf.cu:283-300): block origin to the
// camera, z < 0 rejected, the origin plus half a block (in camera axes,
// computed in double) projected into the image.
__device__ inline bool block_visible(unsigned long long key, const DTsdf& t, const DSensor& s,
                                     const M4f& invT) {
  const float vs = t.vs;
  const int bs = kBlockSize;
  F3 position = f3((float)key_x(key) * vs * (float)bs, (float)key_y(key) * vs * (float)bs,
                   (float)key_z(key) * vs * (float)bs);
  F3 pc = xform(invT, position);
  if (pc.z < 0) return false;
  double half = 0.5 * (double)vs * (double)bs;
  F3 bc = f3((float)((double)pc.x + half), (float)((double)pc.y + half),
             (float)((double)pc.z + half));
  int ix, iy;
  if (!project(bc, s, &ix, &iy)) return false;
  return ix >= 0 && iy >= 0 && ix < s.cols && iy < s.rows;
}

// ------------------------------------------------------------ ray depth bounds
// A ray sample whose voxel lies in no allocated block reads weight 0 and
// steps one truncation distance (tsdf.cu:505-507), so for every 8x8 pixel
// tile the frame's raycast gets a lower bound on the camera depth at which
// any of its rays can first enter an allocated block and an upper bound on
// the depth at which the last one leaves one: below the first and above the
// second (and beyond the near distance, where rays are marched normally) a
// sample needs no lookup, the march adds the truncation distance just as
// the lookup would have made it -- the same steps, so the same depths.
// Band sessions (blocks only near surfaces) skip most of every ray; the
// reference's carving allocation fills the space in front of surfaces, so
// there the far bound is what skips (rays past the scene).  Each allocated
// block contributes its box widened by one voxel beyond the rounding cells
// of its outer voxels, clipped to camera depth >= the near distance,
// projected and widened by one pixel: the tiles its bounding rectangle
// touches get min(near, nearest depth of the box) and max(far, farthest
// depth of the box).
// The bounds buffer of a session with tiles_x x tiles_y fine tiles
// (ray_bounds_words): near and far per fine tile, then near and far per
// coarse tile; a pixel's bounds are min(near) / max(far) over both levels.
struct RayBounds {
  unsigned *near8, *far8, *near64, *far64;
  int cx, cy;
};
__device__ inline RayBounds ray_bounds(unsigned* rb, int tiles_x, int tiles_y) {
  RayBounds B;
  B.cx = (tiles_x + kRbCoarse - 1) / kRbCoarse;
  B.cy = (tiles_y + kRbCoarse - 1) / kRbCoarse;
  B.near8 = rb;
  B.far8 = rb + tiles_x * tiles_y;
  B.near64 = B.far8 + tiles_x * tiles_y;
  B.far64 = B.near64 + B.cx * B.cy;
  return B;
}

__device__ inline float ray_near(const DTsdf& t) { return t.bsm; }

__device__ inline void bound_block(unsigned long long key, const DTsdf& t, const DSensor& s,
                                   const M4f& invT, unsigned* __restrict__ rb, int tiles_x,
                                   int tiles_y, bool near, bool far) {
  const float vs = t.vs;
  const float znear = ray_near(t);
  const float lo[3] = {((float)key_x(key) * 8.0f - 1.5f) * vs,
                       ((float)key_y(key) * 8.0f - 1.5f) * vs,
                       ((float)key_z(key) * 8.0f - 1.5f) * vs};
  const float ext = 11.0f * vs;
  F3 c[8];
  float zmin = 3.0e38f, zmax = -3.0e38f;
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    c[k] = xform(invT, f3(lo[0] + ((k & 1) ? ext : 0.0f), lo[1] + ((k & 2) ? ext : 0.0f),
                          lo[2] + ((k & 4) ? ext : 0.0f)));
    zmin = fminf(zmin, c[k].z);
    zmax = fmaxf(zmax, c[k].z);
  }
  if (!(zmax >= znear)) return;  // wholly nearer than the near distance
  float umin = 3.0e38f, umax = -3.0e38f, vmin = 3.0e38f, vmax = -3.0e38f;
  auto add = [&](float X, float Y, float Z) {
    const float u = s.fx * X / Z + s.cx, w = s.fy * Y / Z + s.cy;
    umin = fminf(umin, u);
    umax = fmaxf(umax, u);
    vmin = fminf(vmin, w);
    vmax = fmaxf(vmax, w);
  };
#pragma unroll
  for (int k = 0; k < 8; ++k)
    if (c[k].z >= znear) add(c[k].x, c[k].y, c[k].z);
  // the 12 box edges (corner pairs differing in one bit) cut by z = znear
#pragma unroll
  for (int k = 0; k < 8; ++k)
#pragma unroll
    for (int bit = 1; bit < 8; bit <<= 1) {
      if (k & bit) continue;
      const F3 a = c[k], b = c[k | bit];
      if ((a.z < znear) != (b.z < znear)) {
        const float f = (znear - a.z) / (b.z - a.z);
        add(a.x + f * (b.x - a.x), a.y + f * (b.y - a.y), znear);
      }
    }
  umin -= 1.0f;
  vmin -= 1.0f;
  umax += 1.0f;
  vmax += 1.0f;
  if (!(umax >= 0.0f && vmax >= 0.0f && umin <= (float)(s.cols - 1) &&
        vmin <= (float)(s.rows - 1)))
    return;
  const int tx0 = umin <= 0.0f ? 0 : min((int)umin / kRbTile, tiles_x - 1);
  const int ty0 = vmin <= 0.0f ? 0 : min((int)vmin / kRbTile, tiles_y - 1);
  const int tx1 = umax >= (float)(s.cols - 1) ? tiles_x - 1 : (int)umax / kRbTile;
  const int ty1 = vmax >= (float)(s.rows - 1) ? tiles_y - 1 : (int)vmax / kRbTile;
  // Non-negative floats order as their bit patterns.  A block whose
  // rectangle spans more than 16 tiles (one close to the camera) goes to
  // the coarse level instead, so that no thread walks hundreds of tiles;
  // the coarse bounds of such blocks are loose only near the camera.
  // Carving sessions' blocks start at the camera: their near bound comes
  // from the blocks that hold observed non-saturated voxels (mixed form,
  // fused_surface_bound_kernel) or stays 0 (FP32 form).
  const unsigned zb = __float_as_uint(fmaxf(zmin, 0.0f)), ze = __float_as_uint(zmax);
  RayBounds B = ray_bounds(rb, tiles_x, tiles_y);
  unsigned *nb = B.near8, *fb = B.far8;
  int tw = tiles_x, x0 = tx0, x1 = tx1, y0 = ty0, y1 = ty1;
  if ((tx1 - tx0 + 1) * (ty1 - ty0 + 1) > 16) {
    nb = B.near64;
    fb = B.far64;
    tw = B.cx;
    x0 = tx0 / kRbCoarse;
    x1 = tx1 / kRbCoarse;
    y0 = ty0 / kRbCoarse;
    y1 = ty1 / kRbCoarse;
  }
  for (int ty = y0; ty <= y1; ++ty)
    for (int tx = x0; tx <= x1; ++tx) {
      if (near) atomicMin(nb + ty * tw + tx, zb);
      if (far) atomicMax(fb + ty * tw + tx, ze);
    }
}

// Free-space blocks of a depth-only frame.  A voxel whose point is nearer
// than (sdist - truncation) of its pixel takes IntegrateScanKernel's
// free-space branch (sdf = truncation).  A visible block is a free-space
// block when that holds for every voxel: the block's voxel points (the box
// of corners origin .. origin + 7 voxels) lie in front of the camera and
// project inside the image (a pixel of margin around the corners'
// projections), and the farthest corner (with 1e-5 relative + 1e-5 m of
// margin) is nearer than the free-space tile map's least (sdist -
// truncation) over the tiles that rectangle touches -- which is 0 wherever
// a pixel's depth is outside the sensor range.  The per-voxel arithmetic
// rounds far below these margins, so its test takes the free-space branch
// for every voxel of such a block, and integration skips the per-voxel
// projection (colours are zero: no RGB).  Blocks whose rectangle covers
// more than 16 coarse tiles (close to the camera) take the per-voxel test.
__device__ inline bool free_space_block(unsigned long long key, const DTsdf& t, const DSensor& s,
                                        const M4f& invT, const unsigned* __restrict__ ftile,
                                        int tiles_x, int tiles_y) {
  const float vs = t.vs, e = 7.0f * vs;
  const float ox = (float)key_x(key) * vs * (float)kBlockSize,
              oy = (float)key_y(key) * vs * (float)kBlockSize,
              oz = (float)key_z(key) * vs * (float)kBlockSize;
  float u0 = 3.0e38f, u1 = -3.0e38f, v0 = 3.0e38f, v1 = -3.0e38f, dm = 0.0f;
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    const F3 c = xform(invT, f3(ox + ((k & 1) ? e : 0.0f), oy + ((k & 2) ? e : 0.0f),
                                oz + ((k & 4) ? e : 0.0f)));
    if (!(c.z > 0.01f)) return false;
    const float u = s.fx * c.x / c.z + s.cx, w = s.fy * c.y / c.z + s.cy;
    u0 = fminf(u0, u);
    u1 = fmaxf(u1, u);
    v0 = fminf(v0, w);
    v1 = fmaxf(v1, w);
    dm = fmaxf(dm, norm3(c));
  }
  if (!(u0 >= 1.0f && v0 >= 1.0f && u1 <= (float)(s.cols - 2) && v1 <= (float)(s.rows - 2)))
    return false;
  const int x0 = (int)floorf(u0) - 1, x1 = (int)ceilf(u1) + 1;
  const int y0 = (int)floorf(v0) - 1, y1 = (int)ceilf(v1) + 1;
  if (x0 < 0 || y0 < 0 || x1 >= s.cols || y1 >= s.rows) return false;
  int tx0 = x0 / kRbTile, tx1 = x1 / kRbTile, ty0 = y0 / kRbTile, ty1 = y1 / kRbTile;
  const unsigned* m = ftile;
  int tw = tiles_x;
  if ((tx1 - tx0 + 1) * (ty1 - ty0 + 1) > 16) {
    m = ftile + tiles_x * tiles_y;
    tw = (tiles_x + kRbCoarse - 1) / kRbCoarse;
    tx0 /= kRbCoarse;
    tx1 /= kRbCoarse;
    ty0 /= kRbCoarse;
    ty1 /= kRbCoarse;
    if ((tx1 - tx0 + 1) * (ty1 - ty0 + 1) > 16) return false;
  }
  unsigned mn = 0xffffffffu;
  for (int ty = ty0; ty <= ty1; ++ty)
    for (int tx = tx0; tx <= tx1; ++tx) mn = min(mn, __ldg(m + ty * tw + tx));
  return dm * (1.0f + 1e-5f) + 1e-5f < __uint_as_float(mn);
}

// Every session's visible blocks appended to one batch-wide list of
// (session, heap index), so integration balances across sessions; the
// session index carries kVisFree for free-space blocks.
__global__ void fused_visible_kernel(const SessDev* __restrict__ tab, int2* __restrict__ gvis,
                                     int* __restrict__ gcount) {
  const SessDev& S = tab[blockIdx.z];
  const VolumeDev& v = S.vol;
  __shared__ M4f invT;
  if (threadIdx.x < 16) invT.m[threadIdx.x] = S.pose->invf[threadIdx.x];
  __syncthreads();
  int n = v.cnt->nalloc;
  if (n > v.t.num_blocks) n = v.t.num_blocks;
  const int lane = threadIdx.x & 31;
  for (int base = blockIdx.x * blockDim.x; base < n; base += gridDim.x * blockDim.x) {
    int i = base + threadIdx.x;
    bool vis = false;
    if (i < n) {
      const unsigned long long key = v.block_keys[i];
      vis = block_visible(key, v.t, S.ls[0], invT);
      // every allocated block (visible or not) enters the ray-start bound
      if (S.rbound) bound_block(key, v.t, S.ls[0], invT, S.rbound, S.rb_tx, S.rb_ty, v.t.band, true);
    }
    bool fr = false;
    if (vis && S.ftile && !v.t.band && !*S.rgb_flag)
      fr = free_space_block(v.block_keys[i], v.t, S.ls[0], invT, S.ftile, S.rb_tx, S.rb_ty);
    unsigned m = __ballot_sync(0xffffffffu, vis);
    int off = 0;
    if (lane == 0 && m) {
      atomicAdd(&v.cnt->visible, __popc(m));
      off = atomicAdd(gcount, __popc(m));
    }
    off = __shfl_sync(0xffffffffu, off, 0);
    if (vis)
      gvis[off + __popc(m & ((1u << lane) - 1))] =
          make_int2((int)blockIdx.z | (fr ? kVisFree : 0), i);
  }
}

// The near ray bound of mixed carving sessions, after integration.  A
// sample whose cell and centre voxel lie only in blocks without observed
// non-saturated voxels (unallocated, unobserved or saturated: f16 value 1)
// steps the truncation distance, or the interpolation of saturated values
// -- the truncation up to the rounding of the weights, never ending the
// march (free_ok) -- as the free-cell shortcut does; so the near bound of a
// tile is the nearest depth of the boxes of the blocks that hold such
// voxels (VolumeDev::nonsat > 0), widened as bound_block widens every box.
__global__ void fused_surface_bound_kernel(const SessDev* __restrict__ tab) {
  const SessDev& S = tab[blockIdx.z];
  const VolumeDev& v = S.vol;
  if (!S.rbound || !v.nonsat || !v.free_ok || v.t.band) return;
  __shared__ M4f invT;
  if (threadIdx.x < 16) invT.m[threadIdx.x] = S.pose->invf[threadIdx.x];
  __syncthreads();
  int n = v.cnt->nalloc;
  if (n > v.t.num_blocks) n = v.t.num_blocks;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    if (v.nonsat[i] > 0)
      bound_block(v.block_keys[i], v.t, S.ls[0], invT, S.rbound, S.rb_tx, S.rb_ty, true, false);
}

// ------------------------------------------------------------ integration
// IntegrateScanKernel voxel loop (tsdf.cu:301-341) + Voxel::mergeVoxel
// (geom_Types.h:79-103) for voxel 'lin' of block 'ptr'.  The voxel updated
// is the thread's own: the reference's camera->world round trip through
// UpdateVoxel lands on the same voxel (the oracle checks this).
// FAST (band sessions, whose allocation already departs from the
// reference's): fused multiply-adds and hardware-approximate division and
// square root throughout.
__device__ inline F3 xform_fma(const M4f& T, F3 v) {
  return f3(__fmaf_rn(T.m[0], v.x, __fmaf_rn(T.m[1], v.y, __fmaf_rn(T.m[2], v.z, T.m[3]))),
            __fmaf_rn(T.m[4], v.x, __fmaf_rn(T.m[5], v.y, __fmaf_rn(T.m[6], v.z, T.m[7]))),
            __fmaf_rn(T.m[8], v.x, __fmaf_rn(T.m[9], v.y, __fmaf_rn(T.m[10], v.z, T.m[11]))));
}
__device__ inline float norm3_fast(F3 v) {
  const float q = __fmaf_rn(v.x, v.x, __fmaf_rn(v.y, v.y, v.z * v.z));
  return q > 0.0f ? q * rsqrtf(q) : 0.0f;
}

// Whether this frame updates voxel 'lin' of block 'ptr', and with which
// sdf and colour (the per-voxel test of IntegrateScanKernel).
// The world position of a block's first voxel (its key times the block's
// extent, as the reference computes it per voxel).
__device__ inline F3 block_origin(const VolumeDev& v, int ptr) {
  const float vs = v.t.vs;
  const unsigned long long key = v.block_keys[ptr];
  return f3((float)key_x(key) * vs * (float)kBlockSize, (float)key_y(key) * vs * (float)kBlockSize,
            (float)key_z(key) * vs * (float)kBlockSize);
}

// Voxel::mergeVoxelColor (geom_Types.h:87-91) of an observation of weight 1
// into a channel of weight w: the byte of (old * w + obs) / (w + 1) in
// FP32.  The numerator is an integer below 2^24 (exact in FP32), and the
// rounded quotient truncates to the floor of the exact one: below an
// integer k <= 255 the quotient is at least 1 / (w + 1) >= 2^-16 away,
// more than the half ulp (at most 2^-17) it would take to round up to k.
// So the integer quotient gives the same byte; it comes from an estimate
// by the reciprocal rcp_d of w + 1 (relative error a few 2^-24, under one
// unit off) corrected by one step.
__device__ inline uint8_t colour_merge(unsigned old, unsigned obs, unsigned w, float rcp_d) {
  const int n = (int)(old * w + obs), d = (int)w + 1;
  int q = __float2int_rz(__int2float_rn(n) * rcp_d);
  const int r = n - q * d;
  q += (int)(r >= d) - (int)(r < 0);
  return (uint8_t)q;
}

template <bool FAST>
__device__ inline bool observe_voxel(const VolumeDev& v, const float* __restrict__ depth,
                                     const float* __restrict__ sdist,
                                     const uint8_t* __restrict__ rgb, const DSensor& s,
                                     const M4f& invT, F3 position, int lin, float& sdf,
                                     uint8_t& c0, uint8_t& c1, uint8_t& c2) {
  const DTsdf& t = v.t;
  const float vs = t.vs;
  const int bx = lin >> 6, by = (lin >> 3) & 7, bz = lin & 7;
  F3 vp = f3(position.x + (float)bx * vs, position.y + (float)by * vs,
             position.z + (float)bz * vs);
  // pixel, depth gate and band decide which voxels a frame updates: IEEE
  // arithmetic in the FP32 and mixed forms, so that the mixed form's
  // weights stay exact
  int px, py;
  float sd, vd, d;
  if (FAST) {
    vp = xform_fma(invT, vp);
    if (!(vp.z > 0.0f)) return false;
    const float rz = __fdividef(1.0f, vp.z);
    const float xf = __fmaf_rn(s.fx * vp.x, rz, s.cx), yf = __fmaf_rn(s.fy * vp.y, rz, s.cy);
    if (!(fabsf(xf) < 2e9f) || !(fabsf(yf) < 2e9f)) return false;
    px = (int)roundf(xf);
    py = (int)roundf(yf);
    if (!(px >= 0 && py >= 0 && px < s.cols && py < s.rows)) return false;
    d = __ldg(depth + py * s.cols + px);
    if (d < t.dmin) return false;
    if (d > t.dmax) return false;
    const F3 p3 = f3(__fdividef(((float)px - s.cx) * d, s.fx),
                     __fdividef(((float)py - s.cy) * d, s.fy), d);
    sd = norm3_fast(p3);
    vd = norm3_fast(vp);
  } else {
    vp = xform(invT, vp);
    if (!project(vp, s, &px, &py)) return false;
    if (!(px >= 0 && py >= 0 && px < s.cols && py < s.rows)) return false;
    d = __ldg(depth + py * s.cols + px);
    if (d < t.dmin) return false;
    if (d > t.dmax) return false;
    sd = __ldg(sdist + py * s.cols + px);  // norm3(point3d_uv(px, py, d, s))
    vd = norm3(vp);
  }
  const int idx = py * s.cols + px;
  if (vd > sd - t.trunc && vd < sd + t.trunc && d < t.dmax) sdf = sd - vd;
  else if (vd < sd - t.trunc) sdf = t.trunc;
  else return false;
  c0 = c1 = c2 = 0;
  if (rgb) {
    c0 = __ldg(rgb + 3 * (size_t)idx);
    c1 = __ldg(rgb + 3 * (size_t)idx + 1);
    c2 = __ldg(rgb + 3 * (size_t)idx + 2);
  }
  return true;
}

// Voxel::mergeVoxel (geom_Types.h:79-103) of one observation into voxel vi.
// Returns the change of the block's count of observed, non-saturated voxels
// (-1, 0 or +1) that the update makes (FP16 form; the FP32 form keeps no
// free-space summaries and returns 0).
template <bool FP16>
__device__ inline int merge_voxel(const VolumeDev& v, size_t vi, float sdf, bool has_rgb,
                                  uint8_t c0, uint8_t c1, uint8_t c2) {
  const DTsdf& t = v.t;
  if (FP16) {
    // mixed form: the same FP32 merge, stored as f16 sdf / truncation
    // (|value| <= 1, free space exactly 1) and a u16 weight
    const unsigned raw = v.vox16[vi];
    const float osdf =
        __half2float(__ushort_as_half((unsigned short)(raw & 0xffffu))) * t.trunc;
    const int w = (int)(raw >> 16);
    const float fw = (float)w;
    const float nsdf = __fdividef(osdf * fw + sdf, fw + 1.0f);
    int nw = w + 1;
    if (nw > t.max_w) nw = t.max_w;
    const unsigned short nh = __half_as_ushort(__float2half_rn(__fdividef(nsdf, t.trunc)));
    v.vox16[vi] = (unsigned)nh | ((unsigned)nw << 16);
    if (v.colors) {
      uchar4 c = v.colors[vi];
      // colour exactly as the FP32 form (truncated to bytes)
      const float rd = __fdividef(1.0f, fw + 1.0f);
      c.x = colour_merge(c.x, c0, (unsigned)w, rd);
      c.y = colour_merge(c.y, c1, (unsigned)w, rd);
      c.z = colour_merge(c.z, c2, (unsigned)w, rd);
      v.colors[vi] = c;
    }
    // saturated: f16 value exactly 1 (free space); unobserved before
    const bool was = w == 0 || (raw & 0xffffu) == 0x3C00u, now = nh == 0x3C00u;
    return (int)was - (int)now;
  }
  dyn_voxel* vox = v.voxels + vi;
  uint2 raw = *reinterpret_cast<const uint2*>(vox);
  uint8_t r0 = raw.x & 0xff, r1 = (raw.x >> 8) & 0xff, r2 = (raw.x >> 16) & 0xff,
          w = raw.x >> 24;
  float osdf = __uint_as_float(raw.y);
  float fw = (float)w;
  float nsdf = (osdf * fw + sdf * 1.0f) / (fw + 1.0f);
  // colour merge (geom_Types.h:87-91); a zero colour merged with a zero
  // colour stays exactly zero, so depth-only frames skip the divisions
  if (has_rgb || (raw.x & 0x00ffffffu)) {
    const float rd = __fdividef(1.0f, fw + 1.0f);
    r0 = colour_merge(r0, c0, w, rd);
    r1 = colour_merge(r1, c1, w, rd);
    r2 = colour_merge(r2, c2, w, rd);
  }
  int nw = (uint8_t)(w + 1);
  if (nw > t.max_w) nw = t.max_w;
  uint2 out;
  out.x = (unsigned)r0 | ((unsigned)r1 << 8) | ((unsigned)r2 << 16) | ((unsigned)nw << 24);
  out.y = __float_as_uint(nsdf);
  *reinterpret_cast<uint2*>(vox) = out;
  return 0;
}

// IntegrateScanKernel voxel loop (tsdf.cu:301-341) + Voxel::mergeVoxel for
// voxel 'lin' of block 'ptr': the nonsat change (merge_voxel), 0 when the
// voxel is not updated.
template <bool FP16, bool FAST>
__device__ inline int integrate_voxel(const VolumeDev& v, const float* __restrict__ depth,
                                       const float* __restrict__ sdist,
                                       const uint8_t* __restrict__ rgb, const DSensor& s,
                                       const M4f& invT, F3 origin, int ptr, int lin) {
  float sdf;
  uint8_t c0, c1, c2;
  if (!observe_voxel<FAST>(v, depth, sdist, rgb, s, invT, origin, lin, sdf, c0, c1, c2)) return 0;
  return merge_voxel<FP16>(v, (size_t)ptr * kBlockVox + lin, sdf, rgb != nullptr, c0, c1, c2);
}

// the batch-wide visible list: each item (session, block) by one CTA
__global__ void __launch_bounds__(kBlockVox)
    fused_integrate_kernel(const SessDev* __restrict__ tab, const int2* __restrict__ gvis,
                           const int* __restrict__ gcount) {
  __shared__ M4f invT;
  __shared__ int cur_s;
  __shared__ float org[2][3];  // the block's origin, by iteration parity
  const int n = *gcount;
  if (threadIdx.x == 0) cur_s = -1;
  __syncthreads();
  int par = 0;
  for (int b = blockIdx.x; b < n; b += gridDim.x, par ^= 1) {
    const int2 entry = gvis[b];
    const int2 item = make_int2(entry.x & ~kVisFree, entry.y);
    if (item.x != cur_s) {  // uniform across the CTA
      __syncthreads();
      if (threadIdx.x < 16) invT.m[threadIdx.x] = tab[item.x].pose->invf[threadIdx.x];
      if (threadIdx.x == 0) cur_s = item.x;
      __syncthreads();
    }
    const SessDev& S = tab[item.x];
    // one thread computes the block's origin (the same expression every
    // voxel would evaluate); the barrier also keeps every thread within one
    // iteration of the others, so the other parity's slot is free
    if (threadIdx.x == 0 && !(entry.x & kVisFree)) {
      const F3 o = block_origin(S.vol, item.y);
      org[par][0] = o.x;
      org[par][1] = o.y;
      org[par][2] = o.z;
    }
    __syncthreads();
    const F3 origin = f3(org[par][0], org[par][1], org[par][2]);
    const uint8_t* rgb = *S.rgb_flag ? S.rgb : nullptr;
    int d;
    if (entry.x & kVisFree) {  // a free-space block: every voxel's sdf is the truncation
      const size_t vi = (size_t)item.y * kBlockVox + threadIdx.x;
      d = S.vol.fp16 ? merge_voxel<true>(S.vol, vi, S.vol.t.trunc, false, 0, 0, 0)
                     : merge_voxel<false>(S.vol, vi, S.vol.t.trunc, false, 0, 0, 0);
    } else if (!S.vol.fp16)
      d = integrate_voxel<false, false>(S.vol, S.raw, S.sdist, rgb, S.ls[0], invT, origin,
                                        item.y, threadIdx.x);
    else if (S.vol.t.band)
      d = integrate_voxel<true, true>(S.vol, S.raw, S.sdist, rgb, S.ls[0], invT, origin,
                                      item.y, threadIdx.x);
    else
      d = integrate_voxel<true, false>(S.vol, S.raw, S.sdist, rgb, S.ls[0], invT, origin,
                                       item.y, threadIdx.x);
    // the block's non-saturated count follows its voxels exactly: each warp
    // adds its voxels' changes (mixed sessions only; most warps change
    // nothing, and no barrier holds the CTA's warps together)
    if (S.vol.nonsat) {
      const unsigned up = __ballot_sync(0xffffffffu, d > 0), dn = __ballot_sync(0xffffffffu, d < 0);
      const int net = __popc(up) - __popc(dn);
      if ((threadIdx.x & 31) == 0 && net != 0) atomicAdd(S.vol.nonsat + item.y, net);
    }
  }
}

// Free-cell flags of the visible blocks (after their integration): a block's
// flag is set when it and its seven upper neighbours (+x, +y, +z and their
// combinations; missing ones count as free) hold no observed non-saturated
// voxel.  A visible block that holds one clears the flags of its seven lower
// neighbours, whose cells read it; those may be blocks that are not visible
// this frame.  Both writers of a flag agree: a block whose flag a neighbour
// clears computes 0 for itself.  Flags are only ever set here, for visible
// blocks, so a flag is never 1 where a cell of its block reads a
// non-saturated voxel.
__global__ void fused_free_cells_kernel(const SessDev* __restrict__ tab,
                                        const int2* __restrict__ gvis,
                                        const int* __restrict__ gcount) {
  const int n = *gcount;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int2 entry = gvis[i];
    const int2 item = make_int2(entry.x & ~kVisFree, entry.y);
    const VolumeDev& v = tab[item.x].vol;
    if (!v.freecell) continue;
    const unsigned long long key = v.block_keys[item.y];
    const int x = key_x(key), y = key_y(key), z = key_z(key);
    const bool own = v.nonsat[item.y] == 0;
    bool free = own && v.free_ok;
#pragma unroll
    for (int k = 1; k < 8; ++k) {
      const int dx = k & 1, dy = (k >> 1) & 1, dz = (k >> 2) & 1;
      if (free) {
        const int p = find_block(v.entries, v.t, x + dx, y + dy, z + dz);
        if (p >= 0 && v.nonsat[p] != 0) free = false;
      }
      if (!own) {
        const int q = find_block(v.entries, v.t, x - dx, y - dy, z - dz);
        if (q >= 0) v.freecell[q] = 0;
      }
    }
    v.freecell[item.y] = free ? 1 : 0;
  }
}

// ------------------------------------------------------------ raycast
struct VoxelSample {
  float sdf;
  float r, g, b;
  int w;
};

struct BlockCache {
  int x, y, z;
  int ptr;
};
// the cache of the mixed march's cell blocks, with the block's free-cell flag
struct FreeCache : BlockCache {
  int free;
};

// voxel_index, blk_of and loc_of (WorldToGlobalVoxelHashing / WorldToBlock /
// WorldToLocalVoxel) are in common.cuh.

// tsdfVolume::GetVoxel, tsdf.cu:227-239, for a voxel already resolved to
// (block, local index); a one-block lookup cache skips repeated bucket
// scans of the same block.
__device__ inline int block_ptr(const VolumeDev& v, int bx, int by, int bz, BlockCache& bc) {
  if (bx != bc.x || by != bc.y || bz != bc.z) {
    bc.x = bx;
    bc.y = by;
    bc.z = bz;
    bc.ptr = find_block(v.entries, v.t, bx, by, bz);
  }
  return bc.ptr;
}
__device__ inline uint2 load_voxel(const VolumeDev& v, int ptr, int lin) {
  if (ptr < 0) return make_uint2(0u, 0u);
  return __ldg(reinterpret_cast<const uint2*>(v.voxels + (size_t)ptr * kBlockVox + lin));
}
__device__ inline int lin_of(int gx, int gy, int gz) {
  return (loc_of(gx) << 6) | (loc_of(gy) << 3) | loc_of(gz);
}

__device__ inline uint2 get_voxel(const VolumeDev& v, F3 pos, float inv_vs, BlockCache& bc) {
  const float vs = v.t.vs;
  int gx = voxel_index(pos.x, vs, inv_vs), gy = voxel_index(pos.y, vs, inv_vs),
      gz = voxel_index(pos.z, vs, inv_vs);
  return load_voxel(v, block_ptr(v, blk_of(gx), blk_of(gy), blk_of(gz), bc), lin_of(gx, gy, gz));
}

__device__ inline int vw(uint2 r) { return (int)(r.x >> 24); }
__device__ inline float vsdf(uint2 r) { return __uint_as_float(r.y); }

// The heap indices of the (up to eight) blocks a 2x2x2 cell touches: the
// cell's low corner is in block b, its high corner steps into b + 1 along
// the axes where the low corner is the block's last voxel (cx, cy, cz).
// Each distinct block is resolved once (the low one through the ray's
// cache); named fields, so that corner selection folds to a few selects.
struct CellBlocks {
  int p0, px, py, pz, pxy, pxz, pyz, pxyz;
};
__device__ inline void cell_blocks(const VolumeDev& v, int bx, int by, int bz, bool cx, bool cy,
                                   bool cz, BlockCache& bc, CellBlocks& cb) {
  const DTsdf& t = v.t;
  cb.p0 = block_ptr(v, bx, by, bz, bc);
  cb.px = cx ? find_block(v.entries, t, bx + 1, by, bz) : -1;
  cb.py = cy ? find_block(v.entries, t, bx, by + 1, bz) : -1;
  cb.pz = cz ? find_block(v.entries, t, bx, by, bz + 1) : -1;
  cb.pxy = (cx && cy) ? find_block(v.entries, t, bx + 1, by + 1, bz) : -1;
  cb.pxz = (cx && cz) ? find_block(v.entries, t, bx + 1, by, bz + 1) : -1;
  cb.pyz = (cy && cz) ? find_block(v.entries, t, bx, by + 1, bz + 1) : -1;
  cb.pxyz = (cx && cy && cz) ? find_block(v.entries, t, bx + 1, by + 1, bz + 1) : -1;
}
// the block of corner (ox, oy, oz) (compile-time offsets after unrolling)
__device__ inline int corner_block(const CellBlocks& cb, bool cx, bool cy, bool cz, int ox,
                                   int oy, int oz) {
  const bool kx = ox && cx, ky = oy && cy, kz = oz && cz;
  return kx ? (ky ? (kz ? cb.pxyz : cb.pxy) : (kz ? cb.pxz : cb.px))
            : (ky ? (kz ? cb.pyz : cb.py) : (kz ? cb.pz : cb.p0));
}

// tsdfVolume::GetInterpolatedVoxel, tsdf.cu:47-175.  The eight corners are
// pos_dual + {0, vs} per axis, so each axis has two coordinate values: they
// are resolved once (six index computations instead of twenty-four) and
// combined per corner; every corner still gets exactly the reference's
// float coordinate.  When the 2x2x2 corners lie in one block (the common
// case) the block is resolved once.  Corners are summed in the reference's
// order.  COLOR false skips the colour sums (the marching loop only reads
// sdf and weight).
template <bool COLOR>
__device__ inline VoxelSample get_interpolated(const VolumeDev& v, F3 position, float inv_vs,
                                               BlockCache& bc) {
  VoxelSample out;
  uint2 v0 = get_voxel(v, position, inv_vs, bc);
  out.w = vw(v0);
  if (out.w == 0) {
    out.sdf = vsdf(v0);
    out.r = (float)(v0.x & 0xff);
    out.g = (float)((v0.x >> 8) & 0xff);
    out.b = (float)((v0.x >> 16) & 0xff);
    return out;
  }
  const float vs = v.t.vs;
  F3 pos_dual = position - f3(vs / 2.0f, vs / 2.0f, vs / 2.0f);
  const float inv = 1.0f / vs;
  F3 vp = position * inv;
  F3 wt = f3(vp.x - floorf(vp.x), vp.y - floorf(vp.y), vp.z - floorf(vp.z));
  int gx[2], gy[2], gz[2];
  voxel_index_pair(pos_dual.x + 0.0f, pos_dual.x + vs, vs, inv_vs, gx[0], gx[1]);
  voxel_index_pair(pos_dual.y + 0.0f, pos_dual.y + vs, vs, inv_vs, gy[0], gy[1]);
  voxel_index_pair(pos_dual.z + 0.0f, pos_dual.z + vs, vs, inv_vs, gz[0], gz[1]);
  // the high corners lie in the next block along an axis where they cross
  const bool cx = blk_of(gx[1]) != blk_of(gx[0]), cy = blk_of(gy[1]) != blk_of(gy[0]),
             cz = blk_of(gz[1]) != blk_of(gz[0]);
  const int off[8][3] = {{0, 0, 0}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1},
                         {1, 1, 0}, {0, 1, 1}, {1, 0, 1}, {1, 1, 1}};
  // the eight corner voxels: one block and constant strides from the low
  // corner in the common case (no axis crosses a block boundary and each
  // high index is the low one + 1), else each corner's block and index
  uint2 cv[8];
  if (!(cx || cy || cz) && gx[1] - gx[0] == 1 && gy[1] - gy[0] == 1 && gz[1] - gz[0] == 1) {
    const int p0 = block_ptr(v, blk_of(gx[0]), blk_of(gy[0]), blk_of(gz[0]), bc);
    const uint2* base = reinterpret_cast<const uint2*>(v.voxels + (size_t)(p0 < 0 ? 0 : p0) *
                                                                      kBlockVox +
                                                       lin_of(gx[0], gy[0], gz[0]));
#pragma unroll
    for (int k = 0; k < 8; ++k)
      cv[k] = p0 < 0 ? make_uint2(0u, 0u)
                     : __ldg(base + (off[k][0] << 6) + (off[k][1] << 3) + off[k][2]);
  } else {
    CellBlocks cells;
    cell_blocks(v, blk_of(gx[0]), blk_of(gy[0]), blk_of(gz[0]), cx, cy, cz, bc, cells);
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      const int ox = off[k][0], oy = off[k][1], oz = off[k][2];
      cv[k] = load_voxel(v, corner_block(cells, cx, cy, cz, ox, oy, oz),
                         lin_of(gx[ox], gy[oy], gz[oz]));
    }
  }
  float dist = 0.0f;
  float cr = 0.0f, cg = 0.0f, cb = 0.0f;
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    const int ox = off[k][0], oy = off[k][1], oz = off[k][2];
    const uint2 vv = cv[k];
    uint2 src = (vw(vv) == 0) ? v0 : vv;
    float a = ox ? wt.x : 1.0f - wt.x;
    float b = oy ? wt.y : 1.0f - wt.y;
    float c = oz ? wt.z : 1.0f - wt.z;
    float coef = a * b * c;
    dist += coef * vsdf(src);
    if (COLOR) {
      cr = cr + (float)(src.x & 0xff) * coef;
      cg = cg + (float)((src.x >> 8) & 0xff) * coef;
      cb = cb + (float)((src.x >> 16) & 0xff) * coef;
    }
  }
  out.sdf = dist;
  out.r = cr;
  out.g = cg;
  out.b = cb;
  return out;
}

constexpr int kRayTX = 16, kRayTY = 16;


// tsdfVolume raycast (tsdf.cu:471-526) of pixel (x, y) from camera pose T:
// march from 0 by the interpolated sdf (a truncation where unobserved) until
// the sdf drops under a voxel or the depth passes max_sensor_depth; then the
// interpolated colour at the hit.  Beyond the near distance, samples before
// skip_to or after skip_far (the tile's ray depth bounds: no allocated block
// there) step by the truncation without a lookup -- what the lookup would
// have returned.  Returns true when the march hit the step cap.
__device__ inline bool raycast_exact_px(const VolumeDev& v, const DSensor& s, const M4f& T, int x,
                                        int y, float skip_to, float skip_far,
                                        float* __restrict__ depth_out,
                                        uint8_t* __restrict__ rgb_out) {
  const int i = y * s.cols + x;
  const DTsdf& t = v.t;
  const float inv_vs = 1.0f / t.vs;
  // getPoint3d (utils.h:104-112) with the pixel's (u - cx), (v - cy) hoisted
  const float ax = (float)x - s.cx, ay = (float)y - s.cy;
  BlockCache bc;
  bc.x = bc.y = bc.z = 0x7fffffff;
  bc.ptr = -1;
  float cur = 0.0f;
  int steps = 0;
  bool over = false;
  const float znear = ray_near(t);
  while (cur < t.dmax) {
    if (steps++ >= t.rc_cap) {
      over = true;
      break;
    }
    if (cur >= znear && (cur < skip_to || cur > skip_far)) {  // no allocated block here
      cur += t.trunc;
      continue;
    }
    F3 pc = f3(ax * cur / s.fx, ay * cur / s.fy, cur);
    F3 point = xform(T, pc);
    VoxelSample vx = get_interpolated<false>(v, point, inv_vs, bc);
    if (vx.w == 0) cur += t.trunc;
    else cur += vx.sdf;
    if (vx.w != 0 && vx.sdf < t.vs) break;
  }
  depth_out[i] = cur;
  if (rgb_out) {
    uint8_t r = 0, g = 0, b = 0;
    if (cur < t.dmax) {
      F3 point = xform(T, point3d_uv(x, y, cur, s));
      VoxelSample vx = get_interpolated<true>(v, point, inv_vs, bc);
      r = (uint8_t)vx.r;
      g = (uint8_t)vx.g;
      b = (uint8_t)vx.b;
    }
    rgb_out[3 * (size_t)i] = r;
    rgb_out[3 * (size_t)i + 1] = g;
    rgb_out[3 * (size_t)i + 2] = b;
  }
  return over;
}


// ------------------------------------------------------------ mixed-precision raycast
// The mixed forms' march: tsdfVolume::GenerateDepthKernel /
// GenerateRgbKernel (tsdf.cu:471-526) with GetInterpolatedVoxel
// (tsdf.cu:47-175) in voxel units: the sample at depth z is q = o + z * d
// (o the camera centre, d the pixel's ray direction per unit depth, both
// divided by the voxel size) by fused multiply-adds.  The reference's step
// rule is kept: from 0, step by the interpolated sdf where the sample's
// voxel (floor(q + 0.5), the reference's rounding of p / vs up to ties) is
// observed, by the truncation distance where it is not, until the sdf drops
// under a voxel or the depth passes max_sensor_depth.  The trilinear cell
// is floor(q) .. floor(q) + 1 with weights q - floor(q) (the reference's
// rounded p - vs/2 and p + vs/2 and its weights from p / vs); unobserved
// corners take the centre voxel's value.  Two shortcuts give what the full
// sample would give:
//  * beyond the near distance, a sample before the tile's near bound or
//    after its far bound (no allocated block there) steps by the truncation
//    without a lookup;
//  * a sample whose cell lies in a free-cell block (every voxel the cell can
//    read is unobserved or saturated, VolumeDev::freecell) steps by the
//    truncation distance without reading voxels: the reference's step there
//    is the truncation (unobserved centre) or the interpolation of
//    saturated values (f16 value exactly 1), which is the truncation up to
//    the rounding of the weights, and never ends the march (free_ok).
// The FP32 drop-in keeps raycast_exact_px: its targets decide the tracked
// poses, whose bar against the reference (1e-4 m / 1e-4 rad per frame)
// holds only with the reference's own rounding in the march -- with this
// march in the FP32 form, tracked poses left that bar after six to nine
// frames on the parity sequences, through the solver's discrete
// convergence test (an extra or a missing iteration moves a pose by up to
// the 1e-3 increment threshold).
template <bool FP16>
struct Vox;
template <>
struct Vox<true> {
  using raw_t = unsigned;
  static __device__ raw_t load(const VolumeDev& v, int ptr, int lin) {
    return ptr < 0 ? 0u : __ldg(v.vox16 + (size_t)ptr * kBlockVox + lin);
  }
  static __device__ int w(raw_t r) { return (int)(r >> 16); }
  static __device__ float val(raw_t r) {
    return __half2float(__ushort_as_half((unsigned short)(r & 0xffffu)));
  }
  static __device__ float unit(const DTsdf& t) { return t.trunc; }
  static __device__ uchar4 color(const VolumeDev& v, raw_t, int ptr, int lin) {
    return (v.colors && ptr >= 0) ? v.colors[(size_t)ptr * kBlockVox + lin]
                                  : make_uchar4(0, 0, 0, 0);
  }
};

// The interpolated sample at q (voxel units) whose centre voxel raw0 (heap
// index ptr0, local index lin0) is observed.  Sums by fused multiply-adds
// in the reference's corner order.
template <bool FP16, bool COLOR>
__device__ inline VoxelSample interp(const VolumeDev& v, F3 q, typename Vox<FP16>::raw_t raw0,
                                     int ptr0, int lin0, BlockCache& bc) {
  using V = Vox<FP16>;
  VoxelSample out;
  const float fx = floorf(q.x), fy = floorf(q.y), fz = floorf(q.z);
  const float wx = q.x - fx, wy = q.y - fy, wz = q.z - fz;
  const int gx = (int)fx, gy = (int)fy, gz = (int)fz;
  const int lx = gx & 7, ly = gy & 7, lz = gz & 7;
  const bool cx = lx == 7, cy = ly == 7, cz = lz == 7;
  CellBlocks cb;
  cell_blocks(v, gx >> 3, gy >> 3, gz >> 3, cx, cy, cz, bc, cb);
  // local index of the low corner and the steps to the high ones (wrapping
  // into the next block where the cell crosses)
  const int base = (lx << 6) | (ly << 3) | lz;
  const int dx = cx ? -448 : 64, dy = cy ? -56 : 8, dz = cz ? -7 : 1;
  const uchar4 c0 = COLOR ? V::color(v, raw0, ptr0, lin0) : make_uchar4(0, 0, 0, 0);
  const float n0 = V::val(raw0);
  const float ax[2] = {1.0f - wx, wx}, ay[2] = {1.0f - wy, wy}, az[2] = {1.0f - wz, wz};
  float dist = 0.0f, cr = 0.0f, cg = 0.0f, cbl = 0.0f;
  const int off[8][3] = {{0, 0, 0}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1},
                         {1, 1, 0}, {0, 1, 1}, {1, 0, 1}, {1, 1, 1}};
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    const int ox = off[k][0], oy = off[k][1], oz = off[k][2];
    const int ptr = corner_block(cb, cx, cy, cz, ox, oy, oz);
    const int lin = base + (ox ? dx : 0) + (oy ? dy : 0) + (oz ? dz : 0);
    const typename V::raw_t r = V::load(v, ptr, lin);
    const bool use0 = V::w(r) == 0;
    const float coef = (ax[ox] * ay[oy]) * az[oz];
    dist = __fmaf_rn(coef, use0 ? n0 : V::val(r), dist);
    if (COLOR) {
      const uchar4 cc = use0 ? c0 : V::color(v, r, ptr, lin);
      cr = __fmaf_rn((float)cc.x, coef, cr);
      cg = __fmaf_rn((float)cc.y, coef, cg);
      cbl = __fmaf_rn((float)cc.z, coef, cbl);
    }
  }
  out.sdf = dist * V::unit(v.t);
  out.w = V::w(raw0);
  out.r = cr;
  out.g = cg;
  out.b = cbl;
  return out;
}

// The block of a cell's low corner through the ray's cache, with its
// free-cell flag (0 where no flags are kept).
__device__ inline int cell_block_free(const VolumeDev& v, int bx, int by, int bz, FreeCache& bc,
                                      int* free) {
  if (bx != bc.x || by != bc.y || bz != bc.z) {
    bc.x = bx;
    bc.y = by;
    bc.z = bz;
    bc.ptr = find_block(v.entries, v.t, bx, by, bz);
    bc.free = (v.freecell && bc.ptr >= 0) ? (int)__ldg(v.freecell + bc.ptr) : 0;
  }
  *free = bc.free;
  return bc.ptr;
}

// The march of pixel (x, y) from camera pose T; the colour at the hit when
// rgb_out is given.  skip_to / skip_far: the tile's ray depth bounds.
// Returns true when the march hit the step cap.  FREE: the session keeps
// free-cell flags (mixed form with carving); without them (band sessions)
// the cell's and the centre voxel's blocks share one lookup cache.
template <bool FP16, bool FREE>
__device__ inline bool raycast_px(const VolumeDev& v, const DSensor& s, const M4f& T, int x,
                                  int y, float skip_to, float skip_far,
                                  float* __restrict__ depth_out, uint8_t* __restrict__ rgb_out) {
  using V = Vox<FP16>;
  const int i = y * s.cols + x;
  const DTsdf& t = v.t;
  const float inv_vs = 1.0f / t.vs;
  const float axf = ((float)x - s.cx) / s.fx, ayf = ((float)y - s.cy) / s.fy;
  const F3 o = f3(T.m[3] * inv_vs, T.m[7] * inv_vs, T.m[11] * inv_vs);
  const F3 d = f3((T.m[0] * axf + T.m[1] * ayf + T.m[2]) * inv_vs,
                  (T.m[4] * axf + T.m[5] * ayf + T.m[6]) * inv_vs,
                  (T.m[8] * axf + T.m[9] * ayf + T.m[10]) * inv_vs);
  FreeCache bc;   // the cell's low-corner block, with its flag
  BlockCache bc0;  // the centre voxel's block where it is another
  bc.x = bc.y = bc.z = bc0.x = bc0.y = bc0.z = 0x7fffffff;
  bc.ptr = bc0.ptr = -1;
  bc.free = 0;
  float cur = 0.0f;
  int steps = 0;
  bool over = false;
  const float znear = ray_near(t);
  while (cur < t.dmax) {
    if (steps++ >= t.rc_cap) {
      over = true;
      break;
    }
    if (cur >= znear && (cur < skip_to || cur > skip_far)) {  // no allocated block: weight 0
      cur += t.trunc;
      continue;
    }
    const F3 q = f3(__fmaf_rn(cur, d.x, o.x), __fmaf_rn(cur, d.y, o.y), __fmaf_rn(cur, d.z, o.z));
    const float flx = floorf(q.x), fly = floorf(q.y), flz = floorf(q.z);
    if (FREE) {
      int free;
      cell_block_free(v, (int)flx >> 3, (int)fly >> 3, (int)flz >> 3, bc, &free);
      if (free) {  // the interpolated sdf is the truncation distance
        cur += t.trunc;
        continue;
      }
    }
    const int gx = (int)flx + (q.x - flx >= 0.5f), gy = (int)fly + (q.y - fly >= 0.5f),
              gz = (int)flz + (q.z - flz >= 0.5f);
    // the centre voxel's block: mostly the cell's own, already resolved
    const int ptr = !FREE ? block_ptr(v, blk_of(gx), blk_of(gy), blk_of(gz), bc)
                    : (blk_of(gx) == bc.x && blk_of(gy) == bc.y && blk_of(gz) == bc.z)
                        ? bc.ptr
                        : block_ptr(v, blk_of(gx), blk_of(gy), blk_of(gz), bc0);
    const int lin = lin_of(gx, gy, gz);
    const typename V::raw_t raw = V::load(v, ptr, lin);
    if (V::w(raw) == 0) {
      cur += t.trunc;
      continue;
    }
    const VoxelSample vx = interp<FP16, false>(v, q, raw, ptr, lin, bc);
    cur += vx.sdf;
    if (vx.sdf < t.vs) break;
  }
  depth_out[i] = cur;
  if (rgb_out) {
    uint8_t r = 0, g = 0, b = 0;
    if (cur < t.dmax) {
      const F3 q =
          f3(__fmaf_rn(cur, d.x, o.x), __fmaf_rn(cur, d.y, o.y), __fmaf_rn(cur, d.z, o.z));
      const int gx = (int)floorf(q.x + 0.5f), gy = (int)floorf(q.y + 0.5f),
                gz = (int)floorf(q.z + 0.5f);
      const int ptr = block_ptr(v, blk_of(gx), blk_of(gy), blk_of(gz), bc0);
      const int lin = lin_of(gx, gy, gz);
      const typename V::raw_t raw = V::load(v, ptr, lin);
      uchar4 c;
      if (V::w(raw) != 0) {
        const VoxelSample vx = interp<FP16, true>(v, q, raw, ptr, lin, bc);
        c = make_uchar4((uint8_t)vx.r, (uint8_t)vx.g, (uint8_t)vx.b, 0);
      } else {
        c = V::color(v, raw, ptr, lin);  // GetInterpolatedVoxel returns the centre voxel
      }
      r = c.x;
      g = c.y;
      b = c.z;
    }
    rgb_out[3 * (size_t)i] = r;
    rgb_out[3 * (size_t)i + 1] = g;
    rgb_out[3 * (size_t)i + 2] = b;
  }
  return over;
}

// One 16x16 pixel tile (tile bx, by) from pose16 (a float 4x4); warps cover
// 8x4 pixel sub-tiles for coherent rays.  Step-cap overruns are counted.
// The tile is TX x TY pixels (multiples of 8 x 4; TX * TY >= 64).
template <bool MIXED, int TX = kRayTX, int TY = kRayTY>
__device__ inline void raycast_tile(const VolumeDev& v, const DSensor& s,
                                    const float* __restrict__ pose16, float* __restrict__ depth_out,
                                    uint8_t* __restrict__ rgb_out, int bx, int by,
                                    const unsigned* __restrict__ rbound, int tiles_x) {
  static_assert(TX % 8 == 0 && TY % 4 == 0 && TX * TY >= 64, "tile of 8x4 warps");
  __shared__ M4f Ts;
  __shared__ int over;
  const int tid = threadIdx.y * TX + threadIdx.x;
  if (tid < 16) Ts.m[tid] = pose16[tid];
  if (tid == 0) over = 0;
  __syncthreads();
  const M4f T = Ts;  // the pose in registers for the whole march
  const int warp = tid >> 5, lane = tid & 31;
  const int lx = (warp % (TX / 8)) * 8 + (lane & 7);
  const int ly = (warp / (TX / 8)) * 4 + (lane >> 3);
  const int x = bx * TX + lx, y = by * TY + ly;
  if (x < s.cols && y < s.rows) {
    float skip_to = 0.0f, skip_far = 3.402823466e+38f;
    if (rbound) {
      const int tx = x / kRbTile, ty = y / kRbTile;
      const RayBounds B =
          ray_bounds(const_cast<unsigned*>(rbound), tiles_x, (s.rows + kRbTile - 1) / kRbTile);
      const int f = ty * tiles_x + tx, c = (ty / kRbCoarse) * B.cx + tx / kRbCoarse;
      skip_to = fminf(__uint_as_float(B.near8[f]), __uint_as_float(B.near64[c]));
      skip_far = fmaxf(__uint_as_float(B.far8[f]), __uint_as_float(B.far64[c]));
    }
    const bool o = MIXED ? (v.freecell ? raycast_px<true, true>(v, s, T, x, y, skip_to, skip_far,
                                                                 depth_out, rgb_out)
                                       : raycast_px<true, false>(v, s, T, x, y, skip_to,
                                                                  skip_far, depth_out, rgb_out))
                         : raycast_exact_px(v, s, T, x, y, skip_to, skip_far, depth_out, rgb_out);
    if (o) atomicAdd(&over, 1);
  }
  __syncthreads();
  if (tid == 0 && over) atomicAdd(&v.cnt->raycast_overruns, over);
}

template <bool MIXED>
__global__ void __launch_bounds__(kRayTX* kRayTY)
    raycast_kernel(VolumeDev v, DSensor s, const PoseState* __restrict__ ps,
                   const float* __restrict__ pose_override, float* __restrict__ depth_out,
                   uint8_t* __restrict__ rgb_out) {
  raycast_tile<MIXED>(v, s, pose_override ? pose_override : ps->posef, depth_out, rgb_out,
                      blockIdx.x, blockIdx.y, nullptr, 0);
}

// next frame's target of every mode-1 session (blockIdx.z) at its new pose;
// one instantiation per voxel form (sessions of the other form return) and
// per tile shape (every pixel's march is independent of the tiling)
// (at least 1024 threads resident per SM: the march is latency-bound, and
// 4 CTAs of 256 hide more of it than the 3 that 76 registers allow)
template <bool MIXED, int TX, int TY>
__global__ void __launch_bounds__(TX* TY, 1024 / (TX * TY))
    fused_raycast_kernel(const SessDev* __restrict__ tab) {
  const SessDev& S = tab[blockIdx.z];
  if (S.mode != 1 || (S.vol.fp16 != 0) != MIXED) return;
  const DSensor& s = S.ls[0];
  if ((int)blockIdx.x * TX >= s.cols || (int)blockIdx.y * TY >= s.rows) return;
  uint8_t* rgb_out = S.use_color ? S.trgb : nullptr;
  raycast_tile<MIXED, TX, TY>(S.vol, s, S.pose->posef, S.ray, rgb_out, blockIdx.x, blockIdx.y,
                              S.rbound, S.rb_tx);
}

template <int TX, int TY>
void launch_fused_raycast(const SessDev* tab, const BatchShape& b, cudaStream_t st) {
  dim3 grid((b.max_cols + TX - 1) / TX, (b.max_rows + TY - 1) / TY, b.n);
  if (b.fp16_mask & 1) fused_raycast_kernel<false, TX, TY><<<grid, dim3(TX, TY), 0, st>>>(tab);
  if (b.fp16_mask & 2) fused_raycast_kernel<true, TX, TY><<<grid, dim3(TX, TY), 0, st>>>(tab);
}

// per-frame counters of every session (all but nalloc, the heap top) and
// the batch visible list
// (and the ray depth bounds to "no block")
__global__ void fused_reset_counters_kernel(const SessDev* __restrict__ tab,
                                            int* __restrict__ gcount) {
  const SessDev& S = tab[blockIdx.z];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (S.rbound) {
    // near: no block (3.4e38), or 0 where unused; far: no block (0)
    const bool near_used = S.vol.t.band || (S.vol.nonsat && S.vol.free_ok);
    const unsigned nb = near_used ? 0x7f7f7f7fu : 0u;
    const RayBounds B = ray_bounds(S.rbound, S.rb_tx, S.rb_ty);
    if (i < S.rb_tx * S.rb_ty) {
      B.near8[i] = nb;
      B.far8[i] = 0u;
    }
    if (i < B.cx * B.cy) {
      B.near64[i] = nb;
      B.far64[i] = 0u;
    }
  }
  if (S.ftile && i < ((S.rb_tx + kRbCoarse - 1) / kRbCoarse) * ((S.rb_ty + kRbCoarse - 1) / kRbCoarse))
    S.ftile[S.rb_tx * S.rb_ty + i] = 0x7f7f7f7fu;  // coarse free-space tiles: min of none
  if (i != 0) return;
  if (blockIdx.z == 0) *gcount = 0;
  Counters* c = S.vol.cnt;
  c->new_blocks = 0;
  c->bucket_full = 0;
  c->heap_exhausted = 0;
  c->dda_overruns = 0;
  c->raycast_overruns = 0;
  c->visible = 0;
  c->unique_probed = 0;
  c->icp_timeout = 0;
}

__global__ void clear_entries_kernel(Entry* e, size_t n) {
  size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  Entry z;
  z.key = kEmptyKey;
  z.ptr = -1;
  z.stamp = -1;
  e[i] = z;
}

__global__ void block_coords_kernel(VolumeDev v, int n, int* coords) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  unsigned long long k = v.block_keys[i];
  coords[3 * i] = key_x(k);
  coords[3 * i + 1] = key_y(k);
  coords[3 * i + 2] = key_z(k);
}

__global__ void find_blocks_kernel(VolumeDev v, const int* __restrict__ coords, int n,
                                   int* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int p = find_block(v.entries, v.t, coords[3 * i], coords[3 * i + 1], coords[3 * i + 2]);
  out[i] = (p >= 0 && p < v.t.num_blocks) ? p : -1;
}

inline int nblk(long long n, int t) { return (int)((n + t - 1) / t); }

}  // namespace

void launch_volume_clear(const VolumeDev& v, cudaStream_t st) {
  size_t ne = (size_t)v.t.num_buckets * v.t.bucket_size;
  clear_entries_kernel<<<nblk((long long)ne, 256), 256, 0, st>>>(v.entries, ne);
  const size_t nv = (size_t)v.t.num_blocks * kBlockVox;
  if (v.voxels) cudaMemsetAsync(v.voxels, 0, sizeof(dyn_voxel) * nv, st);
  if (v.vox16) cudaMemsetAsync(v.vox16, 0, sizeof(unsigned) * nv, st);
  if (v.colors) cudaMemsetAsync(v.colors, 0, sizeof(uchar4) * nv, st);
  if (v.nonsat) cudaMemsetAsync(v.nonsat, 0, sizeof(int) * (size_t)v.t.num_blocks, st);
  if (v.freecell) cudaMemsetAsync(v.freecell, 0, (size_t)v.t.num_blocks, st);
  cudaMemsetAsync(v.cnt, 0, sizeof(Counters), st);
}

void launch_raycast(const VolumeDev& v, const DSensor& s, const PoseState* ps,
                    const float* pose_override, float* depth_out, uint8_t* rgb_out,
                    cudaStream_t st) {
  dim3 grid(nblk(s.cols, kRayTX), nblk(s.rows, kRayTY));
  if (v.fp16)
    raycast_kernel<true><<<grid, dim3(kRayTX, kRayTY), 0, st>>>(v, s, ps, pose_override,
                                                                depth_out, rgb_out);
  else
    raycast_kernel<false><<<grid, dim3(kRayTX, kRayTY), 0, st>>>(v, s, ps, pose_override,
                                                                 depth_out, rgb_out);
}

void launch_block_coords(const VolumeDev& v, int n, int* coords, cudaStream_t st) {
  if (n > 0) block_coords_kernel<<<nblk(n, 256), 256, 0, st>>>(v, n, coords);
}

void launch_find_blocks(const VolumeDev& v, const int* coords, int n, int* ptr_out,
                        cudaStream_t st) {
  if (n > 0) find_blocks_kernel<<<nblk(n, 256), 256, 0, st>>>(v, coords, n, ptr_out);
}

// ---- fused stages
void fused_reset_counters(const SessDev* tab, const BatchShape& b, cudaStream_t st) {
  fused_reset_counters_kernel<<<dim3(nblk(b.max_rb_tiles, 256), 1, b.n), 256, 0, st>>>(
      tab, b.gcount);
}

void fused_allocate(const SessDev* tab, const BatchShape& b, cudaStream_t st) {
  dim3 grid(nblk(b.max_cols, kAllocT), nblk(b.max_rows, kAllocT), b.n);
  fused_allocate_kernel<<<grid, dim3(kAllocT, kAllocT), 0, st>>>(tab);
}

void fused_visible(const SessDev* tab, const BatchShape& b, cudaStream_t st) {
  // grid-stride over each session's heap; about 600 CTAs in all
  int cap = 592 / b.n;
  if (cap < 8) cap = 8;
  int g = nblk(b.max_blocks, 256);
  if (g > cap) g = cap;
  fused_visible_kernel<<<dim3(g, 1, b.n), 256, 0, st>>>(tab, b.gvis, b.gcount);
}

void fused_integrate(const SessDev* tab, const BatchShape& b, cudaStream_t st) {
  fused_integrate_kernel<<<b.integrate_ctas > 0 ? b.integrate_ctas : 148 * 8, kBlockVox, 0,
                           st>>>(tab, b.gvis, b.gcount);
}

void fused_free_cells(const SessDev* tab, const BatchShape& b, cudaStream_t st) {
  fused_free_cells_kernel<<<148 * 2, 256, 0, st>>>(tab, b.gvis, b.gcount);
  if (b.fp16_mask & 2) {  // mixed sessions: the near ray bound from their summaries
    int cap = 592 / b.n;
    if (cap < 8) cap = 8;
    int g = nblk(b.max_blocks, 256);
    if (g > cap) g = cap;
    fused_surface_bound_kernel<<<dim3(g, 1, b.n), 256, 0, st>>>(tab);
  }
}

void fused_raycast(const SessDev* tab, const BatchShape& b, cudaStream_t st) {
  switch (b.ray_tile) {
    case 1: launch_fused_raycast<32, 8>(tab, b, st); break;
    case 2: launch_fused_raycast<8, 8>(tab, b, st); break;
    default: launch_fused_raycast<16, 16>(tab, b, st); break;
  }
}

}  // namespace dyn

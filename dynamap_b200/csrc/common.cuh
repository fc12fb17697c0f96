// common.cuh -- device-side types and exact-arithmetic helpers shared by the
// kernels of libdynamap_b200.
//
// The whole library is compiled with -fmad=false and IEEE division/sqrt, so
// each float expression below rounds once per operation in source order --
// the rounding of the reference's own expressions (include/utils/utils.h,
// include/math/cuda_math.h, include/math/utils_matrix.h) and of the CPU
// oracle.  That is what makes allocation, integration and raycast
// bit-identical to the oracle.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/dynamap.h"

namespace dyn {

constexpr int kBlockSize = 8;  // voxels per block edge (tsdfParams blockSize)
constexpr int kBlockVox = kBlockSize * kBlockSize * kBlockSize;
constexpr unsigned long long kEmptyKey = ~0ull;
constexpr int kLevels = 4;     // pyramid levels kept (scales 1, 2, 4, 8)

struct DSensor {
  int rows, cols;
  float fx, fy, cx, cy;
};

struct DTsdf {
  float vs;          // voxelSize
  float bsm;         // blockSize * voxelSize (metres), tsdf.cu:437-438
  float trunc;
  float dmin, dmax;  // min/maxSensorDepth
  int num_buckets;
  int nb_mask;       // num_buckets - 1 when a power of two, else -1
  int bucket_size;
  int num_blocks;
  int max_w;
  int dda_cap;       // DDA step bound (3*ceil((dmax+trunc)/bsm)+8)
  int band;          // allocation rays start a truncation distance before the surface
  int rc_cap;        // raycast step bound (ceil(dmax/min(vs,trunc))+4)
};

// Hash entry: 16 bytes, one vector load per slot.  key packs the block
// coordinate (21 bits per axis); ptr is the block's heap index (-1: none);
// stamp is the last frame whose allocation rays touched the block.
struct __align__(16) Entry {
  unsigned long long key;
  int ptr;
  int stamp;
};

// Device counters of a session (one per session, zeroed per frame except
// nalloc).
struct Counters {
  int nalloc;          // heap top == allocated blocks (may exceed num_blocks)
  int new_blocks;
  int bucket_full;
  int heap_exhausted;
  int dda_overruns;
  int raycast_overruns;
  int visible;
  int unique_probed;
  int icp_timeout;     // the persistent ICP's grid barrier gave up (bounded wait)
};

struct F3 {
  float x, y, z;
};
__host__ __device__ inline F3 f3(float x, float y, float z) {
  F3 r;
  r.x = x;
  r.y = y;
  r.z = z;
  return r;
}
__device__ inline F3 operator+(F3 a, F3 b) { return f3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ inline F3 operator-(F3 a, F3 b) { return f3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ inline F3 operator*(F3 a, float s) { return f3(a.x * s, a.y * s, a.z * s); }
// utils.h:19-22
__device__ inline float dot3(F3 a, F3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
// cuda_math.h:397-400
__device__ inline F3 cross3(F3 a, F3 b) {
  return f3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
// cuda_math.h:409-413 (IEEE sqrt)
__device__ inline float norm3(F3 v) { return sqrtf(v.x * v.x + v.y * v.y + v.z * v.z); }
// cuda_math.h:415-419 with an exact reciprocal square root (1/sqrt): the
// oracle's host form; the device rsqrtf approximation is not used.
__device__ inline F3 normalize3(F3 v) {
  float inv = 1.0f / sqrtf(dot3(v, v));
  return v * inv;
}

struct M4f {
  float m[16];  // row-major, float4x4 layout (utils_matrix.h:816-839)
};
// float4x4::operator*(float3) with w = 1, utils_matrix.h:923-930
__device__ inline F3 xform(const M4f& T, F3 v) {
  return f3(T.m[0] * v.x + T.m[1] * v.y + T.m[2] * v.z + T.m[3] * 1.0f,
            T.m[4] * v.x + T.m[5] * v.y + T.m[6] * v.z + T.m[7] * 1.0f,
            T.m[8] * v.x + T.m[9] * v.y + T.m[10] * v.z + T.m[11] * 1.0f);
}

// getPoint3d, utils.h:104-112 (scale 1)
__device__ inline F3 point3d(int i, float depth, const DSensor& s) {
  int v = i / s.cols;
  int u = i - s.cols * v;
  F3 p;
  p.z = depth;
  p.x = ((float)u - s.cx) * p.z / s.fx;
  p.y = ((float)v - s.cy) * p.z / s.fy;
  return p;
}
// getPoint3d for pixel (u, v) known as coordinates: the same arithmetic
// without recovering them from the linear index.
__device__ inline F3 point3d_uv(int u, int v, float depth, const DSensor& s) {
  F3 p;
  p.z = depth;
  p.x = ((float)u - s.cx) * p.z / s.fx;
  p.y = ((float)v - s.cy) * p.z / s.fy;
  return p;
}

// Project, utils.h:114-119; non-finite coordinates are rejected (the
// reference converts them to int unchecked).
__device__ inline bool project(F3 p, const DSensor& s, int* px, int* py) {
  float x = ((s.fx * p.x) / p.z) + s.cx;
  float y = ((s.fy * p.y) / p.z) + s.cy;
  float rx = roundf(x), ry = roundf(y);
  if (!(fabsf(rx) < 2e9f) || !(fabsf(ry) < 2e9f)) return false;
  *px = (int)rx;
  *py = (int)ry;
  return true;
}

// WorldToGlobalVoxelHashing for one axis (tsdf.cu:189-193): the voxel index
// g = (int)(fl(p / vs) + sign(p) * 0.5), exactly.  Fast path: t = p * (1/vs)
// + sign * 0.5 differs from the exactly rounded sum by at most 4 ulps (the
// reciprocal, the product and the quotient each round once), so whenever t
// is more than 2^-19 (|t| + 1) (>= 16 ulps) away from every integer,
// truncating t gives the same integer; otherwise the IEEE division decides.
// copysign(0.5, p) is sign(p) * 0.5 for p != 0; for p = +-0 the fast path
// sees t = +-0.5, which truncates to the reference's 0; NaN and infinite t
// fail the test and take the reference's expression.
__device__ inline int voxel_index(float p, float vs, float inv_vs) {
  const float t = __fadd_rn(__fmul_rn(p, inv_vs), copysignf(0.5f, p));
  const float n = rintf(t);
  if (fabsf(t - n) > __fmaf_rn(fabsf(t), 1.9073486328125e-6f, 1.9073486328125e-6f))
    return (int)t;
  const float sg = (float)((p > 0.0f) - (p < 0.0f));
  return (int)(p / vs + sg * 0.5f);
}
// voxel_index of p and of p1 = fl(p + vs), the two corners of a trilinear
// cell along one axis.  When p's fast path applies (t is at least 16 ulps
// from every integer, so the exact p / vs + sign * 0.5 is at least 12 ulps
// away) and p and p1 take the same sign branch with t outside (-1, 0], the
// exact value for p1 is the one for p plus 1 + delta with |delta| below 2
// ulps (the rounding of p + vs and of the reference's quotient and sum),
// so its truncation is the truncation of t plus 1.  Otherwise both indices
// are computed on their own.
__device__ inline void voxel_index_pair(float p, float p1, float vs, float inv_vs, int& g0,
                                        int& g1) {
  const float t = __fadd_rn(__fmul_rn(p, inv_vs), copysignf(0.5f, p));
  const float n = rintf(t);
  if (fabsf(t - n) > __fmaf_rn(fabsf(t), 1.9073486328125e-6f, 1.9073486328125e-6f) &&
      (p > 0.0f || (p1 < 0.0f && t < -1.0f))) {
    g0 = (int)t;
    g1 = g0 + 1;
    return;
  }
  g0 = voxel_index(p, vs, inv_vs);
  g1 = voxel_index(p1, vs, inv_vs);
}
// WorldToBlock / WorldToLocalVoxel (tsdf.cu:195-225) for block size 8: the
// reference's floor division and non-negative remainder are g >> 3, g & 7.
__device__ inline int blk_of(int g) { return g >> 3; }
__device__ inline int loc_of(int g) { return g & 7; }

// HashTable::Hash, hashTable.cu:152-163: wrapping int32 products.
__host__ __device__ inline int hash_slot(int x, int y, int z, int nb, int bsz) {
  int h = (int)(((unsigned)x * 73856093u) ^ ((unsigned)y * 19349669u) ^
                ((unsigned)z * 83492791u));
  int r = h % nb;
  if (r < 0) r += nb;
  return r * bsz;
}

// The same slot: for a power-of-two bucket count the non-negative
// remainder is the low bits of the two's-complement hash.
__device__ inline int hash_slot(int x, int y, int z, const DTsdf& t) {
  if (t.nb_mask < 0) return hash_slot(x, y, z, t.num_buckets, t.bucket_size);
  int h = (int)(((unsigned)x * 73856093u) ^ ((unsigned)y * 19349669u) ^
                ((unsigned)z * 83492791u));
  return (h & t.nb_mask) * t.bucket_size;
}

__host__ __device__ inline unsigned long long pack_key(int x, int y, int z) {
  const unsigned long long m = (1ull << 21) - 1;
  return (((unsigned long long)x & m) << 42) | (((unsigned long long)y & m) << 21) |
         ((unsigned long long)z & m);
}
__host__ __device__ inline int key_x(unsigned long long k) {
  return (int)(((long long)((k >> 42) & 0x1FFFFF) << 43) >> 43);
}
__host__ __device__ inline int key_y(unsigned long long k) {
  return (int)(((long long)((k >> 21) & 0x1FFFFF) << 43) >> 43);
}
__host__ __device__ inline int key_z(unsigned long long k) {
  return (int)(((long long)(k & 0x1FFFFF) << 43) >> 43);
}

// Bucket scan, HashTable::FindHashEntry (hashTable.cu:136-150): heap index
// of the block or -1.
__device__ inline int find_block(const Entry* __restrict__ entries, const DTsdf& t,
                                 int x, int y, int z) {
  int b = hash_slot(x, y, z, t);
  unsigned long long k = pack_key(x, y, z);
  for (int i = 0; i < t.bucket_size; ++i) {
    int4 e = __ldg(reinterpret_cast<const int4*>(entries + b + i));
    unsigned long long ek = ((unsigned long long)(unsigned)e.y << 32) | (unsigned)e.x;
    if (ek == k) return e.z;
    if (ek == kEmptyKey) return -1;  // slots fill in order; none after this
  }
  return -1;
}

// Entry index of a key in its bucket, or -1 (the same scan as find_block).
__device__ inline int find_entry(const Entry* entries, const DTsdf& t, unsigned long long k) {
  int b = hash_slot(key_x(k), key_y(k), key_z(k), t);
  for (int i = 0; i < t.bucket_size; ++i) {
    unsigned long long ek = *(const volatile unsigned long long*)&entries[b + i].key;
    if (ek == k) return b + i;
    if (ek == kEmptyKey) return -1;
  }
  return -1;
}

// Lock-free unique insert into the key's bucket (the set semantics of
// HashTable::AllocateBlock, hashTable.cu:80-110, without its duplicate-
// insert race): scan the bucket in slot order, claim the first empty slot by
// CAS on the key; a lost CAS re-reads the slot.  Slots are claimed in order
// and freed only by eviction, which front-packs the bucket between frames,
// so occupied slots form a prefix of the bucket.  Returns
// the entry index if this call claimed it (heap index assigned later), -1
// if the key was present, -2 if the bucket is full.
__device__ inline int bucket_insert(Entry* entries, const DTsdf& t, unsigned long long key,
                                    int stamp, int* unique) {
  int b = hash_slot(key_x(key), key_y(key), key_z(key), t);
  for (int i = 0; i < t.bucket_size; ++i) {
    Entry* e = entries + b + i;
    unsigned long long cur = *(volatile unsigned long long*)&e->key;
    if (cur == kEmptyKey) {
      cur = atomicCAS(&e->key, kEmptyKey, key);
      if (cur == kEmptyKey) {
        atomicExch(&e->stamp, stamp);
        atomicAdd(unique, 1);
        return b + i;
      }
    }
    if (cur == key) {
      // stamps only move forward to this frame's, so a stamp that already
      // reads 'stamp' was counted by another ray: skip the contended atomic
      if (*(volatile int*)&e->stamp != stamp && atomicExch(&e->stamp, stamp) != stamp)
        atomicAdd(unique, 1);
      return -1;
    }
  }
  return -2;
}

}  // namespace dyn

// dynoracle.cpp -- CPU oracle (test infrastructure; see dynoracle.h).
//
// A serial restatement of the reference's rigid-mapping kernels.  Each
// function names the reference lines it follows (paths relative to the
// alirezaahmadi/dynamap tree).  Compile with -ffp-contract=off: every float
// expression below is evaluated as written, one IEEE rounding per operation,
// which is how the reference's own expressions round on the CPU.
//
// Fixes of reference defects (the CUDA path applies the same ones):
//  F1 integration skips free hash entries (tsdf.cu:283-291 treats them as
//     block (0,0,0));
//  F2 insertion is a unique set insert; a full bucket and an exhausted heap
//     are counted, never silent (hashTable.cu:80-110, heap.cu:14-17);
//  F3 the DDA loop is capped at 3*ceil((maxDepth+trunc)/blockSize)+8 steps
//     and overruns are counted (tsdf.cu:431-452 has no bound);
//  F4 projections whose coordinates are not finite are rejected (utils.h:114-
//     119 converts them to int unchecked);
//  F5 bilateral filter skips out-of-image and invalid (<= 0) taps; an invalid
//     centre stays 0 (pyramid.cu:213-233 reads out of bounds);
//  F6 pyramid levels are 2x2 averages of valid depths with intrinsics
//     f/s, (c+0.5)/s-0.5 (pyramid.cu:49-143 scatters into a 640x480 window);
//  F7 normals are 0 where the centre or a neighbour is invalid or outside the
//     row (rgbdImage.cu:126-145 wraps rows and reads stale vertices);
//  F8 ICP rejects projections with z <= 0 or outside the image
//     (gnSolver.cu:90-93 has no check) and photometric gradient taps outside
//     the image read the centre pixel (gnSolver.cu:182-185);
//  F9 frame order: track frame k, integrate it at the new pose, raycast the
//     target for k+1 (builder.cu:94-132 solves before copying the frame in).
#include "dynoracle.h"

#include <algorithm>
#include <cmath>

#include "../dynamap_b200/csrc/dyn_exp.h"
#include "../dynamap_b200/csrc/mc_tables.h"
#include "gn_algebra.h"
#include <cfloat>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

int g_threads = 1;

template <class R>
struct V3 {
  R x, y, z;
};
template <class R>
inline V3<R> v3(R x, R y, R z) {
  V3<R> r;
  r.x = x;
  r.y = y;
  r.z = z;
  return r;
}
// cuda_math.h:307,321,339,343: component-wise float3 operators
template <class R>
inline V3<R> operator+(V3<R> a, V3<R> b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
template <class R>
inline V3<R> operator-(V3<R> a, V3<R> b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
template <class R>
inline V3<R> operator*(V3<R> a, R s) { return v3(a.x * s, a.y * s, a.z * s); }
// utils.h:19-22 / cuda_math.h:391-394
template <class R>
inline R dot(V3<R> a, V3<R> b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
// cuda_math.h:397-400
template <class R>
inline V3<R> cross(V3<R> a, V3<R> b) {
  return v3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
// cuda_math.h:409-413
template <class R>
inline R norm(V3<R> v) { return std::sqrt(v.x * v.x + v.y * v.y + v.z * v.z); }
// cuda_math.h:415-419 with the host rsqrtf of cuda_math.h:50-53 (1/sqrt)
template <class R>
inline V3<R> normalize(V3<R> v) {
  R inv = R(1) / std::sqrt(dot(v, v));
  return v * inv;
}
// utils.h:88-90
template <class R>
inline R distance(V3<R> a, V3<R> b) { return norm(a - b); }
// utils.h:92-96
inline int sign_i(double n) { return (n > 0) - (n < 0); }
template <class R>
inline R signf_(R v) { return (R)((v > 0) - (v < 0)); }

template <class R>
struct M4 {
  R m[16];  // row-major m11..m44 (utils_matrix.h:816-839)
};
// float4x4::operator*(float3), utils_matrix.h:923-930 (w = 1)
template <class R>
inline V3<R> xform(const M4<R>& T, V3<R> v) {
  return v3(T.m[0] * v.x + T.m[1] * v.y + T.m[2] * v.z + T.m[3] * R(1),
            T.m[4] * v.x + T.m[5] * v.y + T.m[6] * v.z + T.m[7] * R(1),
            T.m[8] * v.x + T.m[9] * v.y + T.m[10] * v.z + T.m[11] * R(1));
}
template <class R, class S>
inline M4<R> m4_from(const S* p) {
  M4<R> M;
  for (int i = 0; i < 16; ++i) M.m[i] = (R)p[i];
  return M;
}

// float4x4::getInverse, utils_matrix.h:970-1086: cofactor expansion of a
// general 4x4 matrix; terms summed in the order written there, the
// determinant from row 0, then every cofactor times 1/det.
template <class R>
M4<R> inverse4(const M4<R>& M) {
  const R* e = M.m;
  R inv[16];
  inv[0] = e[5] * e[10] * e[15] - e[5] * e[11] * e[14] - e[9] * e[6] * e[15] +
           e[9] * e[7] * e[14] + e[13] * e[6] * e[11] - e[13] * e[7] * e[10];
  inv[4] = -e[4] * e[10] * e[15] + e[4] * e[11] * e[14] + e[8] * e[6] * e[15] -
           e[8] * e[7] * e[14] - e[12] * e[6] * e[11] + e[12] * e[7] * e[10];
  inv[8] = e[4] * e[9] * e[15] - e[4] * e[11] * e[13] - e[8] * e[5] * e[15] +
           e[8] * e[7] * e[13] + e[12] * e[5] * e[11] - e[12] * e[7] * e[9];
  inv[12] = -e[4] * e[9] * e[14] + e[4] * e[10] * e[13] + e[8] * e[5] * e[14] -
            e[8] * e[6] * e[13] - e[12] * e[5] * e[10] + e[12] * e[6] * e[9];
  inv[1] = -e[1] * e[10] * e[15] + e[1] * e[11] * e[14] + e[9] * e[2] * e[15] -
           e[9] * e[3] * e[14] - e[13] * e[2] * e[11] + e[13] * e[3] * e[10];
  inv[5] = e[0] * e[10] * e[15] - e[0] * e[11] * e[14] - e[8] * e[2] * e[15] +
           e[8] * e[3] * e[14] + e[12] * e[2] * e[11] - e[12] * e[3] * e[10];
  inv[9] = -e[0] * e[9] * e[15] + e[0] * e[11] * e[13] + e[8] * e[1] * e[15] -
           e[8] * e[3] * e[13] - e[12] * e[1] * e[11] + e[12] * e[3] * e[9];
  inv[13] = e[0] * e[9] * e[14] - e[0] * e[10] * e[13] - e[8] * e[1] * e[14] +
            e[8] * e[2] * e[13] + e[12] * e[1] * e[10] - e[12] * e[2] * e[9];
  inv[2] = e[1] * e[6] * e[15] - e[1] * e[7] * e[14] - e[5] * e[2] * e[15] +
           e[5] * e[3] * e[14] + e[13] * e[2] * e[7] - e[13] * e[3] * e[6];
  inv[6] = -e[0] * e[6] * e[15] + e[0] * e[7] * e[14] + e[4] * e[2] * e[15] -
           e[4] * e[3] * e[14] - e[12] * e[2] * e[7] + e[12] * e[3] * e[6];
  inv[10] = e[0] * e[5] * e[15] - e[0] * e[7] * e[13] - e[4] * e[1] * e[15] +
            e[4] * e[3] * e[13] + e[12] * e[1] * e[7] - e[12] * e[3] * e[5];
  inv[14] = -e[0] * e[5] * e[14] + e[0] * e[6] * e[13] + e[4] * e[1] * e[14] -
            e[4] * e[2] * e[13] - e[12] * e[1] * e[6] + e[12] * e[2] * e[5];
  inv[3] = -e[1] * e[6] * e[11] + e[1] * e[7] * e[10] + e[5] * e[2] * e[11] -
           e[5] * e[3] * e[10] - e[9] * e[2] * e[7] + e[9] * e[3] * e[6];
  inv[7] = e[0] * e[6] * e[11] - e[0] * e[7] * e[10] - e[4] * e[2] * e[11] +
           e[4] * e[3] * e[10] + e[8] * e[2] * e[7] - e[8] * e[3] * e[6];
  inv[11] = -e[0] * e[5] * e[11] + e[0] * e[7] * e[9] + e[4] * e[1] * e[11] -
            e[4] * e[3] * e[9] - e[8] * e[1] * e[7] + e[8] * e[3] * e[5];
  inv[15] = e[0] * e[5] * e[10] - e[0] * e[6] * e[9] - e[4] * e[1] * e[10] +
            e[4] * e[2] * e[9] + e[8] * e[1] * e[6] - e[8] * e[2] * e[5];
  R det = e[0] * inv[0] + e[1] * inv[4] + e[2] * inv[8] + e[3] * inv[12];
  R detr = R(1) / det;
  M4<R> out;
  for (int i = 0; i < 16; ++i) out.m[i] = inv[i] * detr;
  return out;
}

template <class R>
struct Sensor {
  int rows, cols;
  R fx, fy, cx, cy;
};
template <class R>
Sensor<R> mk_sensor(const dyn_sensor& s) {
  Sensor<R> o;
  o.rows = (int)s.rows;
  o.cols = (int)s.cols;
  o.fx = (R)s.fx;
  o.fy = (R)s.fy;
  o.cx = (R)s.cx;
  o.cy = (R)s.cy;
  return o;
}

// getPoint3d, utils.h:104-112 (scale 1: f/1 == f exactly)
template <class R>
inline V3<R> getPoint3d(int i, R depth, const Sensor<R>& s) {
  int v = i / s.cols;
  int u = i - s.cols * v;
  V3<R> p;
  p.z = depth;
  p.x = ((R)u - s.cx) * p.z / s.fx;
  p.y = ((R)v - s.cy) * p.z / s.fy;
  return p;
}
// Project, utils.h:114-119, plus F4 (non-finite -> rejected)
template <class R>
inline bool project(V3<R> p, const Sensor<R>& s, int* px, int* py) {
  R x = ((s.fx * p.x) / p.z) + s.cx;
  R y = ((s.fy * p.y) / p.z) + s.cy;
  R rx = std::round(x), ry = std::round(y);
  if (!(std::fabs(rx) < (R)2e9) || !(std::fabs(ry) < (R)2e9)) return false;
  *px = (int)rx;
  *py = (int)ry;
  return true;
}

// ------------------------------------------------------------- hash table
// HashTable::Hash, hashTable.cu:152-163.  The int32 products wrap exactly
// as the 32-bit device multiply does (computed in uint32 to avoid UB).
inline int32_t hash_slot(int32_t x, int32_t y, int32_t z, int32_t nb,
                         int32_t bsz) {
  const uint32_t p1 = 73856093u, p2 = 19349669u, p3 = 83492791u;
  int32_t h = (int32_t)(((uint32_t)x * p1) ^ ((uint32_t)y * p2) ^
                        ((uint32_t)z * p3));
  int32_t r = h % nb;
  if (r < 0) r += nb;
  return r * bsz;
}

template <class R>
struct Voxel {
  uint8_t c[3];
  uint8_t w;
  R sdf;
};

// Voxel::mergeVoxel, geom_Types.h:79-103 (new voxel weight is always 1 on
// the path; written for a general weight).
template <class R>
inline void merge_voxel(Voxel<R>& o, R sdf, const uint8_t col[3], uint8_t w,
                        int max_w) {
  o.sdf = (o.sdf * (R)o.w + sdf * (R)w) / ((R)o.w + (R)w);
  for (int k = 0; k < 3; ++k)
    o.c[k] = (uint8_t)(((float)o.c[k] * (float)o.w + (float)col[k] * (float)w) /
                       ((float)o.w + (float)w));
  int nw = (uint8_t)(o.w + w);
  if (nw > max_w) nw = max_w;
  o.w = (uint8_t)nw;
}

template <class R>
struct Volume {
  dyn_tsdf_params p;
  int nentries;
  std::vector<int32_t> ex, ey, ez, eptr;  // HashEntry, hashTable.h:20-25
  std::vector<Voxel<R>> vox;              // num_blocks * bs^3
  std::vector<int32_t> bx, by, bz;        // block coordinate per heap index
  int64_t nalloc = 0;

  explicit Volume(const dyn_tsdf_params& pp) : p(pp) {
    nentries = p.num_buckets * p.bucket_size;
    ex.assign(nentries, 0);  // InitEntriesKernel, hashTable.cu:12-19
    ey.assign(nentries, 0);
    ez.assign(nentries, 0);
    eptr.assign(nentries, -1);
    int bs3 = p.block_size * p.block_size * p.block_size;
    Voxel<R> z;
    z.c[0] = z.c[1] = z.c[2] = 0;
    z.w = 0;
    z.sdf = 0;
    vox.assign((size_t)p.num_blocks * bs3, z);  // InitHeapKernel :22-39
    bx.assign(p.num_blocks, 0);
    by.assign(p.num_blocks, 0);
    bz.assign(p.num_blocks, 0);
  }
  // HashTable::FindHashEntry, hashTable.cu:136-150 (returns ptr or -1)
  int find(int x, int y, int z) const {
    int b = hash_slot(x, y, z, p.num_buckets, p.bucket_size);
    for (int i = 0; i < p.bucket_size; ++i) {
      int k = b + i;
      if (ex[k] == x && ey[k] == y && ez[k] == z && eptr[k] != -1) return eptr[k];
    }
    return -1;
  }
  // HashTable::AllocateBlock, hashTable.cu:80-110, serial; F2.
  // returns 1 new, 0 present, -1 bucket full, -2 heap exhausted
  int allocate(int x, int y, int z) {
    int b = hash_slot(x, y, z, p.num_buckets, p.bucket_size);
    int free_idx = -1;
    for (int i = 0; i < p.bucket_size; ++i) {
      int k = b + i;
      if (ex[k] == x && ey[k] == y && ez[k] == z && eptr[k] != -1) return 0;
      if (free_idx == -1 && eptr[k] == -1) free_idx = k;
    }
    if (free_idx == -1) return -1;
    // Heap::Consume, heap.cu:14-17 over the identity stack of
    // InitHeapKernel (hashTable.cu:26-31): indices come out 0, 1, 2, ...
    if (nalloc >= p.num_blocks) return -2;
    int ptr = (int)nalloc++;
    ex[free_idx] = x;
    ey[free_idx] = y;
    ez[free_idx] = z;
    eptr[free_idx] = ptr;
    bx[ptr] = x;
    by[ptr] = y;
    bz[ptr] = z;
    return 1;
  }
  // tsdf.cu:189-193 WorldToGlobalVoxelHashing
  V3<int> world_to_global(V3<R> pos) const {
    R vs = (R)p.voxel_size;
    V3<int> g;
    g.x = (int)(pos.x / vs + signf_(pos.x) * (R)0.5);
    g.y = (int)(pos.y / vs + signf_(pos.y) * (R)0.5);
    g.z = (int)(pos.z / vs + signf_(pos.z) * (R)0.5);
    return g;
  }
  // tsdf.cu:195-214 WorldToBlock and :216-225 WorldToLocalVoxel
  void world_to_block_local(V3<R> pos, V3<int>* blk, int* lin) const {
    V3<int> g = world_to_global(pos);
    int bs = p.block_size;
    int gv[3] = {g.x, g.y, g.z}, bv[3], lv[3];
    for (int k = 0; k < 3; ++k) {
      bv[k] = gv[k] < 0 ? (gv[k] - bs + 1) / bs : gv[k] / bs;
      lv[k] = gv[k] % bs;
      if (lv[k] < 0) lv[k] += bs;
    }
    blk->x = bv[0];
    blk->y = bv[1];
    blk->z = bv[2];
    *lin = lv[0] * bs * bs + lv[1] * bs + lv[2];  // VoxelBlock::at, geom_Types.h:116-119
  }
  // tsdfVolume::GetVoxel, tsdf.cu:227-239
  Voxel<R> get_voxel(V3<R> pos) const {
    V3<int> b;
    int lin;
    world_to_block_local(pos, &b, &lin);
    int ptr = find(b.x, b.y, b.z);
    if (ptr < 0) {
      Voxel<R> z;
      z.c[0] = z.c[1] = z.c[2] = 0;
      z.w = 0;
      z.sdf = 0;
      return z;
    }
    int bs3 = p.block_size * p.block_size * p.block_size;
    return vox[(size_t)ptr * bs3 + lin];
  }
  // tsdfVolume::GetInterpolatedVoxel, tsdf.cu:47-175.  Fractional weights
  // come from position/voxelSize (not the shifted position), corners with
  // weight 0 use the centre voxel, corners summed in the order below.
  Voxel<R> get_interpolated(V3<R> position) const {
    Voxel<R> v0 = get_voxel(position);
    if (v0.w == 0) return v0;
    R vs = (R)p.voxel_size;
    V3<R> pos_dual = position - v3(vs / R(2), vs / R(2), vs / R(2));
    R inv = R(1) / vs;  // float3 / float -> a * (1/s), cuda_math.h:357-361
    V3<R> vp = position * inv;
    V3<R> w = v3(vp.x - std::floor(vp.x), vp.y - std::floor(vp.y),
                 vp.z - std::floor(vp.z));
    static const int off[8][3] = {{0, 0, 0}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1},
                                  {1, 1, 0}, {0, 1, 1}, {1, 0, 1}, {1, 1, 1}};
    R dist = 0;
    V3<R> col = v3(R(0), R(0), R(0));
    for (int k = 0; k < 8; ++k) {
      V3<R> q = pos_dual + v3(off[k][0] ? vs : R(0), off[k][1] ? vs : R(0),
                              off[k][2] ? vs : R(0));
      Voxel<R> v = get_voxel(q);
      const Voxel<R>& s = (v.w == 0) ? v0 : v;
      R a = off[k][0] ? w.x : R(1) - w.x;
      R b = off[k][1] ? w.y : R(1) - w.y;
      R c = off[k][2] ? w.z : R(1) - w.z;
      R coef = a * b * c;
      dist += coef * s.sdf;
      col = col + v3((R)s.c[0], (R)s.c[1], (R)s.c[2]) * coef;
    }
    Voxel<R> out;
    out.c[0] = (uint8_t)col.x;
    out.c[1] = (uint8_t)col.y;
    out.c[2] = (uint8_t)col.z;
    out.w = v0.w;
    out.sdf = dist;
    return out;
  }
};

// ---------------------------------------------------------- mesh vertices
// MeshExtractor's TrilinearInterpolation (meshExtractor.cu:22-93): the
// 2x2x2 cell around position, false as soon as a corner is unobserved
// (unlike GetInterpolatedVoxel, which substitutes the centre voxel);
// weights from position * (1/vs), corners summed in the order below.
template <class R>
bool mesh_trilinear(const Volume<R>& V, V3<R> position, R* dist) {
  R vs = (R)V.p.voxel_size;
  V3<R> pos_dual = position - v3(vs / R(2), vs / R(2), vs / R(2));
  V3<R> vp = position * (R(1) / vs);  // float3 / float, cuda_math.h:357-361
  V3<R> w = v3(vp.x - std::floor(vp.x), vp.y - std::floor(vp.y), vp.z - std::floor(vp.z));
  static const int off[8][3] = {{0, 0, 0}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1},
                                {1, 1, 0}, {0, 1, 1}, {1, 0, 1}, {1, 1, 1}};
  R d = 0;
  for (int k = 0; k < 8; ++k) {
    Voxel<R> v = V.get_voxel(pos_dual + v3(off[k][0] ? vs : R(0), off[k][1] ? vs : R(0),
                                           off[k][2] ? vs : R(0)));
    if (v.w == 0) return false;
    R a = off[k][0] ? w.x : R(1) - w.x;
    R b = off[k][1] ? w.y : R(1) - w.y;
    R c = off[k][2] ? w.z : R(1) - w.z;
    d += a * b * c * v.sdf;
  }
  *dist = d;
  return true;
}

// MeshExtractor::ExtractMesh (meshExtractor.cu:364-407) up to the vertices:
// the grid of the box [lo, hi) with twice the box's extent in voxel steps
// (as the reference's grid_size), per grid position the eight corner
// samples at +-vs/2 (ExtractMeshAtPosition :126-214) and, on every cube
// edge whose ends are on opposite sides of 0, the vertex VertexInterpolation
// (:95-121) places, coloured by the centre voxel.  Each vertex is
// {x, y, z, r, g, b}; the reference's triangles (its marching-cubes table)
// use exactly these vertices.  Returns the count (at most cap written).
// The cell walk shared by mesh_vertices and mesh_triangles: for every grid
// cell with all corners observed and a zero crossing, cell(cube, vert)
// with vert[e] = {x, y, z, r, g, b} for every cut edge e.
// cell(z, cube, vert) is called for the cells of z-slice z in grid order,
// the slices in parallel (OpenMP); the callers keep one output per slice
// and join them in slice order, so the result is the serial walk's.
template <class F>
void mesh_cells(const Volume<float>& V, const float lo[3], const float hi[3], F&& cell) {
  const float vs = (float)V.p.voxel_size;
  V3<float> size = v3(std::fabs(lo[0] - hi[0]), std::fabs(lo[1] - hi[1]),
                      std::fabs(lo[2] - hi[2]));
  const int gx = (int)(size.x / vs * 2), gy = (int)(size.y / vs * 2), gz = (int)(size.z / vs * 2);
  const float P = vs / 2.0f, M = -P;
  // corners in the reference's cube-index order (bit k: corner k inside)
  // and the 12 edges between them
  static const int corner[8][3] = {{0, 1, 0}, {1, 1, 0}, {1, 0, 0}, {0, 0, 0},
                                   {0, 1, 1}, {1, 1, 1}, {1, 0, 1}, {0, 0, 1}};
  static const int edge[12][2] = {{0, 1}, {1, 2}, {2, 3}, {3, 0}, {4, 5}, {5, 6},
                                  {6, 7}, {7, 4}, {0, 4}, {1, 5}, {2, 6}, {3, 7}};
  const int nt = std::max(1, g_threads);
#pragma omp parallel for num_threads(nt) schedule(dynamic, 1)
  for (int pz = 0; pz < gz; ++pz)
  for (int64_t j = 0; j < (int64_t)gx * gy; ++j) {
    const int px = (int)(j % gx), py = (int)(j / gx);
    const V3<float> pos = v3((float)px * vs + lo[0], (float)py * vs + lo[1], (float)pz * vs + lo[2]);
    V3<float> p[8];
    float d[8];
    bool ok = true;
    for (int k = 0; k < 8 && ok; ++k) {
      p[k] = pos + v3(corner[k][0] ? P : M, corner[k][1] ? P : M, corner[k][2] ? P : M);
      ok = mesh_trilinear(V, p[k], &d[k]);
    }
    if (!ok) continue;
    unsigned cube = 0;
    for (int k = 0; k < 8; ++k)
      if (d[k] < 0.0f) cube |= 1u << k;
    if (cube == 0 || cube == 255) continue;
    const Voxel<float> c = V.get_voxel(pos);
    const float rgb0[3] = {(float)c.c[0] * (1.0f / 255.f), (float)c.c[1] * (1.0f / 255.f),
                           (float)c.c[2] * (1.0f / 255.f)};
    float vert[12][6];
    for (int e = 0; e < 12; ++e) {
      const int a = edge[e][0], b = edge[e][1];
      if (((cube >> a) & 1u) == ((cube >> b) & 1u)) continue;
      float* vtx = vert[e];
      const float d1 = d[a], d2 = d[b];
      const V3<float> p1 = p[a], p2 = p[b];
      bool end = true;
      V3<float> q = p1;
      if (std::fabs(0.0f - d1) < 0.00001f) q = p1;
      else if (std::fabs(0.0f - d2) < 0.00001f) q = p2;
      else if (std::fabs(d1 - d2) < 0.00001f) q = p1;
      else end = false;
      if (end) {
        vtx[3] = rgb0[0];
        vtx[4] = rgb0[1];
        vtx[5] = rgb0[2];
      } else {
        const float mu = (0.0f - d1) / (d2 - d1);
        q = v3(p1.x + mu * (p2.x - p1.x), p1.y + mu * (p2.y - p1.y), p1.z + mu * (p2.z - p1.z));
        for (int k = 0; k < 3; ++k)
          vtx[3 + k] = (float)((float)c.c[k] + mu * (float)(c.c[k] - c.c[k])) / 255.f;
      }
      vtx[0] = q.x;
      vtx[1] = q.y;
      vtx[2] = q.z;
    }
    cell(pz, cube, vert);
  }
}

// The slice outputs of mesh_cells joined in slice order: 'per' floats per
// item, at most cap items into out; returns the item count.
static int64_t join_slices(const std::vector<std::vector<float>>& sl, int per, float* out,
                           int64_t cap) {
  int64_t n = 0;
  for (const std::vector<float>& v : sl) {
    const int64_t k = (int64_t)v.size() / per;
    for (int64_t i = 0; i < k; ++i, ++n)
      if (n < cap) std::copy(v.begin() + i * per, v.begin() + (i + 1) * per, out + n * per);
  }
  return n;
}

// The number of z-slices mesh_cells walks.
static size_t mesh_slices(const Volume<float>& V, const float lo[3], const float hi[3]) {
  const float vs = (float)V.p.voxel_size;
  const int gz = (int)(std::fabs(lo[2] - hi[2]) / vs * 2);
  return gz > 0 ? (size_t)gz : 0;
}

int64_t mesh_vertices(const Volume<float>& V, const float lo[3], const float hi[3],
                      float* out, int64_t cap) {
  static const int edge[12][2] = {{0, 1}, {1, 2}, {2, 3}, {3, 0}, {4, 5}, {5, 6},
                                  {6, 7}, {7, 4}, {0, 4}, {1, 5}, {2, 6}, {3, 7}};
  std::vector<std::vector<float>> sl(mesh_slices(V, lo, hi));
  mesh_cells(V, lo, hi, [&](int z, unsigned cube, const float (*vert)[6]) {
    for (int e = 0; e < 12; ++e) {
      if (((cube >> edge[e][0]) & 1u) == ((cube >> edge[e][1]) & 1u)) continue;
      sl[z].insert(sl[z].end(), vert[e], vert[e] + 6);
    }
  });
  return join_slices(sl, 6, out, cap);
}

// The mesh of the same cells with this project's marching-cubes table
// (dynamap_b200/csrc/mc_tables.h, generated by dynamap_b200/mc_tables.py,
// not the reference's table): 18 floats per triangle, three vertices
// {x, y, z, r, g, b}.  Returns the triangle count.
int64_t mesh_triangles(const Volume<float>& V, const float lo[3], const float hi[3],
                       float* out, int64_t cap) {
  std::vector<std::vector<float>> sl(mesh_slices(V, lo, hi));
  mesh_cells(V, lo, hi, [&](int z, unsigned cube, const float (*vert)[6]) {
    const signed char* row = dyn::kMcTriangles[cube];
    for (int j = 0; j + 2 < dyn::kMcMaxTriIdx && row[j] >= 0; j += 3)
      for (int k = 0; k < 3; ++k) sl[z].insert(sl[z].end(), vert[row[j + k]], vert[row[j + k]] + 6);
  });
  return join_slices(sl, 18, out, cap);
}

// AllocateFromDepthKernel, tsdf.cu:346-453 for one pixel: visits blocks in
// the reference's DDA order and calls f(x, y, z) for each (the `diff`
// pre-step included).  Returns false if the step cap (F3) cut the ray.
template <class R, class F>
bool dda_ray(V3<R> start_pt, V3<R> point, R trunc, R block_size, int cap,
             F&& f) {
  V3<R> dir = normalize(point - start_pt);
  R surface_distance = distance(start_pt, point);
  V3<R> ray_start = start_pt;
  V3<R> ray_end = start_pt + dir * (surface_distance + trunc);
  int bpx = (int)std::floor(ray_start.x / block_size);
  int bpy = (int)std::floor(ray_start.y / block_size);
  int bpz = (int)std::floor(ray_start.z / block_size);
  int ebx = (int)std::floor(ray_end.x / block_size);
  int eby = (int)std::floor(ray_end.y / block_size);
  int ebz = (int)std::floor(ray_end.z / block_size);
  int sx = sign_i(dir.x), sy = sign_i(dir.y), sz = sign_i(dir.z);
  R dtx = dir.x != 0 ? std::fabs(block_size / dir.x) : (R)FLT_MAX;
  R dty = dir.y != 0 ? std::fabs(block_size / dir.y) : (R)FLT_MAX;
  R dtz = dir.z != 0 ? std::fabs(block_size / dir.z) : (R)FLT_MAX;
  R bdx = ((R)bpx + (R)sx) * block_size;
  R bdy = ((R)bpy + (R)sy) * block_size;
  R bdz = ((R)bpz + (R)sz) * block_size;
  R mx = dir.x != 0 ? (bdx - ray_start.x) / dir.x : (R)FLT_MAX;
  R my = dir.y != 0 ? (bdy - ray_start.y) / dir.y : (R)FLT_MAX;
  R mz = dir.z != 0 ? (bdz - ray_start.z) / dir.z : (R)FLT_MAX;
  int dx = 0, dy = 0, dz = 0;
  bool neg = false;
  if (bpx != ebx && dir.x < 0) { dx--; neg = true; }
  if (bpy != eby && dir.y < 0) { dy--; neg = true; }
  if (bpz != ebz && dir.z < 0) { dz--; neg = true; }
  f(bpx, bpy, bpz);
  if (neg) {
    bpx += dx;
    bpy += dy;
    bpz += dz;
    f(bpx, bpy, bpz);
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
    f(bpx, bpy, bpz);
  }
  return true;
}

inline int dda_cap(const dyn_tsdf_params& p) {
  double bs = (double)p.block_size * (double)p.voxel_size;
  return 3 * (int)std::ceil(((double)p.max_sensor_depth +
                             (double)p.truncation_distance) / bs) + 8;
}

inline uint64_t pack_key(int x, int y, int z) {
  const uint64_t m = (1ull << 21) - 1;
  return (((uint64_t)x & m) << 42) | (((uint64_t)y & m) << 21) | ((uint64_t)z & m);
}

template <class R>
void volume_allocate(Volume<R>& V, const R* depth, const Sensor<R>& s,
                     const M4<R>& T, int64_t* cnt) {
  const dyn_tsdf_params& p = V.p;
  R trunc = (R)p.truncation_distance;
  R block_size = (R)p.block_size * (R)p.voxel_size;  // tsdf.cu:437-438
  R dmin = (R)p.min_sensor_depth, dmax = (R)p.max_sensor_depth;
  V3<R> start_pt = v3(T.m[3], T.m[7], T.m[11]);  // tsdf.cu:440
  int n = s.rows * s.cols;
  int cap = dda_cap(p);
  // rays in parallel; insertion serial in pixel order (== serial order)
  int nt = std::max(1, g_threads);
  std::vector<std::vector<uint64_t>> keys(nt);
  std::vector<int64_t> over(nt, 0);
#pragma omp parallel for num_threads(nt) schedule(static)
  for (int t = 0; t < nt; ++t) {
    int lo = (int)((int64_t)n * t / nt), hi = (int)((int64_t)n * (t + 1) / nt);
    std::vector<uint64_t>& K = keys[t];
    for (int i = lo; i < hi; ++i) {
      R d = depth[i];
      if (d < dmin || d > dmax) continue;  // tsdf.cu:442-444
      V3<R> point = xform(T, getPoint3d(i, d, s));
      if (point.x == 0 && point.y == 0 && point.z == 0) continue;
      uint64_t last = ~0ull;
      bool ok = dda_ray(start_pt, point, trunc, block_size, cap,
                        [&](int x, int y, int z) {
                          uint64_t k = pack_key(x, y, z);
                          if (k != last) K.push_back(k);
                          last = k;
                        });
      if (!ok) over[t]++;
    }
  }
  std::vector<uint64_t> uniq;
  for (int t = 0; t < nt; ++t) {
    cnt[DYO_C_DDA_OVERRUNS] += over[t];
    for (uint64_t k : keys[t]) {
      // unpack the 21-bit fields with sign extension
      int x = (int)(((int64_t)((k >> 42) & 0x1FFFFF) << 43) >> 43);
      int y = (int)(((int64_t)((k >> 21) & 0x1FFFFF) << 43) >> 43);
      int z = (int)(((int64_t)(k & 0x1FFFFF) << 43) >> 43);
      int r = V.allocate(x, y, z);
      if (r == 1) cnt[DYO_C_NEW_BLOCKS]++;
      else if (r == -1) cnt[DYO_C_BUCKET_FULL]++;
      else if (r == -2) cnt[DYO_C_HEAP_EXHAUSTED]++;
      uniq.push_back(k);
    }
  }
  std::sort(uniq.begin(), uniq.end());
  cnt[DYO_C_UNIQUE_PROBED] +=
      (int64_t)(std::unique(uniq.begin(), uniq.end()) - uniq.begin());
}

// IntegrateScanKernel, tsdf.cu:268-344, per allocated block (F1).  The
// reference hands each voxel to UpdateVoxel (tsdf.cu:252-266) after the
// camera -> world round trip; that round trip is done here too and any
// voxel it moves is counted (DYO_C_REHASH_MISMATCH) and updated where the
// reference would update it.
template <class R>
void volume_integrate(Volume<R>& V, const R* depth, const uint8_t* rgb,
                      const Sensor<R>& s, const M4<R>& T, int64_t* cnt) {
  const dyn_tsdf_params& p = V.p;
  M4<R> invT = inverse4(T);  // tsdf.cu:464
  int block_size = p.block_size;
  R voxel_size = (R)p.voxel_size;
  R trunc = (R)p.truncation_distance;
  R dmin = (R)p.min_sensor_depth, dmax = (R)p.max_sensor_depth;
  int bs3 = block_size * block_size * block_size;
  int64_t nb = V.nalloc;
  int nt = std::max(1, g_threads);
  int64_t vis = 0, mism = 0;
#pragma omp parallel for num_threads(nt) schedule(dynamic, 16) reduction(+ : vis, mism)
  for (int64_t b = 0; b < nb; ++b) {
    V3<R> position = v3((R)V.bx[b] * voxel_size * (R)block_size,
                        (R)V.by[b] * voxel_size * (R)block_size,
                        (R)V.bz[b] * voxel_size * (R)block_size);
    V3<R> pc = xform(invT, position);
    if (pc.z < 0) continue;
    double half = 0.5 * (double)voxel_size * (double)block_size;
    V3<R> bc = v3((R)((double)pc.x + half), (R)((double)pc.y + half),
                  (R)((double)pc.z + half));
    int ix, iy;
    if (!project(bc, s, &ix, &iy)) continue;
    if (!(ix >= 0 && iy >= 0 && ix < s.cols && iy < s.rows)) continue;
    vis++;
    V3<R> start_pt = v3(R(0), R(0), R(0));
    for (int x = 0; x < block_size; ++x)
      for (int y = 0; y < block_size; ++y)
        for (int z = 0; z < block_size; ++z) {
          V3<R> vpos = v3(position.x + (R)x * voxel_size,
                          position.y + (R)y * voxel_size,
                          position.z + (R)z * voxel_size);
          vpos = xform(invT, vpos);
          int px, py;
          if (!project(vpos, s, &px, &py)) continue;
          if (!(px >= 0 && py >= 0 && px < s.cols && py < s.rows)) continue;
          int idx = py * s.cols + px;
          R d = depth[idx];
          if (d < dmin) continue;
          if (d > dmax) continue;
          V3<R> p3 = getPoint3d(idx, d, s);
          R sd = distance(start_pt, p3);
          R vd = distance(start_pt, vpos);
          R sdf;
          if (vd > sd - trunc && vd < sd + trunc && d < dmax) {
            sdf = sd - vd;
          } else if (vd < sd - trunc) {
            sdf = trunc;
          } else {
            continue;
          }
          uint8_t col[3] = {0, 0, 0};
          if (rgb) {
            col[0] = rgb[3 * idx + 0];
            col[1] = rgb[3 * idx + 1];
            col[2] = rgb[3 * idx + 2];
          }
          V3<R> world = xform(T, vpos);
          V3<int> blk;
          int lin;
          V.world_to_block_local(world, &blk, &lin);
          int own = x * block_size * block_size + y * block_size + z;
          int64_t target = -1;
          if (blk.x == V.bx[b] && blk.y == V.by[b] && blk.z == V.bz[b] &&
              lin == own) {
            target = b * bs3 + own;
          } else {
            mism++;
            int ptr = V.find(blk.x, blk.y, blk.z);
            if (ptr >= 0) target = (int64_t)ptr * bs3 + lin;
          }
          if (target >= 0)
            merge_voxel(V.vox[(size_t)target], sdf, col, (uint8_t)1,
                        p.max_sdf_weight);
        }
  }
  cnt[DYO_C_VISIBLE] += vis;
  cnt[DYO_C_REHASH_MISMATCH] += mism;
}

inline int raycast_cap(const dyn_tsdf_params& p) {
  double step = std::min((double)p.voxel_size, (double)p.truncation_distance);
  return (int)std::ceil((double)p.max_sensor_depth / step) + 4;
}

// GenerateDepthKernel / GenerateRgbKernel, tsdf.cu:471-526.
template <class R>
void volume_raycast(const Volume<R>& V, const M4<R>& T, const Sensor<R>& s,
                    R* depth_out, uint8_t* rgb_out, int64_t* cnt) {
  const dyn_tsdf_params& p = V.p;
  R maxd = (R)p.max_sensor_depth, trunc = (R)p.truncation_distance,
    vs = (R)p.voxel_size;
  int n = s.rows * s.cols;
  int cap = raycast_cap(p);
  int nt = std::max(1, g_threads);
  int64_t over = 0;
#pragma omp parallel for num_threads(nt) schedule(dynamic, 256) reduction(+ : over)
  for (int i = 0; i < n; ++i) {
    R cur = 0;
    int steps = 0;
    while (cur < maxd) {
      if (steps++ >= cap) {
        over++;
        break;
      }
      V3<R> point = xform(T, getPoint3d(i, cur, s));
      Voxel<R> v = V.get_interpolated(point);
      if (v.w == 0) cur += trunc;
      else cur += v.sdf;
      if (v.w != 0 && v.sdf < vs) break;
    }
    depth_out[i] = cur;
    if (rgb_out) {
      if (cur < maxd) {
        V3<R> point = xform(T, getPoint3d(i, cur, s));
        Voxel<R> v = V.get_interpolated(point);
        rgb_out[3 * i + 0] = v.c[0];
        rgb_out[3 * i + 1] = v.c[1];
        rgb_out[3 * i + 2] = v.c[2];
      } else {
        rgb_out[3 * i + 0] = rgb_out[3 * i + 1] = rgb_out[3 * i + 2] = 0;
      }
    }
  }
  cnt[DYO_C_RAYCAST_OVERRUNS] += over;
}

// ------------------------------------------------------------------ images
// pyramid::gaussian, pyramid.cu:208-211 (double)
inline double gaussian_d(double x, double sigma) {
  return std::exp(-(std::pow(x, 2)) / (2 * std::pow(sigma, 2))) /
         (2 * M_PI * std::pow(sigma, 2));
}

// applyBilateralFilter, pyramid.cu:213-233 with F5.  Window 2r taps per
// axis, offsets -r .. r-1 (pyramid.cu:218-224, 250).
template <class R>
void bilateral(const R* src, R* dst, int rows, int cols, int r, double sI,
               double sS) {
  int diameter = 2 * r, half = diameter / 2;
  // spatial weights: gaussian(vertexDistance(x, y, nx, ny), sigmaS) in
  // float as pyramid.cu:226 computes them (pyramid.cu:201-206)
  std::vector<R> gs((size_t)diameter * diameter);
  for (int i = 0; i < diameter; ++i)
    for (int j = 0; j < diameter; ++j) {
      float dx = (float)(half - i), dy = (float)(half - j);
      float dd = std::sqrt(dx * dx + dy * dy + 0.0f * 0.0f);
      gs[(size_t)i * diameter + j] = (R)(float)gaussian_d((double)dd, sS);
    }
  // range weight: FP32 through dyn_expf (dynamap_b200/csrc/dyn_exp.h), the
  // operation sequence the CUDA kernel runs; FP64 through exp, as
  // pyramid.cu:208-211 computes it.
  const float inv2s2 = (float)(1.0 / (2.0 * sI * sI));
  const float norm = (float)(1.0 / (2.0 * M_PI * sI * sI));
  int nt = std::max(1, g_threads);
#pragma omp parallel for num_threads(nt) schedule(static)
  for (int x = 0; x < rows; ++x) {
    for (int y = 0; y < cols; ++y) {
      int pid = x * cols + y;
      R c = src[pid];
      if (!(c > 0)) {
        dst[pid] = 0;
        continue;
      }
      R acc = 0, wp = 0;
      for (int i = 0; i < diameter; ++i) {
        int nx = x - (half - i);
        if (nx < 0 || nx >= rows) continue;
        for (int j = 0; j < diameter; ++j) {
          int ny = y - (half - j);
          if (ny < 0 || ny >= cols) continue;
          R nv = src[nx * cols + ny];
          if (!(nv > 0)) continue;
          R gi;
          if (sizeof(R) == 8) gi = (R)gaussian_d((double)(nv - c), sI);
          else gi = (R)dyn::range_weight((float)(nv - c), inv2s2, norm);
          R w = gi * gs[(size_t)i * diameter + j];
          acc += nv * w;
          wp += w;
        }
      }
      dst[pid] = acc / wp;
    }
  }
}

// F6: one 2x pyramid step (average of the valid depths of each 2x2 cell)
template <class R>
void downsample_depth(const R* src, int rows, int cols, R* dst) {
  int r2 = rows / 2, c2 = cols / 2;
  for (int y = 0; y < r2; ++y)
    for (int x = 0; x < c2; ++x) {
      R s = 0;
      int n = 0;
      const int oy[4] = {0, 0, 1, 1}, ox[4] = {0, 1, 0, 1};
      for (int k = 0; k < 4; ++k) {
        R d = src[(2 * y + oy[k]) * cols + 2 * x + ox[k]];
        if (d > 0) {
          s += d;
          n++;
        }
      }
      dst[y * c2 + x] = n ? s / (R)n : (R)0;
    }
}
template <class R>
void downsample_intensity(const R* src, int rows, int cols, R* dst) {
  int r2 = rows / 2, c2 = cols / 2;
  for (int y = 0; y < r2; ++y)
    for (int x = 0; x < c2; ++x) {
      const R* a = src + (2 * y) * cols + 2 * x;
      dst[y * c2 + x] = (((a[0] + a[1]) + a[cols]) + a[cols + 1]) * (R)0.25;
    }
}
// gnSolver::Intensity of ColorToFloat (gnSolver.cu:457-459, utils.h:98-102)
template <class R>
inline R intensity_of(const uint8_t* c) {
  float r = (float)c[0] / 255, g = (float)c[1] / 255, b = (float)c[2] / 255;
  return (R)(float)(0.2126 * (double)r + 0.7152 * (double)g + 0.0722 * (double)b);
}

// creatPointCloudKernel (rgbdImage.cu:23-38) + vertextoNormal
// (rgbdImage.cu:126-145: neighbours +-2 columns, +-1 row) with F7.
template <class R>
void maps(const R* depth, const Sensor<R>& s, R* v4, R* n4) {
  int rows = s.rows, cols = s.cols;
  int nt = std::max(1, g_threads);
#pragma omp parallel for num_threads(nt) schedule(static)
  for (int y = 0; y < rows; ++y)
    for (int x = 0; x < cols; ++x) {
      int i = y * cols + x;
      R d = depth[i];
      R* vo = v4 + 4 * (size_t)i;
      R* no = n4 + 4 * (size_t)i;
      no[0] = no[1] = no[2] = no[3] = 0;
      if (!(d > 0)) {
        vo[0] = vo[1] = vo[2] = vo[3] = 0;
        continue;
      }
      V3<R> p = getPoint3d(i, d, s);
      vo[0] = p.x;
      vo[1] = p.y;
      vo[2] = p.z;
      vo[3] = 1;
      if (x - 2 < 0 || x + 2 >= cols || y - 1 < 0 || y + 1 >= rows) continue;
      int il = i - 2, ir = i + 2, iu = i - cols, id = i + cols;
      R dl = depth[il], dr = depth[ir], du = depth[iu], dd = depth[id];
      if (!(dl > 0) || !(dr > 0) || !(du > 0) || !(dd > 0)) continue;
      V3<R> left = getPoint3d(il, dl, s), right = getPoint3d(ir, dr, s);
      V3<R> up = getPoint3d(iu, du, s), down = getPoint3d(id, dd, s);
      V3<R> c = cross(right - left, down - up);
      R dd2 = dot(c, c);
      if (!(dd2 > 0)) continue;
      V3<R> nrm = c * (R(1) / std::sqrt(dd2));
      no[0] = nrm.x;
      no[1] = nrm.y;
      no[2] = nrm.z;
    }
}

template <class R>
inline bool normal_ok(const R* n4, int i) {
  R x = n4[4 * (size_t)i], y = n4[4 * (size_t)i + 1], z = n4[4 * (size_t)i + 2];
  if (std::isnan(x) || std::isnan(y) || std::isnan(z)) return false;
  return !(x == 0 && y == 0 && z == 0);
}

// buildNLSKernel's terms for one source pixel, gnSolver.cu:55-190 (in R)
// with F8: A (6x6, full), b and the residual r; false when the pixel has no
// correspondence.
template <class R>
bool icp_pixel_terms(const R* sd, const R* sn, const R* si, const R* td, const R* tn,
                     const R* ti, const Sensor<R>& s, const dyn_gn_params& g, const M4<R>& T,
                     int idx, R A[36], R b[6], R* res) {
  R dmin = (R)g.icp_min_depth, dmax = (R)g.icp_max_depth;
  R thr = (R)g.normal_cos_thresh;
  R cw = (R)g.color_weight;
  R d = sd[idx];
  if (d < dmin || d > dmax || !normal_ok(sn, idx)) return false;
  V3<R> s_n = v3(sn[4 * (size_t)idx], sn[4 * (size_t)idx + 1], sn[4 * (size_t)idx + 2]);
  V3<R> p = xform(T, getPoint3d(idx, d, s));
  if (!(p.z > 0)) return false;
  int px, py;
  if (!project(p, s, &px, &py)) return false;
  if (px < 0 || py < 0 || px >= s.cols || py >= s.rows) return false;
  int index = py * s.cols + px;
  R tdd = td[index];
  if (tdd < dmin || tdd > dmax || !normal_ok(tn, index)) return false;
  V3<R> nn = v3(tn[4 * (size_t)index], tn[4 * (size_t)index + 1], tn[4 * (size_t)index + 2]);
  R cosT = dot(nn, s_n);
  V3<R> q = getPoint3d(index, tdd, s);
  if (!(std::fabs(cosT) > thr)) return false;
  V3<R> c = cross(p, nn);
  R cn[6] = {c.x, c.y, c.z, nn.x, nn.y, nn.z};
  V3<R> pq = p - q;
  for (int i = 0; i < 6; ++i)
    for (int j = 0; j < 6; ++j) A[i * 6 + j] = cn[i] * cn[j];
  for (int k = 0; k < 6; ++k)
    b[k] = pq.x * (cn[k] * nn.x) + pq.y * (cn[k] * nn.y) + pq.z * (cn[k] * nn.z);
  if (cw != 0) {
    // gnSolver.cu:137-190: J_c = grad(I_t) [ -p^ | I ]
    int il = px >= 1 ? index - 1 : index;
    int iu = py >= 1 ? index - s.cols : index;
    R gx = (ti[index] - ti[il]) / 2;
    R gy = (ti[index] - ti[iu]) / 2;
    R D[3][6] = {{0, p.z, -p.y, 1, 0, 0},
                 {-p.z, 0, p.x, 0, 1, 0},
                 {p.y, -p.x, 0, 0, 0, 1}};
    R Jc[6];
    for (int j = 0; j < 6; ++j) Jc[j] = gx * D[0][j] + gy * D[1][j] + R(0) * D[2][j];
    R ediff = ti[index] - si[idx];
    for (int i = 0; i < 6; ++i)
      for (int j = 0; j < 6; ++j)
        A[i * 6 + j] = (R(1) - cw) * A[i * 6 + j] + (cw * Jc[i]) * Jc[j];
    for (int k = 0; k < 6; ++k) b[k] = (R(1) - cw) * b[k] + (cw * Jc[k]) * ediff;
  }
  *res = dot(pq, nn);
  return true;
}

// The normal equations of a level, sums in double: out[0..20] the upper
// triangle of A, out[21..26] acc_b (= -sum b), out[27] sum r^2, out[28]
// count.
template <class R>
void icp_normal_equations(const R* sd, const R* sn, const R* si, const R* td,
                          const R* tn, const R* ti, const Sensor<R>& s,
                          const dyn_gn_params& g, const M4<R>& T,
                          double out[29]) {
  int n = s.rows * s.cols;
  int nt = std::max(1, g_threads);
  std::vector<double> part((size_t)nt * 29, 0.0);
#pragma omp parallel for num_threads(nt) schedule(static)
  for (int t = 0; t < nt; ++t) {
    double* acc = &part[(size_t)t * 29];
    int lo = (int)((int64_t)n * t / nt), hi = (int)((int64_t)n * (t + 1) / nt);
    for (int idx = lo; idx < hi; ++idx) {
      R A[36], b[6], r;
      if (!icp_pixel_terms(sd, sn, si, td, tn, ti, s, g, T, idx, A, b, &r)) continue;
      int u = 0;
      for (int i = 0; i < 6; ++i)
        for (int j = i; j < 6; ++j) acc[u++] += (double)A[i * 6 + j];
      for (int k = 0; k < 6; ++k) acc[21 + k] -= (double)b[k];
      acc[27] += (double)r * (double)r;
      acc[28] += 1.0;
    }
  }
  for (int k = 0; k < 29; ++k) out[k] = 0;
  for (int t = 0; t < nt; ++t)
    for (int k = 0; k < 29; ++k) out[k] += part[(size_t)t * 29 + k];
}

// The same terms summed as the reference's buildNLSKernel sums them when
// its pixels run one after another: FP32 accumulators of the full 6x6 A and
// of -b, in pixel order (gnSolver.cu:192-193).  Returns the pixel count.
int64_t icp_normal_equations_refsum(const float* sd, const float* sn, const float* si,
                                    const float* td, const float* tn, const float* ti,
                                    const Sensor<float>& s, const dyn_gn_params& g,
                                    const M4<float>& T, float A_out[36], float b_out[6]) {
  for (int j = 0; j < 36; ++j) A_out[j] = 0.0f;
  for (int j = 0; j < 6; ++j) b_out[j] = 0.0f;
  int64_t cnt = 0;
  const int n = s.rows * s.cols;
  for (int idx = 0; idx < n; ++idx) {
    float A[36], b[6], r;
    if (!icp_pixel_terms(sd, sn, si, td, tn, ti, s, g, T, idx, A, b, &r)) continue;
    for (int j = 0; j < 36; ++j) A_out[j] += A[j];
    for (int j = 0; j < 6; ++j) b_out[j] += -b[j];
    ++cnt;
  }
  return cnt;
}

// ------------------------------------------------------------- GN algebra
using dyo_gn::ldlt6;
using dyo_gn::se3_exp;

void matmul4d(const double* A, const double* B, double* C) {
  double t[16];
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) {
      double s = 0;
      for (int k = 0; k < 4; ++k) s += A[i * 4 + k] * B[k * 4 + j];
      t[i * 4 + j] = s;
    }
  std::memcpy(C, t, sizeof(t));
}

// One GN update from accumulated normal equations, gnSolver.cu:389-415.
// Returns true when |delta| <= min_increment (converged).
bool gn_update(const double* acc, const dyn_gn_params& g, int it, double* inc,
               double* prev) {
  double A[36], b[6];
  int u = 0;
  for (int i = 0; i < 6; ++i)
    for (int j = i; j < 6; ++j) {
      A[i * 6 + j] = acc[u];
      A[j * 6 + i] = acc[u];
      ++u;
    }
  for (int k = 0; k < 6; ++k) b[k] = acc[21 + k];
  double mx = A[0];
  for (int k = 1; k < 36; ++k) mx = std::max(mx, A[k]);
  double scaling = 1 / mx;  // :400-402
  for (int k = 0; k < 6; ++k) b[k] *= scaling;
  for (int k = 0; k < 36; ++k) A[k] *= scaling;
  double mx2 = A[0];
  for (int k = 1; k < 36; ++k) mx2 = std::max(mx2, A[k]);
  double alpha = (double)g.regularization * mx2;  // :404-405
  for (int k = 0; k < 6; ++k) A[k * 6 + k] += alpha / it;
  double d[6] = {0, 0, 0, 0, 0, 0};
  if (!ldlt6(A, b, d)) {
    for (int k = 0; k < 6; ++k) d[k] = NAN;
  }
  double ch = 0;
  for (int k = 0; k < 6; ++k) {
    inc[k] += d[k];
    double c = inc[k] - prev[k];
    ch += c * c;
  }
  bool conv = std::fabs(std::sqrt(ch)) <= (double)g.min_increment;
  if (!conv)
    for (int k = 0; k < 6; ++k) prev[k] = inc[k];
  return conv;
}

// gnSolver::solve's loop (gnSolver.cu:340-430) with every level at the
// full-resolution images and the normal equations summed as the reference
// sums them (icp_normal_equations_refsum): xi from zero, iterations 1..N-1
// per level, then the NaN and max_increment guards.  Returns xi in inc.
void gn_solve_refsum(const float* sd, const float* sn, const float* td, const float* tn,
                     const Sensor<float>& s, const dyn_gn_params& g, double inc[6]) {
  double prev[6] = {0, 0, 0, 0, 0, 0};
  for (int k = 0; k < 6; ++k) inc[k] = 0;
  for (int pl = 0; pl < 3; ++pl)
    for (int it = 1; it < g.lvl_iteration_num[pl]; ++it) {
      double Td[16];
      se3_exp(inc, Td);
      M4<float> T;
      for (int k = 0; k < 16; ++k) T.m[k] = (float)Td[k];
      float A[36], b[6];
      icp_normal_equations_refsum(sd, sn, nullptr, td, tn, nullptr, s, g, T, A, b);
      double acc[29];
      int u = 0;
      for (int i = 0; i < 6; ++i)
        for (int j = i; j < 6; ++j) acc[u++] = (double)A[i * 6 + j];
      for (int k = 0; k < 6; ++k) acc[21 + k] = (double)b[k];
      if (gn_update(acc, g, it, inc, prev)) break;
    }
  double sum = 0;
  for (int k = 0; k < 6; ++k) sum += inc[k];
  if (std::isnan(sum) || std::isinf(sum) || sum >= (double)g.max_increment)
    for (int k = 0; k < 6; ++k) inc[k] = 0;
}

int scale_level(int scale) {
  int l = 0;
  while ((1 << l) < scale && l < 7) ++l;
  return l;
}

// ------------------------------------------------------------ the session
template <class R>
struct Session {
  dyn_tsdf_params tp;
  dyn_gn_params gp;
  dyn_bilateral_params bp;
  dyn_sensor sensor;
  Volume<R> vol;
  int frame = 0;
  double pose[16];
  int nlev = 4;
  int rows[4], cols[4];
  Sensor<R> ls[4];
  std::vector<R> raw, filt;
  std::vector<R> sdep[4], snrm[4], sint[4], svtx[4];
  std::vector<R> tdep[4], tnrm[4], tint[4], tvtx[4];
  std::vector<uint8_t> trgb;
  bool have_target = false;

  Session(const dyn_tsdf_params& t, const dyn_gn_params& g,
          const dyn_bilateral_params& b, const dyn_sensor& s)
      : tp(t), gp(g), bp(b), sensor(s), vol(t) {
    for (int i = 0; i < 16; ++i) pose[i] = (i % 5 == 0) ? 1.0 : 0.0;
    for (int l = 0; l < nlev; ++l) {
      dyn_sensor ds;
      dyo_level_sensor(&s, 1 << l, &ds);
      ls[l] = mk_sensor<R>(ds);
      rows[l] = (int)ds.rows;
      cols[l] = (int)ds.cols;
      size_t n = (size_t)rows[l] * cols[l];
      sdep[l].assign(n, 0);
      sint[l].assign(n, 0);
      snrm[l].assign(4 * n, 0);
      svtx[l].assign(4 * n, 0);
      tdep[l].assign(n, 0);
      tint[l].assign(n, 0);
      tnrm[l].assign(4 * n, 0);
      tvtx[l].assign(4 * n, 0);
    }
    raw.assign((size_t)s.rows * s.cols, 0);
    filt.assign((size_t)s.rows * s.cols, 0);
    trgb.assign((size_t)s.rows * s.cols * 3, 0);
  }

  M4<R> pose_r() const { return m4_from<R>(pose); }

  void ingest(const uint16_t* depth, const uint8_t* rgb) {
    size_t n = raw.size();
    for (size_t i = 0; i < n; ++i) raw[i] = (R)depth[i] / (R)sensor.depth_scaler;
    if (bp.enabled)
      bilateral(raw.data(), filt.data(), (int)sensor.rows, (int)sensor.cols,
                bp.diameter, (double)bp.sigma_i, (double)bp.sigma_s);
    else
      filt = raw;
    sdep[0] = filt;
    for (int l = 1; l < nlev; ++l)
      downsample_depth(sdep[l - 1].data(), rows[l - 1], cols[l - 1], sdep[l].data());
    for (size_t i = 0; i < n; ++i) sint[0][i] = rgb ? intensity_of<R>(rgb + 3 * i) : (R)0;
    for (int l = 1; l < nlev; ++l)
      downsample_intensity(sint[l - 1].data(), rows[l - 1], cols[l - 1], sint[l].data());
    for (int l = 0; l < nlev; ++l) maps(sdep[l].data(), ls[l], svtx[l].data(), snrm[l].data());
  }

  void target_from_source() {
    for (int l = 0; l < nlev; ++l) {
      tdep[l] = sdep[l];
      tnrm[l] = snrm[l];
      tvtx[l] = svtx[l];
      tint[l] = sint[l];
    }
    have_target = true;
  }

  void target_from_raycast(int64_t* cnt) {
    M4<R> T = pose_r();
    volume_raycast(vol, T, ls[0], tdep[0].data(), trgb.data(), cnt);
    R maxd = (R)tp.max_sensor_depth;
    size_t n = tdep[0].size();
    for (size_t i = 0; i < n; ++i)
      if (!(tdep[0][i] < maxd)) tdep[0][i] = 0;  // ray missed: invalid
    for (int l = 1; l < nlev; ++l)
      downsample_depth(tdep[l - 1].data(), rows[l - 1], cols[l - 1], tdep[l].data());
    for (size_t i = 0; i < n; ++i) tint[0][i] = intensity_of<R>(&trgb[3 * i]);
    for (int l = 1; l < nlev; ++l)
      downsample_intensity(tint[l - 1].data(), rows[l - 1], cols[l - 1], tint[l].data());
    for (int l = 0; l < nlev; ++l) maps(tdep[l].data(), ls[l], tvtx[l].data(), tnrm[l].data());
    have_target = true;
  }

  // gnSolver::solve, gnSolver.cu:317-438
  void track(dyn_frame_stats* st) {
    double inc[6] = {0, 0, 0, 0, 0, 0}, prev[6] = {0, 0, 0, 0, 0, 0};
    for (int pl = 0; pl < 3; ++pl) {
      int l = scale_level(gp.lvl_scale[pl]);
      int iters = 0;
      for (int it = 1; it < gp.lvl_iteration_num[pl]; ++it) {
        double Td[16];
        se3_exp(inc, Td);
        M4<R> T;
        for (int k = 0; k < 16; ++k) T.m[k] = (R)(float)Td[k];
        if (sizeof(R) == 8)
          for (int k = 0; k < 16; ++k) T.m[k] = (R)Td[k];
        double acc[29];
        icp_normal_equations(sdep[l].data(), snrm[l].data(), sint[l].data(),
                             tdep[l].data(), tnrm[l].data(), tint[l].data(),
                             ls[l], gp, T, acc);
        ++iters;
        if (st) {
          st->icp_inliers[pl] = (int32_t)acc[28];
          st->icp_rms[pl] = acc[28] > 0 ? (float)std::sqrt(acc[27] / acc[28]) : 0.f;
        }
        if (gn_update(acc, gp, it, inc, prev)) break;
      }
      if (st) st->icp_iterations[pl] = iters;
    }
    double s = 0;
    for (int k = 0; k < 6; ++k) s += inc[k];
    bool reset = false;
    if (std::isnan(s) || std::isinf(s)) reset = true;  // :426
    else if (s >= (double)gp.max_increment) reset = true;  // :428
    if (reset)
      for (int k = 0; k < 6; ++k) inc[k] = 0;
    double E[16];
    se3_exp(inc, E);
    if (gp.compose_left) matmul4d(E, pose, pose);  // :429
    else matmul4d(pose, E, pose);
    if (st) {
      st->icp_reset = reset ? 1 : 0;
      for (int k = 0; k < 6; ++k) st->pose_increment[k] = inc[k];
    }
  }

  void integrate_at_pose(int64_t* cnt) {
    M4<R> T = pose_r();
    volume_allocate(vol, raw.data(), ls[0], T, cnt);
    volume_integrate(vol, raw.data(), rgb_keep.empty() ? nullptr : rgb_keep.data(),
                     ls[0], T, cnt);
  }
  std::vector<uint8_t> rgb_keep;

  void frame_step(const uint16_t* depth, const uint8_t* rgb, dyn_frame_stats* st) {
    int64_t cnt[DYO_C_N] = {0};
    if (st) {
      std::memset(st, 0, sizeof(*st));
      st->frame_index = frame;
    }
    ingest(depth, rgb);
    if (rgb) rgb_keep.assign(rgb, rgb + (size_t)sensor.rows * sensor.cols * 3);
    else rgb_keep.clear();
    if (frame > 0 && have_target) track(st);
    integrate_at_pose(cnt);
    if (gp.mode == 1) target_from_raycast(cnt);
    else target_from_source();
    if (st) {
      st->blocks_total = (int32_t)vol.nalloc;
      st->blocks_new = (int32_t)cnt[DYO_C_NEW_BLOCKS];
      st->blocks_visible = (int32_t)cnt[DYO_C_VISIBLE];
      st->unique_blocks_probed = (int32_t)cnt[DYO_C_UNIQUE_PROBED];
      st->bucket_full = (int32_t)cnt[DYO_C_BUCKET_FULL];
      st->heap_exhausted = (int32_t)cnt[DYO_C_HEAP_EXHAUSTED];
      st->dda_overruns = (int32_t)cnt[DYO_C_DDA_OVERRUNS];
      st->raycast_overruns = (int32_t)cnt[DYO_C_RAYCAST_OVERRUNS];
    }
    ++frame;
  }
};

struct AnyVolume {
  int fp64;
  void* v;
};
struct AnySession {
  int fp64;
  void* s;
  AnyVolume vol;
};

template <class R>
static std::vector<R> to_r(const float* d, size_t n) {
  return std::vector<R>(d, d + n);
}

template <class R>
static int64_t download(Volume<R>& V, int32_t* coords, uint8_t* rgbw, R* sdf,
                        int64_t cap) {
  int bs3 = V.p.block_size * V.p.block_size * V.p.block_size;
  int64_t n = std::min<int64_t>(cap, V.nalloc);
  for (int64_t b = 0; b < n; ++b) {
    if (coords) {
      coords[3 * b] = V.bx[b];
      coords[3 * b + 1] = V.by[b];
      coords[3 * b + 2] = V.bz[b];
    }
    for (int k = 0; k < bs3; ++k) {
      const Voxel<R>& vx = V.vox[(size_t)b * bs3 + k];
      if (rgbw) {
        uint8_t* o = rgbw + 4 * ((size_t)b * bs3 + k);
        o[0] = vx.c[0];
        o[1] = vx.c[1];
        o[2] = vx.c[2];
        o[3] = vx.w;
      }
      if (sdf) sdf[(size_t)b * bs3 + k] = vx.sdf;
    }
  }
  return V.nalloc;
}
// The inverse of download for FP32 volumes: each block allocated in turn
// (heap indices follow the order given) and its voxels set.  Returns the
// blocks placed; stops at the first that does not fit.
static int64_t upload(Volume<float>& V, const int32_t* coords, const uint8_t* rgbw,
                      const float* sdf, int64_t n) {
  const int bs3 = V.p.block_size * V.p.block_size * V.p.block_size;
  for (int64_t b = 0; b < n; ++b) {
    const int x = coords[3 * b], y = coords[3 * b + 1], z = coords[3 * b + 2];
    if (V.allocate(x, y, z) < 0) return b;
    const int ptr = V.find(x, y, z);
    for (int k = 0; k < bs3; ++k) {
      Voxel<float>& vx = V.vox[(size_t)ptr * bs3 + k];
      const uint8_t* c = rgbw + 4 * ((size_t)b * bs3 + k);
      vx.c[0] = c[0];
      vx.c[1] = c[1];
      vx.c[2] = c[2];
      vx.w = c[3];
      vx.sdf = sdf[(size_t)b * bs3 + k];
    }
  }
  return n;
}
}  // namespace

extern "C" {

void dyo_set_threads(int n) { g_threads = n < 1 ? 1 : n; }
int dyo_get_threads(void) { return g_threads; }

int32_t dyo_hash(int32_t x, int32_t y, int32_t z, int32_t nb, int32_t bsz) {
  return hash_slot(x, y, z, nb, bsz);
}

int32_t dyo_dda_blocks(const float start[3], const float point[3], float trunc,
                       float block_size, int32_t cap, int32_t* out_xyz, int32_t max_out) {
  int32_t n = 0;
  bool ok = dda_ray(v3(start[0], start[1], start[2]), v3(point[0], point[1], point[2]),
                    trunc, block_size, cap, [&](int x, int y, int z) {
                      if (n < max_out) {
                        out_xyz[3 * n] = x;
                        out_xyz[3 * n + 1] = y;
                        out_xyz[3 * n + 2] = z;
                      }
                      ++n;
                    });
  return ok ? n : -n;
}

void dyo_merge_voxel(uint8_t rgbw[4], float* sdf, float new_sdf, const uint8_t new_rgb[3],
                     int32_t new_w, int32_t max_w) {
  Voxel<float> v;
  v.c[0] = rgbw[0];
  v.c[1] = rgbw[1];
  v.c[2] = rgbw[2];
  v.w = rgbw[3];
  v.sdf = *sdf;
  merge_voxel(v, new_sdf, new_rgb, (uint8_t)new_w, max_w);
  rgbw[0] = v.c[0];
  rgbw[1] = v.c[1];
  rgbw[2] = v.c[2];
  rgbw[3] = v.w;
  *sdf = v.sdf;
}

void dyo_level_sensor(const dyn_sensor* s, int32_t scale, dyn_sensor* out) {
  *out = *s;
  out->rows = s->rows / (uint32_t)scale;
  out->cols = s->cols / (uint32_t)scale;
  out->fx = s->fx / (float)scale;
  out->fy = s->fy / (float)scale;
  out->cx = (s->cx + 0.5f) / (float)scale - 0.5f;
  out->cy = (s->cy + 0.5f) / (float)scale - 0.5f;
}

void dyo_depth_from_raw(const uint16_t* raw, int64_t n, float scaler, float* out) {
  for (int64_t i = 0; i < n; ++i) out[i] = (float)raw[i] / scaler;
}
void dyo_bilateral(const float* src, float* dst, int32_t rows, int32_t cols,
                   const dyn_bilateral_params* p) {
  bilateral<float>(src, dst, rows, cols, p->diameter, (double)p->sigma_i,
                   (double)p->sigma_s);
}
void dyo_downsample_depth(const float* src, int32_t rows, int32_t cols, float* dst) {
  downsample_depth<float>(src, rows, cols, dst);
}
void dyo_intensity(const uint8_t* rgb, int64_t n, float* out) {
  for (int64_t i = 0; i < n; ++i) out[i] = intensity_of<float>(rgb + 3 * i);
}
void dyo_downsample_intensity(const float* src, int32_t rows, int32_t cols, float* dst) {
  downsample_intensity<float>(src, rows, cols, dst);
}
void dyo_maps(const float* depth, const dyn_sensor* level, float* v4, float* n4) {
  maps<float>(depth, mk_sensor<float>(*level), v4, n4);
}
void dyo_icp_normal_equations(const float* sd, const float* sn, const float* si,
                              const float* td, const float* tn, const float* ti,
                              const dyn_sensor* level, const dyn_gn_params* gn,
                              const float T[16], double out[29]) {
  icp_normal_equations<float>(sd, sn, si, td, tn, ti, mk_sensor<float>(*level),
                              *gn, m4_from<float>(T), out);
}
int64_t dyo_icp_normal_equations_refsum(const float* sd, const float* sn, const float* si,
                                        const float* td, const float* tn, const float* ti,
                                        const dyn_sensor* level, const dyn_gn_params* gn,
                                        const float T[16], float A_out[36], float b_out[6]) {
  return icp_normal_equations_refsum(sd, sn, si, td, tn, ti, mk_sensor<float>(*level), *gn,
                                     m4_from<float>(T), A_out, b_out);
}
void dyo_gn_solve_refsum(const float* sd, const float* sn, const float* td, const float* tn,
                         const dyn_sensor* level, const dyn_gn_params* gn, double inc_out[6]) {
  gn_solve_refsum(sd, sn, td, tn, mk_sensor<float>(*level), *gn, inc_out);
}
void dyo_inverse4(const float m[16], float out[16]) {
  M4<float> r = inverse4(m4_from<float>(m));
  std::memcpy(out, r.m, sizeof(r.m));
}
void dyo_se3_exp(const double xi[6], double out[16]) { se3_exp(xi, out); }
int dyo_ldlt_solve6(const double A[36], const double b[6], double x[6]) {
  return ldlt6(A, b, x);
}

void* dyo_volume_create(const dyn_tsdf_params* p, int32_t fp64) {
  AnyVolume* a = new AnyVolume;
  a->fp64 = fp64;
  a->v = fp64 ? (void*)new Volume<double>(*p) : (void*)new Volume<float>(*p);
  return a;
}
void dyo_volume_destroy(void* v) {
  AnyVolume* a = (AnyVolume*)v;
  if (!a) return;
  if (a->fp64) delete (Volume<double>*)a->v;
  else delete (Volume<float>*)a->v;
  delete a;
}


void dyo_volume_allocate(void* v, const float* depth, const dyn_sensor* s,
                         const float pose[16], int64_t cnt[DYO_C_N]) {
  AnyVolume* a = (AnyVolume*)v;
  size_t n = (size_t)s->rows * s->cols;
  if (a->fp64) {
    std::vector<double> d = to_r<double>(depth, n);
    volume_allocate(*(Volume<double>*)a->v, d.data(), mk_sensor<double>(*s),
                    m4_from<double>(pose), cnt);
  } else {
    volume_allocate(*(Volume<float>*)a->v, depth, mk_sensor<float>(*s),
                    m4_from<float>(pose), cnt);
  }
}
void dyo_volume_integrate(void* v, const float* depth, const uint8_t* rgb,
                          const dyn_sensor* s, const float pose[16],
                          int64_t cnt[DYO_C_N]) {
  AnyVolume* a = (AnyVolume*)v;
  size_t n = (size_t)s->rows * s->cols;
  if (a->fp64) {
    std::vector<double> d = to_r<double>(depth, n);
    volume_integrate(*(Volume<double>*)a->v, d.data(), rgb, mk_sensor<double>(*s),
                     m4_from<double>(pose), cnt);
  } else {
    volume_integrate(*(Volume<float>*)a->v, depth, rgb, mk_sensor<float>(*s),
                     m4_from<float>(pose), cnt);
  }
}
void dyo_volume_raycast(void* v, const float pose[16], const dyn_sensor* s,
                        float* depth_out, uint8_t* rgb_out, int64_t cnt[DYO_C_N]) {
  AnyVolume* a = (AnyVolume*)v;
  size_t n = (size_t)s->rows * s->cols;
  if (a->fp64) {
    std::vector<double> d(n);
    volume_raycast(*(Volume<double>*)a->v, m4_from<double>(pose),
                   mk_sensor<double>(*s), d.data(), rgb_out, cnt);
    for (size_t i = 0; i < n; ++i) depth_out[i] = (float)d[i];
  } else {
    volume_raycast(*(Volume<float>*)a->v, m4_from<float>(pose),
                   mk_sensor<float>(*s), depth_out, rgb_out, cnt);
  }
}
int64_t dyo_volume_num_blocks(void* v) {
  AnyVolume* a = (AnyVolume*)v;
  return a->fp64 ? ((Volume<double>*)a->v)->nalloc : ((Volume<float>*)a->v)->nalloc;
}

int64_t dyo_mesh_vertices(void* v, const float lo[3], const float hi[3], float* out,
                          int64_t cap) {
  AnyVolume* a = (AnyVolume*)v;
  if (a->fp64) return -1;
  return mesh_vertices(*(Volume<float>*)a->v, lo, hi, out, cap);
}
int64_t dyo_mesh_triangles(void* v, const float lo[3], const float hi[3], float* out,
                           int64_t cap) {
  AnyVolume* a = (AnyVolume*)v;
  if (a->fp64) return -1;
  return mesh_triangles(*(Volume<float>*)a->v, lo, hi, out, cap);
}
int64_t dyo_volume_download(void* v, int32_t* coords, uint8_t* rgbw,
                            void* sdf_out, int64_t cap) {
  AnyVolume* a = (AnyVolume*)v;
  if (a->fp64)
    return download(*(Volume<double>*)a->v, coords, rgbw, (double*)sdf_out, cap);
  return download(*(Volume<float>*)a->v, coords, rgbw, (float*)sdf_out, cap);
}

int64_t dyo_volume_upload(void* v, const int32_t* coords, const uint8_t* rgbw,
                          const float* sdf, int64_t n) {
  AnyVolume* a = (AnyVolume*)v;
  if (a->fp64) return -1;
  return upload(*(Volume<float>*)a->v, coords, rgbw, sdf, n);
}

void* dyo_session_create(const dyn_tsdf_params* t, const dyn_gn_params* g,
                         const dyn_bilateral_params* b, const dyn_sensor* s,
                         int32_t fp64) {
  AnySession* a = new AnySession;
  a->fp64 = fp64;
  if (fp64) {
    Session<double>* S = new Session<double>(*t, *g, *b, *s);
    a->s = S;
    a->vol.fp64 = 1;
    a->vol.v = &S->vol;
  } else {
    Session<float>* S = new Session<float>(*t, *g, *b, *s);
    a->s = S;
    a->vol.fp64 = 0;
    a->vol.v = &S->vol;
  }
  return a;
}
void dyo_session_destroy(void* s) {
  AnySession* a = (AnySession*)s;
  if (!a) return;
  if (a->fp64) delete (Session<double>*)a->s;
  else delete (Session<float>*)a->s;
  delete a;
}
void dyo_session_set_pose(void* s, const float pose[16]) {
  AnySession* a = (AnySession*)s;
  double* P = a->fp64 ? ((Session<double>*)a->s)->pose : ((Session<float>*)a->s)->pose;
  for (int i = 0; i < 16; ++i) P[i] = (double)pose[i];
}
void dyo_session_get_pose_f64(void* s, double pose[16]) {
  AnySession* a = (AnySession*)s;
  double* P = a->fp64 ? ((Session<double>*)a->s)->pose : ((Session<float>*)a->s)->pose;
  for (int i = 0; i < 16; ++i) pose[i] = P[i];
}
void dyo_session_get_pose(void* s, float pose[16]) {
  double P[16];
  dyo_session_get_pose_f64(s, P);
  for (int i = 0; i < 16; ++i) pose[i] = (float)P[i];
}
void dyo_session_frame(void* s, const uint16_t* depth, const uint8_t* rgb,
                       float pose_out[16], dyn_frame_stats* st) {
  AnySession* a = (AnySession*)s;
  if (a->fp64) ((Session<double>*)a->s)->frame_step(depth, rgb, st);
  else ((Session<float>*)a->s)->frame_step(depth, rgb, st);
  if (pose_out) dyo_session_get_pose(s, pose_out);
}
void dyo_session_integrate_with_pose(void* s, const uint16_t* depth,
                                     const uint8_t* rgb, const float pose[16]) {
  AnySession* a = (AnySession*)s;
  dyo_session_set_pose(s, pose);
  int64_t cnt[DYO_C_N] = {0};
  if (a->fp64) {
    Session<double>* S = (Session<double>*)a->s;
    S->ingest(depth, rgb);
    if (rgb) S->rgb_keep.assign(rgb, rgb + (size_t)S->sensor.rows * S->sensor.cols * 3);
    else S->rgb_keep.clear();
    S->integrate_at_pose(cnt);
    S->target_from_raycast(cnt);
    S->frame++;
  } else {
    Session<float>* S = (Session<float>*)a->s;
    S->ingest(depth, rgb);
    if (rgb) S->rgb_keep.assign(rgb, rgb + (size_t)S->sensor.rows * S->sensor.cols * 3);
    else S->rgb_keep.clear();
    S->integrate_at_pose(cnt);
    S->target_from_raycast(cnt);
    S->frame++;
  }
}
void* dyo_session_volume(void* s) { return &((AnySession*)s)->vol; }

int dyo_session_image(void* s, int32_t which, int32_t level, void* out, int64_t bytes) {
  AnySession* a = (AnySession*)s;
  if (a->fp64 || level < 0 || level > 3) return 0;
  Session<float>* S = (Session<float>*)a->s;
  const void* src = nullptr;
  size_t n = 0;
  switch (which) {
    case 0: src = S->raw.data(); n = S->raw.size() * 4; break;
    case 1: src = S->filt.data(); n = S->filt.size() * 4; break;
    case 2: src = S->sdep[level].data(); n = S->sdep[level].size() * 4; break;
    case 3: src = S->svtx[level].data(); n = S->svtx[level].size() * 4; break;
    case 4: src = S->snrm[level].data(); n = S->snrm[level].size() * 4; break;
    case 5: src = S->tdep[level].data(); n = S->tdep[level].size() * 4; break;
    case 6: src = S->tvtx[level].data(); n = S->tvtx[level].size() * 4; break;
    case 7: src = S->tnrm[level].data(); n = S->tnrm[level].size() * 4; break;
    case 8: src = S->trgb.data(); n = S->trgb.size(); break;
    case 9: src = S->sint[level].data(); n = S->sint[level].size() * 4; break;
    case 10: src = S->tint[level].data(); n = S->tint[level].size() * 4; break;
    default: return 0;
  }
  if ((int64_t)n > bytes) return 0;
  std::memcpy(out, src, n);
  return 1;
}

}  // extern "C"

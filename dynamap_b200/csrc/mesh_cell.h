// mesh_cell.h -- the arithmetic of one cell of the mesh extraction, shared by
// the CUDA kernels (mesh.cu) and a host build of the same source that the
// tests run against the oracle.  Plain C++ plus DYN_HD qualifiers; no CUDA
// types.
//
// The walk is MeshExtractor::ExtractMesh's (meshExtractor.cu:364-407): a
// grid of cells at lo + i * vs (i < n, n = (int)(|lo - hi| / vs * 2) per
// axis), each cell's eight corners at +-vs/2, each corner sampled by
// TrilinearInterpolation (:22-93), which gives up at the first unobserved
// voxel; then the cube index, the cut edges' vertices by VertexInterpolation
// (:95-121) coloured by the cell's centre voxel, and the triangles of this
// project's marching-cubes table (mc_tables.h).  Every float operation is
// the reference's, in its order; callers compile without FMA contraction.
//
// A Sampler supplies two things: index(p), the global voxel index of world
// coordinate p on one axis (WorldToGlobalVoxelHashing, tsdf.cu:189-193),
// and fetch(gx, gy, gz), the voxel there (weight 0 where unobserved or not
// allocated).
#pragma once

#include <math.h>

#if defined(__CUDACC__)
#define DYN_HD __host__ __device__ __forceinline__
#else
#define DYN_HD inline
#endif

namespace dyn {
namespace mesh {

// A voxel as the 8-byte FP32 layout: r | g << 8 | b << 16 | weight << 24,
// and the sdf in metres.
struct VoxelBits {
  unsigned rgbw;
  float sdf;
};

struct Grid {
  float lo[3];
  int n[3];    // cells per axis
  float vs;    // voxel size
  float half;  // vs / 2
  float inv;   // 1 / vs, IEEE
};

// Cells per axis as the reference's int3 grid_size: (int)(|lo - hi| / vs * 2);
// false when the box is not finite, inverted to NaN, or too large for an
// int (the reference overflows there).
DYN_HD bool make_grid(const float lo[3], const float hi[3], float vs, Grid* g) {
  if (!(vs > 0.0f)) return false;
  for (int a = 0; a < 3; ++a) {
    const float size = fabsf(lo[a] - hi[a]);
    const float c = size / vs * 2.0f;
    if (!(c >= 0.0f) || !(c < 16777216.0f)) return false;  // NaN, inf, > 2^24 cells
    g->lo[a] = lo[a];
    g->n[a] = (int)c;
  }
  g->vs = vs;
  g->half = vs / 2.0f;
  g->inv = 1.0f / vs;
  return true;
}

// World coordinate of cell i on an axis (ExtractMeshKernel, :389-392).
DYN_HD float cell_coord(const Grid& g, int axis, int i) {
  return (float)i * g.vs + g.lo[axis];
}

// The voxel index of the first sample of corner 3, (-,-,-): the smallest
// index any of the cell's 64 samples has on that axis (every step from the
// cell coordinate to a sample is monotone), so a cell that meshes has this
// voxel observed, hence its block allocated.
template <class S>
DYN_HD int key_index(const Grid& g, const S& s, int axis, int i) {
  const float p = cell_coord(g, axis, i) + (-g.half);
  const float dual = p - g.vs / 2.0f;
  return s.index(dual + 0.0f);
}

// The cells [first, last) of one axis whose key voxel lies in block b (block
// size 8): key_index is non-decreasing in i, so both ends are lower bounds.
template <class S>
DYN_HD int key_lower_bound(const Grid& g, const S& s, int axis, int target) {
  int lo = 0, hi = g.n[axis];
  while (lo < hi) {
    const int mid = lo + (hi - lo) / 2;
    if (key_index(g, s, axis, mid) < target) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

// TrilinearInterpolation (:22-93) at p; false at the first unobserved voxel.
template <class S>
DYN_HD bool corner_sdf(const Grid& g, const S& s, float px, float py, float pz, float* dist) {
  const float vs = g.vs;
  const float dx = px - vs / 2.0f, dy = py - vs / 2.0f, dz = pz - vs / 2.0f;
  const float vx = px * g.inv, vy = py * g.inv, vz = pz * g.inv;
  const float wx = vx - floorf(vx), wy = vy - floorf(vy), wz = vz - floorf(vz);
  const int ix[2] = {s.index(dx + 0.0f), s.index(dx + vs)};
  const int iy[2] = {s.index(dy + 0.0f), s.index(dy + vs)};
  const int iz[2] = {s.index(dz + 0.0f), s.index(dz + vs)};
  const int off[8][3] = {{0, 0, 0}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1},
                         {1, 1, 0}, {0, 1, 1}, {1, 0, 1}, {1, 1, 1}};
  float d = 0.0f;
#if defined(__CUDA_ARCH__)
#pragma unroll
#endif
  for (int k = 0; k < 8; ++k) {
    const int ox = off[k][0], oy = off[k][1], oz = off[k][2];
    const VoxelBits v = s.fetch(ix[ox], iy[oy], iz[oz]);
    if ((v.rgbw >> 24) == 0u) return false;
    const float a = ox ? wx : 1.0f - wx;
    const float b = oy ? wy : 1.0f - wy;
    const float c = oz ? wz : 1.0f - wz;
    d += a * b * c * v.sdf;
  }
  *dist = d;
  return true;
}

// Corner k of the cube index (ExtractMeshAtPosition, :126-214): offsets of
// +-vs/2 per axis, 1 meaning +; cube bit k set when corner k is below zero.
DYN_HD int corner_axis(int k, int axis) {
  // (0,1,0) (1,1,0) (1,0,0) (0,0,0) (0,1,1) (1,1,1) (1,0,1) (0,0,1)
  const unsigned bits = axis == 0 ? 0x66u : axis == 1 ? 0x33u : 0xF0u;
  return (int)((bits >> k) & 1u);
}
DYN_HD void corner_pos(const Grid& g, const float pos[3], int k, float p[3]) {
  for (int a = 0; a < 3; ++a) p[a] = pos[a] + (corner_axis(k, a) ? g.half : -g.half);
}
// Cube edges 0..11: their corner pairs (0,1) (1,2) (2,3) (3,0) (4,5) (5,6)
// (6,7) (7,4) (0,4) (1,5) (2,6) (3,7).
DYN_HD int edge_end(int e, int which) {
  if (e < 8) {
    const int base = e < 4 ? 0 : 4;
    return which ? base + ((e + 1) & 3) : e;
  }
  return which ? e - 4 : e - 8;
}

// The cell (ix, iy, iz): its centre, its corner distances and cube index.
// Returns the cube index, or -1 when a corner is unobserved.
template <class S>
DYN_HD int cell_cube(const Grid& g, const S& s, int ix, int iy, int iz, float pos[3],
                     float d[8]) {
  pos[0] = cell_coord(g, 0, ix);
  pos[1] = cell_coord(g, 1, iy);
  pos[2] = cell_coord(g, 2, iz);
  int cube = 0;
  for (int k = 0; k < 8; ++k) {
    float p[3];
    corner_pos(g, pos, k, p);
    if (!corner_sdf(g, s, p[0], p[1], p[2], &d[k])) return -1;
    if (d[k] < 0.0f) cube |= 1 << k;
  }
  return cube;
}

// Triangles of a cube index in the table (rows of edge triples, -1 ended).
DYN_HD int cube_triangles(const signed char* row, int width) {
  int n = 0;
  while (3 * n + 2 < width && row[3 * n] >= 0) ++n;
  return n;
}

// VertexInterpolation (:95-121) on edge e of the cell: {x, y, z, r, g, b},
// the colour the centre voxel's (rgb, 0..255), scaled to 0..1 as the
// reference's Vertex colour.
DYN_HD void edge_vertex(const Grid& g, const float pos[3], const float d[8], unsigned rgb,
                        int e, float out[6]) {
  const int a = edge_end(e, 0), b = edge_end(e, 1);
  float p1[3], p2[3];
  corner_pos(g, pos, a, p1);
  corner_pos(g, pos, b, p2);
  const float d1 = d[a], d2 = d[b];
  const int c[3] = {(int)(rgb & 0xffu), (int)((rgb >> 8) & 0xffu), (int)((rgb >> 16) & 0xffu)};
  const float* q = p1;
  bool end = true;
  if (fabsf(0.0f - d1) < 0.00001f) q = p1;
  else if (fabsf(0.0f - d2) < 0.00001f) q = p2;
  else if (fabsf(d1 - d2) < 0.00001f) q = p1;
  else end = false;
  if (end) {
    for (int k = 0; k < 3; ++k) {
      out[k] = q[k];
      out[3 + k] = (float)c[k] * (1.0f / 255.f);
    }
    return;
  }
  const float mu = (0.0f - d1) / (d2 - d1);
  for (int k = 0; k < 3; ++k) {
    out[k] = p1[k] + mu * (p2[k] - p1[k]);
    out[3 + k] = (float)((float)c[k] + mu * (float)(c[k] - c[k])) / 255.f;
  }
}

}  // namespace mesh
}  // namespace dyn

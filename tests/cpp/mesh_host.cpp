// Host build of the mesh extraction's per-block walk (dynamap_b200/csrc/
// mesh.cu) over the same mesh_cell.h arithmetic, for the CPU tests: the
// kernel's block-driven cell selection, its tile staging with the global
// fallback and its output order, run serially on a volume given as blocks.
// Compile with -ffp-contract=off (the library builds with -fmad=false).
#include <cmath>
#include <cstdint>
#include <cstring>
#include <unordered_map>
#include <vector>

#include "../../dynamap_b200/csrc/mc_tables.h"
#include "../../dynamap_b200/csrc/mesh_cell.h"

namespace {

struct Key {
  int x, y, z;
  bool operator==(const Key& o) const { return x == o.x && y == o.y && z == o.z; }
};
struct KeyHash {
  size_t operator()(const Key& k) const {
    return ((size_t)(unsigned)k.x * 73856093u) ^ ((size_t)(unsigned)k.y * 19349669u) ^
           ((size_t)(unsigned)k.z * 83492791u);
  }
};

struct Blocks {
  std::unordered_map<Key, int, KeyHash> ptr;
  const uint8_t* rgbw;  // n * 512 * 4
  const float* sdf;     // n * 512
  float vs;
  dyn::mesh::VoxelBits voxel(int gx, int gy, int gz) const {
    const Key k{gx >> 3, gy >> 3, gz >> 3};  // floor division by 8
    auto it = ptr.find(k);
    dyn::mesh::VoxelBits b{0u, 0.0f};
    if (it == ptr.end()) return b;
    const size_t i = (size_t)it->second * 512 + (size_t)(((gx & 7) << 6) | ((gy & 7) << 3) | (gz & 7));
    const uint8_t* c = rgbw + 4 * i;
    b.rgbw = (unsigned)c[0] | ((unsigned)c[1] << 8) | ((unsigned)c[2] << 16) | ((unsigned)c[3] << 24);
    b.sdf = sdf[i];
    return b;
  }
};

constexpr int kTile = 11;

// The kernel's TileSampler: staged tile from (ox, oy, oz), else the volume;
// the voxel index by the reference's expression (tsdf.cu:189-193).
struct HostSampler {
  const Blocks* B;
  const dyn::mesh::VoxelBits* tile;
  int ox, oy, oz;
  int index(float p) const {
    const float sg = (float)((p > 0.0f) - (p < 0.0f));
    return (int)(p / B->vs + sg * 0.5f);
  }
  dyn::mesh::VoxelBits fetch(int gx, int gy, int gz) const {
    const unsigned tx = (unsigned)(gx - ox), ty = (unsigned)(gy - oy), tz = (unsigned)(gz - oz);
    if (tx < (unsigned)kTile && ty < (unsigned)kTile && tz < (unsigned)kTile)
      return tile[(tx * kTile + ty) * kTile + tz];
    return B->voxel(gx, gy, gz);
  }
};

}  // namespace

extern "C" {

// Triangles (18 floats each) of the box [lo, hi] in the kernel's order;
// returns the count (at most cap written), -1 for an invalid box.
int64_t mesh_host_extract(const int32_t* coords, const uint8_t* rgbw, const float* sdf,
                          int64_t n, float vs, const float lo[3], const float hi[3], float* out,
                          int64_t cap) {
  dyn::mesh::Grid g;
  if (!dyn::mesh::make_grid(lo, hi, vs, &g)) return -1;
  Blocks B;
  B.rgbw = rgbw;
  B.sdf = sdf;
  B.vs = vs;
  for (int64_t i = 0; i < n; ++i) B.ptr[Key{coords[3 * i], coords[3 * i + 1], coords[3 * i + 2]}] = (int)i;
  std::vector<dyn::mesh::VoxelBits> tile((size_t)kTile * kTile * kTile);
  int64_t total = 0;
  if (g.n[0] == 0 || g.n[1] == 0 || g.n[2] == 0) return 0;
  for (int64_t blk = 0; blk < n; ++blk) {
    const int b[3] = {coords[3 * blk], coords[3 * blk + 1], coords[3 * blk + 2]};
    HostSampler S{&B, tile.data(), 8 * b[0], 8 * b[1], 8 * b[2]};
    int range[3][2];
    for (int t = 0; t < 6; ++t)
      range[t >> 1][t & 1] = dyn::mesh::key_lower_bound(g, S, t >> 1, 8 * b[t >> 1] + 8 * (t & 1));
    const int nx = range[0][1] - range[0][0], ny = range[1][1] - range[1][0],
              nz = range[2][1] - range[2][0];
    if (nx <= 0 || ny <= 0 || nz <= 0) continue;
    for (int i = 0; i < kTile * kTile * kTile; ++i) {
      const int tx = i / (kTile * kTile), ty = (i / kTile) % kTile, tz = i % kTile;
      tile[i] = B.voxel(8 * b[0] + tx, 8 * b[1] + ty, 8 * b[2] + tz);
    }
    const long long ncell = (long long)nx * ny * nz;
    for (long long c = 0; c < ncell; ++c) {
      const int ix = range[0][0] + (int)(c % nx), iy = range[1][0] + (int)((c / nx) % ny),
                iz = range[2][0] + (int)(c / ((long long)nx * ny));
      float pos[3], d[8];
      const int cube = dyn::mesh::cell_cube(g, S, ix, iy, iz, pos, d);
      if (cube <= 0 || cube >= 255) continue;
      const signed char* row = dyn::kMcTriangles[cube];
      const int ntri = dyn::mesh::cube_triangles(row, dyn::kMcMaxTriIdx);
      const dyn::mesh::VoxelBits centre = S.fetch(S.index(pos[0]), S.index(pos[1]), S.index(pos[2]));
      for (int j = 0; j < ntri; ++j, ++total) {
        if (total >= cap) continue;
        for (int k = 0; k < 3; ++k)
          dyn::mesh::edge_vertex(g, pos, d, centre.rgbw & 0xffffffu, row[3 * j + k],
                                 out + 18 * total + 6 * k);
      }
    }
  }
  return total;
}

}  // extern "C"

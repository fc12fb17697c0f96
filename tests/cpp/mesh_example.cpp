// The reference driver's mesh step (src/dynaMap.cpp:306-318) through the
// C++ drop-in: frames integrated at their poses by builder::buildModelGT,
// then builder::ExtractMesh over a box and Mesh::SaveToFile.
//   mesh_example FRAMES OBJ lx ly lz ux uy uz
// FRAMES as tests/cpp/dropin_example.cpp reads it; prints the triangle count.
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "builder/builder.h"

using namespace DynaMap;

int main(int argc, char** argv) {
  if (argc != 9) return 2;
  FILE* f = std::fopen(argv[1], "rb");
  if (!f) return 2;
  int rows, cols, n;
  float fx, fy, cx, cy, sc;
  if (std::fscanf(f, "%d %d %f %f %f %f %f %d\n", &rows, &cols, &fx, &fy, &cx, &cy, &sc, &n) != 8)
    return 2;
  std::vector<uint16_t> depth((size_t)rows * cols * n);
  std::vector<float> poses((size_t)16 * n);
  if (std::fread(depth.data(), 2, depth.size(), f) != depth.size()) return 2;
  if (std::fread(poses.data(), 4, poses.size(), f) != poses.size()) return 2;
  std::fclose(f);
  rgbdSensor s;
  s.rows = rows;
  s.cols = cols;
  s.f = {fx, fy};
  s.c = {cx, cy};
  s.depthScaler = sc;
  tsdf::tsdfProperties tp;
  tp.voxelSize = 0.008f;
  tp.numBuckets = 1 << 16;
  tp.numBlocks = 1 << 15;
  tp.truncationDistance = 0.032f;
  tp.maxSensorDepth = 3.0f;
  tp.minSensorDepth = 0.15f;
  solver::Properties op;
  gaussianKernal k;
  builder b;
  b.init(tp, op, s, k);
  for (int i = 0; i < n; ++i)
    b.buildModelGT(&depth[(size_t)i * rows * cols], nullptr,
                   Matrix4f::from_row_major(&poses[(size_t)16 * i]));
  geometry::float3_ lo{(float)std::atof(argv[3]), (float)std::atof(argv[4]),
                       (float)std::atof(argv[5])};
  geometry::float3_ hi{(float)std::atof(argv[6]), (float)std::atof(argv[7]),
                       (float)std::atof(argv[8])};
  geometry::Mesh mesh = b.ExtractMesh(lo, hi);
  const int saved = mesh.SaveToFile(argv[2]);
  std::printf("triangles %u saved %d\n", mesh.num_triangles_, saved);
  return 0;
}

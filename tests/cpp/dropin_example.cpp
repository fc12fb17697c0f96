// Exercises the C++ drop-in classes (include/builder, include/geometry,
// include/solver) the way the reference's driver uses builder
// (src/dynaMap.cpp:218-301): init, per-frame buildModelLS, GenerateDepth.
// Reads frames from a raw file written by the test: header
// "rows cols fx fy cx cy scaler nframes" then nframes u16 depth images and
// nframes*16 float row-major ground-truth poses.
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "builder/builder.h"

using namespace DynaMap;

int main(int argc, char** argv) {
  if (argc < 2) return 2;
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
  op.lvlIterationNum[0] = 10;
  op.lvlIterationNum[1] = 5;
  op.lvlIterationNum[2] = 4;
  op.icpMaxDepth = 3.0f;
  gaussianKernal k;
  builder b;
  b.init(tp, op, s, k);
  b.setInitialPose(Matrix4f::from_row_major(&poses[0]));
  for (int i = 0; i < n; ++i) b.buildModelLS(&depth[(size_t)i * rows * cols], nullptr, 1);
  Matrix4f P = b.getCurrentPose();
  const float* g = &poses[(size_t)16 * (n - 1)];
  double dt = 0;
  for (int r = 0; r < 3; ++r) dt += (P(r, 3) - g[r * 4 + 3]) * (P(r, 3) - g[r * 4 + 3]);
  const float* d = b.GenerateDepth(cols, rows);
  int hits = 0;
  for (int i = 0; i < rows * cols; ++i) hits += (d[i] > 0 && d[i] < tp.maxSensorDepth);
  std::printf("frames %d blocks %d trans_err %.5f raycast_hits %d\n", n, b.lastStats.blocks_total,
              std::sqrt(dt), hits);
  return (std::sqrt(dt) < 0.03 && hits > rows * cols / 10) ? 0 : 1;
}

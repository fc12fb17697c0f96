// Reads a TUM-layout directory through DynaMap::utils::dataSet (the C++
// drop-in) and writes what it decoded, for the tests to compare against
// OpenCV and the Python reader.
//   dataset_example DIR OUTDIR [DEPTH_PREFIX RGB_PREFIX]
//                                per frame: OUTDIR/depth_K.bin (uint16),
//                                OUTDIR/rgb_K.bin (uint8 RGB); stdout one
//                                line "stamp rows cols has_gt p00 .. p33"
//   dataset_example --png FILE OUT   OUT: rows cols channels bits (int32)
//                                    then the unfiltered bytes
//   dataset_example --track DIR LOG rows cols fx fy cx cy scaler
//       the reference driver's loop (src/dynaMap.cpp:218-301): builder over
//       the dataset, first pose from ground truth, each tracked pose
//       appended to LOG by builder::writePoseToTxt (needs a GPU)
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>

#include "builder/builder.h"
#include "utils/dataSet.h"

static int track(char** a) {
  using namespace DynaMap;
  utils::dataSet ds(a[0]);
  rgbdSensor s;
  s.rows = (unsigned)std::atoi(a[2]);
  s.cols = (unsigned)std::atoi(a[3]);
  s.f = {(float)std::atof(a[4]), (float)std::atof(a[5])};
  s.c = {(float)std::atof(a[6]), (float)std::atof(a[7])};
  s.depthScaler = (float)std::atof(a[8]);
  tsdf::tsdfProperties tp;  // the 5 mm volume of the 640x480 sequence preset
  tp.voxelSize = 0.005f;
  tp.numBuckets = 1 << 20;
  tp.numBlocks = 1 << 19;
  tp.truncationDistance = 0.02f;
  tp.maxSensorDepth = 3.0f;
  tp.minSensorDepth = 0.15f;
  solver::Properties op;
  op.lvlIterationNum[0] = 10;
  op.lvlIterationNum[1] = 5;
  op.lvlIterationNum[2] = 4;
  op.colorWeight = 0.1f;
  op.icpMaxDepth = 3.0f;
  gaussianKernal k;
  builder b;
  b.init(tp, op, s, k);
  while (ds.curID < ds.size()) {
    ds.invokeNextFrame();
    if (ds.curID == 1 && !ds.groundTruthLine.empty()) b.setInitialPose(ds.getCurrentPose());
    b.buildModelLS(ds, 1);
    std::vector<double> line = ds.groundTruthLine;
    if (line.empty()) line.push_back(ds.stamp);
    line[0] = ds.stamp;
    builder::writePoseToTxt(a[1], line, b.getCurrentPose(), b.frameNum);
  }
  std::printf("frames %d blocks %d\n", b.frameNum, b.lastStats.blocks_total);
  return 0;
}

static void put(const std::string& path, const void* p, size_t n) {
  std::ofstream f(path, std::ios::binary);
  f.write(static_cast<const char*>(p), (std::streamsize)n);
}

int main(int argc, char** argv) {
  if (argc == 4 && std::strcmp(argv[1], "--png") == 0) {
    const DynaMap::utils::png::Image im = DynaMap::utils::png::read(argv[2]);
    std::ofstream f(argv[3], std::ios::binary);
    const int32_t h[4] = {im.rows, im.cols, im.channels, im.bits};
    f.write(reinterpret_cast<const char*>(h), sizeof h);
    f.write(reinterpret_cast<const char*>(im.data.data()), (std::streamsize)im.data.size());
    return 0;
  }
  if (argc == 11 && std::strcmp(argv[1], "--track") == 0) return track(argv + 2);
  if (argc != 3 && argc != 5) {
    std::fprintf(stderr,
                 "usage: dataset_example DIR OUTDIR [DEPTH_PREFIX RGB_PREFIX] | --png FILE OUT"
                 " | --track ...\n");
    return 2;
  }
  DynaMap::utils::dataSet ds(argv[1]);
  if (argc == 5) {  // another layout: re-list with its prefixes
    ds.depthPrefix = argv[3];
    ds.rgbPrefix = argv[4];
    ds.loadData();
  }
  for (size_t k = 0; ds.curID < ds.size(); ++k) {
    ds.invokeNextFrame();
    const std::string o = std::string(argv[2]) + "/";
    put(o + "depth_" + std::to_string(k) + ".bin", ds.image.depth.data(),
        ds.image.depth.size() * sizeof(uint16_t));
    put(o + "rgb_" + std::to_string(k) + ".bin", ds.image.rgb.data(), ds.image.rgb.size());
    const DynaMap::Matrix4f p = ds.getCurrentPose();
    std::printf("%.6f %d %d %d", ds.stamp, ds.image.rows, ds.image.cols,
                ds.groundTruthLine.empty() ? 0 : 1);
    for (int r = 0; r < 4; ++r)
      for (int c = 0; c < 4; ++c) std::printf(" %.9g", p(r, c));
    std::printf("\n");
  }
  return 0;
}

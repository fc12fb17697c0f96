// The reference's own calls, written as its driver and builder write them
// (src/dynaMap.cpp:180-301, include/builder/builder.cu:70-139): a builder
// over a TUM-layout dataset with the per-frame loop, the target cloud's
// normals read back, a mesh of a box; gnSolver::solve on two rgbdImage
// frames with their point clouds; a tsdfVolume initialised from its
// properties alone, integrating an rgbdImage at a float4x4 pose and
// rendering depth / colour; and the HashTable calls it inherits.  Compiled
// against include/ only (no Eigen, OpenCV or CUDA headers needed).
//   reference_idiom DIR rows cols fx fy cx cy scaler
// Prints one line per part and returns 0 when every check holds.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <iostream>
#include <vector>

#include "builder/builder.h"
#include "utils/dataSet.h"

using namespace DynaMap;

static bool fail(const char* what) {
  std::printf("FAILED: %s\n", what);
  return false;
}

static double trans_err(const Matrix4f& a, const Matrix4f& b) {
  double d = 0;
  for (int r = 0; r < 3; ++r) d += (a(r, 3) - b(r, 3)) * (a(r, 3) - b(r, 3));
  return std::sqrt(d);
}

int main(int argc, char** argv) {
  if (argc != 9) return 2;
  rgbdSensor Xtion;
  Xtion.rows = (unsigned)std::atoi(argv[2]);
  Xtion.cols = (unsigned)std::atoi(argv[3]);
  Xtion.f.x = (float)std::atof(argv[4]);
  Xtion.f.y = (float)std::atof(argv[5]);
  Xtion.c.x = (float)std::atof(argv[6]);
  Xtion.c.y = (float)std::atof(argv[7]);
  Xtion.depthScaler = (float)std::atof(argv[8]);
  bool ok = true;

  // ---- the driver's set-up and loop (dynaMap.cpp:180-301)
  utils::dataSet Dataset(argv[1]);
  gaussianKernal gKernel;
  gKernel.diameter = 8;
  gKernel.sigmaI = 10.0f;
  gKernel.sigmaS = 1.0f;
  solver::Properties OptimizerProp;
  OptimizerProp.lvlIterationNum[0] = 10;
  OptimizerProp.lvlIterationNum[1] = 5;
  OptimizerProp.lvlIterationNum[2] = 4;
  OptimizerProp.lvlScale[0] = 4;
  OptimizerProp.lvlScale[1] = 2;
  OptimizerProp.lvlScale[2] = 1;
  OptimizerProp.maxIteration = 19;
  OptimizerProp.minIncrement = 0.001f;
  OptimizerProp.maxIncrement = 0.3f;
  OptimizerProp.regularization = 0.02f;
  OptimizerProp.icpMaxDepth = 3.0f;
  tsdf::tsdfProperties tsdfProp;
  tsdfProp.voxelSize = 0.005f;
  tsdfProp.numBuckets = 1 << 18;
  tsdfProp.bucketSize = 10;
  tsdfProp.numBlocks = 1 << 16;
  tsdfProp.blockSize = 8;
  tsdfProp.maxSDFWeight = 64;
  tsdfProp.truncationDistance = 0.02f;
  tsdfProp.maxSensorDepth = 3.0f;
  tsdfProp.minSensorDepth = 0.15f;
  builder mapBuilder;
  mapBuilder.init(tsdfProp, OptimizerProp, Xtion, gKernel);
  const int framesToIntegrate = (int)Dataset.rgbFileNames.size();
  for (std::vector<std::string>::iterator it = Dataset.rgbFileNames.begin();
       it != Dataset.rgbFileNames.begin() + framesToIntegrate; ++it) {
    Dataset.invokeNextFrame();
    if (Dataset.curID == 1) mapBuilder.setInitialPose(Dataset.getCurrentPose());
    mapBuilder.buildModelLS(Dataset, 1);
  }
  int normals = 0;
  for (unsigned i = 0; i < Xtion.rows; i++)
    for (unsigned j = 0; j < Xtion.cols; j++) {
      const float3 n = mapBuilder.targetPCL->normals[i * Xtion.cols + j];
      normals += (n.x != 0.0f || n.y != 0.0f || n.z != 0.0f);
    }
  std::cout << mapBuilder.getCurrentPose() << std::endl;
  const double eb = trans_err(mapBuilder.getCurrentPose(), Dataset.getCurrentPose());
  geometry::Mesh mesh = mapBuilder.ExtractMesh(make_float3(-1, -1, 0), make_float3(1, 1, 2));
  std::printf("builder frames %d err %.5f normals %d triangles %u\n", mapBuilder.frameNum, eb,
              normals, mesh.num_triangles_);
  if (mapBuilder.frameNum != framesToIntegrate) ok = fail("builder frames");
  if (!(eb < 0.02)) ok = fail("builder pose");
  if (normals < (int)(Xtion.rows * Xtion.cols / 10)) ok = fail("target normals");

  // ---- two frames as rgbdImage, as builder.cu:105-113 fills them
  utils::dataSet frames(argv[1]);
  rgbdImage targetImage, sourceImage;
  targetImage.init(Xtion);
  sourceImage.init(Xtion);
  Matrix4f pose0, pose1;
  for (rgbdImage* img : {&targetImage, &sourceImage}) {
    frames.invokeNextFrame();
    const std::vector<float> m = frames.image.depthMetres(Xtion.depthScaler);
    for (unsigned i = 0; i < Xtion.rows; i++)
      for (unsigned j = 0; j < Xtion.cols; j++) {
        const size_t k = i * Xtion.cols + j;
        img->depth[k] = m[k];
        img->rgb[k] = make_uchar3(frames.image.rgb[3 * k], frames.image.rgb[3 * k + 1],
                                  frames.image.rgb[3 * k + 2]);
      }
    (img == &targetImage ? pose0 : pose1) = frames.getCurrentPose();
  }

  // gnSolver::solve (gnSolver.h:72-76) from the identity: the source's
  // motion relative to the target
  std::vector<geometry::PointXYZ> tp(targetImage.size()), sp(sourceImage.size());
  std::vector<geometry::NormalXYZ> tn(targetImage.size()), sn(sourceImage.size());
  geometry::PointCloudXYZ targetPCL, sourcePCL;
  targetPCL.points = tp.data();
  targetPCL.normals = tn.data();
  sourcePCL.points = sp.data();
  sourcePCL.normals = sn.data();
  solver::gnSolver GNSolver;
  GNSolver.init(OptimizerProp, Xtion);
  Matrix4f currentPose;
  currentPose.setIdentity();
  Vector6d prev_increment_ = {0, 0, 0, 0, 0, 0};
  GNSolver.solve(currentPose, prev_increment_, targetImage, sourceImage, targetPCL, sourcePCL);
  // the true relative motion pose0^-1 pose1 (rigid inverse)
  double rel[3] = {0, 0, 0};
  for (int r = 0; r < 3; ++r)
    for (int k = 0; k < 3; ++k) rel[r] += pose0(k, r) * (pose1(k, 3) - pose0(k, 3));
  double es = 0, moved = 0;
  for (int r = 0; r < 3; ++r) {
    es += (currentPose(r, 3) - rel[r]) * (currentPose(r, 3) - rel[r]);
    moved += rel[r] * rel[r];
  }
  es = std::sqrt(es);
  moved = std::sqrt(moved);
  int zmatch = 0, valid = 0;
  for (size_t k = 0; k < targetImage.size(); ++k)
    if (targetImage.depth[k] > 0) {
      ++valid;
      zmatch += tp[k].z == targetImage.depth[k];
    }
  std::printf("solver iterations %d err %.5f moved %.5f cloud %d/%d\n", GNSolver.iterationNum,
              es, moved, zmatch, valid);
  if (!(es < 0.5 * moved + 0.002)) ok = fail("solver pose");
  if (valid == 0 || zmatch != valid) ok = fail("solver target cloud");

  // rgbdImage::getPointCloudXYZ / getNormalsfromVertices on their own
  geometry::PointCloudXYZ cloud;
  std::vector<geometry::PointXYZ> cp(sourceImage.size(), make_float3(7, 7, 7));
  std::vector<geometry::NormalXYZ> cn(sourceImage.size());
  cloud.points = cp.data();
  cloud.normals = cn.data();
  sourceImage.getPointCloudXYZ(cloud);
  sourceImage.getNormalsfromVertices(cloud);
  int untouched = 0, unit = 0;
  for (size_t k = 0; k < sourceImage.size(); ++k) {
    if (!(sourceImage.depth[k] > 0)) untouched += cp[k].x == 7.0f;
    const float l = cn[k].x * cn[k].x + cn[k].y * cn[k].y + cn[k].z * cn[k].z;
    unit += std::fabs(l - 1.0f) < 1e-4f;
  }
  const geometry::PointXYZ q = sourceImage.getPointXYZ(Xtion.cols / 2, Xtion.rows / 2);
  const geometry::PointXYZ c = cp[(Xtion.rows / 2) * Xtion.cols + Xtion.cols / 2];
  std::printf("cloud unit-normals %d untouched %d\n", unit, untouched);
  if (unit < (int)(sourceImage.size() / 4)) ok = fail("cloud normals");
  if (q.z > 0 && (q.x != c.x || q.y != c.y || q.z != c.z)) ok = fail("getPointXYZ");

  // ---- tsdfVolume from its properties alone (tsdf.h:45)
  tsdf::tsdfVolume volume;
  volume.init(tsdfProp);
  float4x4 pose_cuda = float4x4(pose0.data()).getTranspose();
  volume.IntegrateScan(targetImage, pose_cuda);
  float* virtual_depth = volume.GenerateDepth(pose_cuda, Xtion);
  uchar3* virtual_rgb = volume.GenerateRgb(pose_cuda, Xtion);
  int hits = 0, coloured = 0;
  for (size_t k = 0; k < targetImage.size(); ++k) {
    hits += virtual_depth[k] < tsdfProp.maxSensorDepth;
    coloured += (virtual_rgb[k].x | virtual_rgb[k].y | virtual_rgb[k].z) != 0;
  }
  // HashTable (hashTable.h:32-142) through the volume
  std::vector<int32_t> coords;
  std::vector<dyn_voxel> voxels;
  volume.DownloadBlocks(coords, voxels);
  const int64_t nb = volume.GetNumAllocatedBlocks();
  const int3 b0 = make_int3(coords[0], coords[1], coords[2]);
  const tsdf::HashEntry e0 = volume.FindHashEntry(b0);
  const bool del = volume.DeleteBlock(b0);
  const tsdf::HashEntry e1 = volume.FindHashEntry(b0);
  const bool del2 = volume.DeleteBlock(b0);
  const int a1 = volume.AllocateBlock(b0), a2 = volume.AllocateBlock(b0);
  const tsdf::HashEntry e2 = volume.FindHashEntry(b0);
  std::printf("volume hits %d coloured %d blocks %lld entries %d hash %d %d %d %d %d %d %d\n",
              hits, coloured, (long long)nb, volume.GetNumEntries(), e0.pointer, (int)del,
              e1.pointer, (int)del2, a1, a2, e2.pointer);
  if (hits < (int)(targetImage.size() / 10) || coloured < hits / 2) ok = fail("volume render");
  if (nb <= 1 || volume.GetNumEntries() != tsdfProp.numBuckets * tsdfProp.bucketSize)
    ok = fail("volume counts");
  if (e0.pointer < 0 || !del || e1.pointer != tsdf::kFreeEntry || del2 || a1 != 1 || a2 != 0 ||
      e2.pointer < 0 || volume.GetNumAllocatedBlocks() != nb)
    ok = fail("hash table calls");
  return ok ? 0 : 1;
}

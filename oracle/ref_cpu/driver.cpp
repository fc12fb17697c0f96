// driver.cpp -- C entry points over the REFERENCE's own classes, compiled
// for the CPU (oracle/_ref/libdynref.so).  Test infrastructure: used to
// generate the golden vectors that pin the oracle (tests/golden/) and, on a
// box without the reference tree, never built.
//
// The reference's sources (tsdf.cu, hashTable.cu, heap.cu, rgbdImage.cu,
// pyramid.cu, conv2D.cu, kernel2D.cu, gnSolver.cu) are compiled unmodified
// apart from the launch syntax (build_ref.sh); this file only drives them:
//   tsdfVolume::init / IntegrateScan / GenerateDepth / GenerateRgb
//   (include/geometry/tsdf/tsdf.cu:18-550), the vertex map and normals of
//   rgbdImage (include/image/sensor/rgbdImage.cu:23-167),
//   pyramid::applyBilateralFilter (include/image/pyramid/pyramid.cu:213-233)
//   the ICP of gnSolver: buildNLSKernel's normal equations and the whole
//   gnSolver::solve (include/solver/gnSolver/gnSolver.cu:26-438, with the
//   Eigen calls answered by shim/eigen_stub.h), and
//   MeshExtractor::ExtractMesh (include/geometry/mesh/meshExtractor/
//   meshExtractor.cu:364-407) with mesh.cu / meshSTD.cu.
#include <cstdint>
#include <cstring>

#include "../../include/dynamap.h"
#include "gnSolver/gnSolver.h"
#include "meshExtractor/meshExtractor.h"
#include "pyramid/pyramid.h"
#include "tsdf/tsdf.h"

using namespace DynaMap;

// defined in gnSolver.cu, not declared in its header
namespace DynaMap {
namespace solver {
void buildNLSKernel(gnSolver& solver, uchar3* target_rgb, float* target_depth, uchar3* source_rgb,
                    float* source_depth, rgbdSensor sensor, float4x4 last_transform,
                    mat6x6* acc_A, mat6x1* acc_b, geometry::PointCloudXYZ& targetCloud,
                    geometry::PointCloudXYZ& sourceCloud, float scale, float huberConstant);
}  // namespace solver
}  // namespace DynaMap

namespace {

struct Peek : tsdf::HashTable {
  static geometry::VoxelBlock* blocks(tsdf::HashTable* h) { return h->*(&Peek::voxel_blocks_); }
  static int hash(tsdf::HashTable* h, int3 p) { return (h->*(&Peek::Hash))(p); }
};

rgbdSensor to_sensor(const dyn_sensor* s) {
  rgbdSensor r;
  r.rows = s->rows;
  r.cols = s->cols;
  r.f = make_float2(s->fx, s->fy);
  r.c = make_float2(s->cx, s->cy);
  r.depthScaler = s->depth_scaler;
  return r;
}

}  // namespace

extern "C" {

void ref_set_threads(int n) { dynref::nthreads() = n < 1 ? 1 : n; }
// buildNLSKernel's photometric weight (the reference's constant 0 at
// gnSolver.cu:180, made settable by build_ref.sh)
void ref_set_color_weight(float w) { dynref::color_weight() = w; }

void* ref_volume_create(const dyn_tsdf_params* p) {
  tsdf::tsdfProperties props;
  std::memset(&props, 0, sizeof(props));
  props.voxelSize = p->voxel_size;
  props.numBuckets = p->num_buckets;
  props.bucketSize = p->bucket_size;
  props.numBlocks = p->num_blocks;
  props.blockSize = p->block_size;
  props.maxSDFWeight = p->max_sdf_weight;
  props.truncationDistance = p->truncation_distance;
  props.maxSensorDepth = p->max_sensor_depth;
  props.minSensorDepth = p->min_sensor_depth;
  tsdf::tsdfVolume* v = new tsdf::tsdfVolume();
  v->init(props);
  return v;
}

void ref_volume_destroy(void* v) { delete (tsdf::tsdfVolume*)v; }

// builder::buildModelGT's integration step (builder.cu:140-156):
// IntegrateScan(image, pose) = AllocateFromDepthKernel + IntegrateScanKernel.
void ref_volume_integrate(void* v, const float* depth, const uint8_t* rgb, const dyn_sensor* s,
                          const float pose[16]) {
  rgbdImage img;
  img.init(to_sensor(s));
  size_t n = (size_t)s->rows * s->cols;
  std::memcpy(img.depth, depth, n * sizeof(float));
  for (size_t i = 0; i < n; ++i)
    img.rgb[i] = rgb ? make_uchar3(rgb[3 * i], rgb[3 * i + 1], rgb[3 * i + 2]) : make_uchar3(0, 0, 0);
  ((tsdf::tsdfVolume*)v)->IntegrateScan(img, float4x4(pose));
}

void ref_volume_generate(void* v, const float pose[16], const dyn_sensor* s, float* depth_out,
                         uint8_t* rgb_out) {
  tsdf::tsdfVolume* vol = (tsdf::tsdfVolume*)v;
  size_t n = (size_t)s->rows * s->cols;
  float* d = vol->GenerateDepth(float4x4(pose), to_sensor(s));
  std::memcpy(depth_out, d, n * sizeof(float));
  cudaFree(d);
  if (rgb_out) {
    uchar3* c = vol->GenerateRgb(float4x4(pose), to_sensor(s));
    for (size_t i = 0; i < n; ++i) {
      rgb_out[3 * i] = c[i].x;
      rgb_out[3 * i + 1] = c[i].y;
      rgb_out[3 * i + 2] = c[i].z;
    }
    cudaFree(c);
  }
}

int32_t ref_hash(void* v, int32_t x, int32_t y, int32_t z) {
  return Peek::hash((tsdf::HashTable*)(tsdf::tsdfVolume*)v, make_int3(x, y, z));
}

// Every non-free entry: coordinates, then its 512 voxels (x-major).
int64_t ref_volume_download(void* v, int32_t* coords, uint8_t* rgbw, float* sdf, int64_t cap) {
  tsdf::tsdfVolume* vol = (tsdf::tsdfVolume*)v;
  geometry::VoxelBlock* blocks = Peek::blocks(vol);
  int64_t k = 0;
  for (int i = 0; i < vol->GetNumEntries(); ++i) {
    tsdf::HashEntry e = vol->GetHashEntry(i);
    if (e.pointer < 0) continue;
    if (k < cap) {
      coords[3 * k] = e.position.x;
      coords[3 * k + 1] = e.position.y;
      coords[3 * k + 2] = e.position.z;
      for (int j = 0; j < 512; ++j) {
        geometry::Voxel& vx = blocks[e.pointer].at(j);
        rgbw[4 * (512 * k + j)] = vx.color.x;
        rgbw[4 * (512 * k + j) + 1] = vx.color.y;
        rgbw[4 * (512 * k + j) + 2] = vx.color.z;
        rgbw[4 * (512 * k + j) + 3] = vx.weight;
        sdf[512 * k + j] = vx.sdf;
      }
    }
    ++k;
  }
  return k;
}

// rgbdImage::getPointCloudXYZ + getNormalsfromVertices (the cloud buffers are
// zeroed first, as builder.cu:75-80 intends).
void ref_normals(const float* depth, const dyn_sensor* s, float* points3, float* normals3) {
  rgbdImage img;
  img.init(to_sensor(s));
  size_t n = (size_t)s->rows * s->cols;
  std::memcpy(img.depth, depth, n * sizeof(float));
  geometry::PointCloudXYZ cloud;
  cudaMallocManaged(&cloud.points, n * sizeof(float3));
  cudaMallocManaged(&cloud.normals, n * sizeof(float3));
  img.getPointCloudXYZ(cloud, 1);
  img.getNormalsfromVertices(cloud);
  std::memcpy(points3, cloud.points, n * sizeof(float3));
  std::memcpy(normals3, cloud.normals, n * sizeof(float3));
  cudaFree(cloud.points);
  cudaFree(cloud.normals);
}

// pyramid::applyBilateralFilter for one pixel (row x, column y); the caller
// keeps the window inside the image (the reference does not bound it).
float ref_bilateral_pixel(const float* src, int rows, int cols, int x, int y, int diameter,
                          float sigma_i, float sigma_s) {
  static pyramid* p = nullptr;
  if (!p) p = new pyramid();
  rgbdSensor s;
  s.rows = rows;
  s.cols = cols;
  s.f = make_float2(1, 1);
  s.c = make_float2(0, 0);
  s.depthScaler = 1;
  float out = 0;
  std::vector<float> dst((size_t)rows * cols, 0.f);
  p->applyBilateralFilter(dst.data(), const_cast<float*>(src), x, y, 2 * diameter, sigma_i,
                          sigma_s, s);
  out = dst[(size_t)x * cols + y];
  return out;
}

// buildNLSKernel at pyramid scale 1 on one host thread, so its float
// atomics sum the pixels' terms in index order: the 6x6 A (all 36 entries)
// and b accumulated as the reference accumulates them (b with its minus
// sign).  Normals are float3 per pixel; T is the row-major source-to-target
// transform; the reference's depth window (0.15, 2.0 m) and colour weight
// (0) are its own constants.  The caller keeps every valid source pixel's
// projection, and its left and upper neighbours, inside the image (the
// reference does not check them).
void ref_icp_normal_equations(const float* src_depth, const float* src_n3, const float* tgt_depth,
                              const float* tgt_n3, const uint8_t* src_rgb, const uint8_t* tgt_rgb,
                              const dyn_sensor* s, const float T[16], float A_out[36],
                              float b_out[6]) {
  static solver::gnSolver* g = nullptr;  // never destroyed: its pyramids own no buffers
  if (!g) g = new solver::gnSolver();
  const size_t n = (size_t)s->rows * s->cols;
  std::vector<float> sd(src_depth, src_depth + n), td(tgt_depth, tgt_depth + n);
  std::vector<float3> sn(n), tn(n);
  std::vector<uchar3> sc(n), tc(n);
  for (size_t i = 0; i < n; ++i) {
    sn[i] = make_float3(src_n3[3 * i], src_n3[3 * i + 1], src_n3[3 * i + 2]);
    tn[i] = make_float3(tgt_n3[3 * i], tgt_n3[3 * i + 1], tgt_n3[3 * i + 2]);
    sc[i] = src_rgb ? make_uchar3(src_rgb[3 * i], src_rgb[3 * i + 1], src_rgb[3 * i + 2])
                    : make_uchar3(0, 0, 0);
    tc[i] = tgt_rgb ? make_uchar3(tgt_rgb[3 * i], tgt_rgb[3 * i + 1], tgt_rgb[3 * i + 2])
                    : make_uchar3(0, 0, 0);
  }
  geometry::PointCloudXYZ src_cloud, tgt_cloud;
  src_cloud.points = nullptr;
  src_cloud.normals = sn.data();
  tgt_cloud.points = nullptr;
  tgt_cloud.normals = tn.data();
  mat6x6 A;
  mat6x1 b;
  A.setZero();
  b.setZero();
  const int saved = dynref::nthreads();
  dynref::nthreads() = 1;
  DYNREF_LAUNCH(solver::buildNLSKernel)(*g, tc.data(), td.data(), sc.data(), sd.data(),
                                        to_sensor(s), float4x4(T), &A, &b, tgt_cloud, src_cloud,
                                        1.0f, 0.0f);
  dynref::nthreads() = saved;
  for (int j = 0; j < 36; ++j) A_out[j] = A(j);
  for (int j = 0; j < 6; ++j) b_out[j] = b(j);
}

// MeshExtractor::Init + ExtractMesh + GetMesh over the box [lo, hi] of a
// volume (one host thread, so triangles come out in grid order): per
// triangle its three vertices' positions and colours, 18 floats, into out
// (at most cap triangles).  Returns the triangle count.
int64_t ref_extract_mesh(void* v, const float lo[3], const float hi[3], float voxel_size,
                         float* out, int64_t cap) {
  tsdf::tsdfVolume* vol = (tsdf::tsdfVolume*)v;
  geometry::MeshExtractor* me = new geometry::MeshExtractor();  // kept: its mesh is read below
  me->Init((unsigned)(cap > 0 ? cap : 1), voxel_size);
  const int saved = dynref::nthreads();
  dynref::nthreads() = 1;
  me->ExtractMesh(vol, make_float3(lo[0], lo[1], lo[2]), make_float3(hi[0], hi[1], hi[2]));
  dynref::nthreads() = saved;
  geometry::Mesh m = me->GetMesh();
  const int64_t n = (int64_t)m.num_triangles_;
  for (int64_t i = 0; i < n && i < cap; ++i) {
    const geometry::Vertex* vs[3] = {&m.triangles_[i].v0, &m.triangles_[i].v1,
                                     &m.triangles_[i].v2};
    for (int k = 0; k < 3; ++k) {
      float* o = out + 18 * i + 6 * k;
      o[0] = vs[k]->position.x;
      o[1] = vs[k]->position.y;
      o[2] = vs[k]->position.z;
      o[3] = vs[k]->color.x;
      o[4] = vs[k]->color.y;
      o[5] = vs[k]->color.z;
    }
  }
  return n;
}

// gnSolver::init + solve (gnSolver.cu:12-21, 317-438) of a source frame
// against a target frame, every pyramid level at scale 1 (the reference's
// pyramid is only defined there), from the identity: the final increment
// xi = [w; t] (prev_increment_ on return) and the composed pose (row-major).
// The caller keeps every valid source pixel's projection inside the image,
// as for ref_icp_normal_equations.
void ref_gn_solve(const float* src_depth, const float* tgt_depth, const uint8_t* src_rgb,
                  const uint8_t* tgt_rgb, const dyn_sensor* s, const int32_t iters[3],
                  float min_increment, float max_increment, float regularization,
                  double inc_out[6], float pose_out[16]) {
  const rgbdSensor sensor = to_sensor(s);
  solver::Properties P;
  for (int l = 0; l < 3; ++l) {
    P.lvlIterationNum[l] = iters[l];
    P.lvlScale[l] = 1;
  }
  P.maxIteration = iters[0] + iters[1] + iters[2];
  P.minIncrement = min_increment;
  P.maxIncrement = max_increment;
  P.regularization = regularization;
  P.huberConstant = 0.0f;
  // never destroyed: the reference's pyramids are not meant to be freed here
  solver::gnSolver* g = new solver::gnSolver();
  g->init(P, sensor);
  rgbdImage* tgt = new rgbdImage();
  rgbdImage* src = new rgbdImage();
  tgt->init(sensor);
  src->init(sensor);
  const size_t n = (size_t)s->rows * s->cols;
  std::memcpy(tgt->depth, tgt_depth, n * sizeof(float));
  std::memcpy(src->depth, src_depth, n * sizeof(float));
  for (size_t i = 0; i < n; ++i) {
    tgt->rgb[i] = tgt_rgb ? make_uchar3(tgt_rgb[3 * i], tgt_rgb[3 * i + 1], tgt_rgb[3 * i + 2])
                          : make_uchar3(0, 0, 0);
    src->rgb[i] = src_rgb ? make_uchar3(src_rgb[3 * i], src_rgb[3 * i + 1], src_rgb[3 * i + 2])
                          : make_uchar3(0, 0, 0);
  }
  geometry::PointCloudXYZ tc, sc;
  for (geometry::PointCloudXYZ* c : {&tc, &sc}) {
    cudaMallocManaged(&c->points, n * sizeof(float3));
    cudaMallocManaged(&c->normals, n * sizeof(float3));
    std::memset(c->points, 0, n * sizeof(float3));
    std::memset(c->normals, 0, n * sizeof(float3));
  }
  Eigen::Matrix4f pose;
  for (int i = 0; i < 16; ++i) pose.v[i] = (i % 5 == 0) ? 1.0f : 0.0f;
  solver::Vector6d prev;
  for (int i = 0; i < 6; ++i) prev(i) = 0.0;
  const int saved = dynref::nthreads();
  dynref::nthreads() = 1;
  g->solve(pose, prev, *tgt, *src, tc, sc);
  dynref::nthreads() = saved;
  for (int i = 0; i < 6; ++i) inc_out[i] = prev(i);
  for (int r = 0; r < 4; ++r)
    for (int c = 0; c < 4; ++c) pose_out[r * 4 + c] = pose(r, c);
}

}  // extern "C"

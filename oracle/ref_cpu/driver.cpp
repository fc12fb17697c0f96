// driver.cpp -- C entry points over the REFERENCE's own classes, compiled
// for the CPU (oracle/_ref/libdynref.so).  Test infrastructure: used to
// generate the golden vectors that pin the oracle (tests/golden/) and, on a
// box without the reference tree, never built.
//
// The reference's sources (tsdf.cu, hashTable.cu, heap.cu, rgbdImage.cu,
// pyramid.cu, conv2D.cu, kernel2D.cu) are compiled unmodified apart from the
// launch syntax (build_ref.sh); this file only drives them:
//   tsdfVolume::init / IntegrateScan / GenerateDepth / GenerateRgb
//   (include/geometry/tsdf/tsdf.cu:18-550), the vertex map and normals of
//   rgbdImage (include/image/sensor/rgbdImage.cu:23-167), and
//   pyramid::applyBilateralFilter (include/image/pyramid/pyramid.cu:213-233).
#include <cstdint>
#include <cstring>

#include "../../include/dynamap.h"
#include "meshExtractor/meshExtractor.h"
#include "pyramid/pyramid.h"
#include "tsdf/tsdf.h"

using namespace DynaMap;

// tsdf.cu's ExtractMesh names the mesh extractor; mesh extraction is not on
// the path, so these definitions only satisfy the linker.
namespace DynaMap {
namespace geometry {
void MeshExtractor::Init(unsigned int, float) {}
void MeshExtractor::ExtractMesh(tsdf::tsdfVolume*, float3, float3) {}
Mesh MeshExtractor::GetMesh() { return Mesh(); }
}  // namespace geometry
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

}  // extern "C"

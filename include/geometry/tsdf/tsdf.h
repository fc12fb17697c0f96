// geometry/tsdf/tsdf.h -- C++ drop-in for DynaMap::tsdf::tsdfVolume and
// tsdfProperties (reference include/geometry/tsdf/tsdf.h:19-81), header-only
// over the C ABI of dynamap.h.
//
// Differences from the reference interface, all forced by the boundary:
//  - init also takes the sensor (the volume owns its image buffers);
//  - IntegrateScan takes the sensor's uint16 depth (and RGB) on the host,
//    the input the reference converts at utils_Dataset.cpp:233-235;
//  - GenerateDepth/GenerateRgb return std::vector instead of leaked managed
//    buffers (tsdf.cu:527-550).
#pragma once

#include <cstdint>
#include <vector>

#include "../../dynamap.h"
#include "../../dynamap/types.h"
#include "../../image/sensor/rgbdImage.h"
#include "../mesh/mesh.h"

namespace DynaMap {
namespace tsdf {

// tsdf.h:19-35 (entriesNum and voxelNumPerAxes are derived, as in the
// reference they are unused on the path)
struct tsdfProperties {
  float voxelSize = 0.01f;
  int numBuckets = 2500;
  int bucketSize = 10;
  int numBlocks = 25000;
  int blockSize = 8;
  int entriesNum = 0;
  int voxelNumPerAxes = 0;
  int maxSDFWeight = 64;
  float truncationDistance = 0.05f;
  float maxSensorDepth = 5.0f;
  float minSensorDepth = 0.3f;

  dyn_tsdf_params to_c() const {
    dyn_tsdf_params p;
    p.voxel_size = voxelSize;
    p.num_buckets = numBuckets;
    p.bucket_size = bucketSize;
    p.num_blocks = numBlocks;
    p.block_size = blockSize;
    p.max_sdf_weight = maxSDFWeight;
    p.truncation_distance = truncationDistance;
    p.max_sensor_depth = maxSensorDepth;
    p.min_sensor_depth = minSensorDepth;
    return p;
  }
};

class tsdfVolume {
 public:
  tsdfProperties Properties;

  tsdfVolume() = default;
  tsdfVolume(const tsdfVolume&) = delete;
  tsdfVolume& operator=(const tsdfVolume&) = delete;
  virtual ~tsdfVolume() { Free(); }

  void init(const tsdfProperties& props, const rgbdSensor& sensor, int device = 0) {
    Free();
    Properties = props;
    sensor_ = sensor;
    dyn_gn_params g;
    dyn_bilateral_params b;
    dyn_default_params(nullptr, &g, &b, nullptr);
    dyn_tsdf_params t = props.to_c();
    dyn_sensor s = sensor.to_c();
    dyn_throw("tsdfVolume::init", dyn_session_create(&t, &g, &b, &s, DYN_PRECISION_FP32, device,
                                                     &session_));
  }
  void Free() {
    if (session_) dyn_session_destroy(session_);
    session_ = nullptr;
  }

  // tsdf.cu:454-469: allocate blocks along the rays, integrate the frame.
  void IntegrateScan(const rgbdImage& image, float4x4 camera_pose) {
    dyn_throw("tsdfVolume::IntegrateScan",
              dyn_integrate_with_pose(session_, image.depth, image.rgb, camera_pose.entries));
  }

  // tsdf.cu:527-538
  std::vector<float> GenerateDepth(float4x4 camera_pose, rgbdSensor sensor) {
    std::vector<float> d((size_t)sensor.rows * sensor.cols);
    dyn_sensor s = sensor.to_c();
    dyn_throw("tsdfVolume::GenerateDepth",
              dyn_raycast(session_, camera_pose.entries, &s, d.data(), nullptr));
    return d;
  }
  // tsdf.cu:539-550 (RGB triplets, row-major)
  std::vector<uint8_t> GenerateRgb(float4x4 camera_pose, rgbdSensor sensor) {
    std::vector<float> d((size_t)sensor.rows * sensor.cols);
    std::vector<uint8_t> c(d.size() * 3);
    dyn_sensor s = sensor.to_c();
    dyn_throw("tsdfVolume::GenerateRgb",
              dyn_raycast(session_, camera_pose.entries, &s, d.data(), c.data()));
    return c;
  }

  // tsdf.cu:551-560: the mesh of the box between the corners
  geometry::Mesh ExtractMesh(const geometry::float3_& lower_corner,
                             const geometry::float3_& upper_corner) {
    const float lo[3] = {lower_corner.x, lower_corner.y, lower_corner.z};
    const float hi[3] = {upper_corner.x, upper_corner.y, upper_corner.z};
    return geometry::ExtractMesh(session_, lo, hi);
  }

  // HashTable::GetNumAllocatedBlocks, hashTable.cu:165
  int64_t GetNumAllocatedBlocks() {
    int64_t n = 0;
    dyn_throw("tsdfVolume::GetNumAllocatedBlocks", dyn_num_blocks(session_, &n));
    return n;
  }
  // every allocated block's coordinate and voxels (x-major per block)
  void DownloadBlocks(std::vector<int32_t>& coords, std::vector<dyn_voxel>& voxels) {
    int64_t n = GetNumAllocatedBlocks(), got = 0;
    coords.resize((size_t)n * 3);
    voxels.resize((size_t)n * 512);
    dyn_throw("tsdfVolume::DownloadBlocks",
              dyn_download_blocks(session_, coords.data(), voxels.data(), n, &got));
  }

  // HashTable::DeleteBlock (hashTable.cu:112-134) for many blocks at once,
  // and its use for a memory budget: the blocks at 'coords' (x, y, z per
  // block), or those the allocation has not touched in the last maxAge + 1
  // frames, are removed; their coordinates and voxels are returned (heap
  // order) for UploadBlocks to bring back.
  int64_t DeleteBlocks(const std::vector<int32_t>& coords, std::vector<int32_t>* removedCoords,
                       std::vector<dyn_voxel>* removedVoxels) {
    return removed("tsdfVolume::DeleteBlocks", removedCoords, removedVoxels,
                   [&](int32_t* c, dyn_voxel* v, int64_t cap, int64_t* n) {
                     return dyn_delete_blocks(session_, coords.data(),
                                              (int64_t)(coords.size() / 3), c, v, cap, n);
                   });
  }
  int64_t EvictBlocks(int maxAge, std::vector<int32_t>* removedCoords,
                      std::vector<dyn_voxel>* removedVoxels) {
    return removed("tsdfVolume::EvictBlocks", removedCoords, removedVoxels,
                   [&](int32_t* c, dyn_voxel* v, int64_t cap, int64_t* n) {
                     return dyn_evict_blocks(session_, maxAge, c, v, cap, n);
                   });
  }
  // blocks placed (keys already present are left as they are)
  int64_t UploadBlocks(const std::vector<int32_t>& coords, const std::vector<dyn_voxel>& voxels) {
    int64_t counts[4] = {0, 0, 0, 0};
    const int64_t n = (int64_t)(coords.size() / 3);
    if ((int64_t)voxels.size() < n * 512) dyn_throw("tsdfVolume::UploadBlocks", DYN_ERR_INVALID_ARG);
    dyn_throw("tsdfVolume::UploadBlocks",
              dyn_upload_blocks(session_, coords.data(), voxels.data(), n, counts));
    return counts[0];
  }

  dyn_session* session() const { return session_; }

 private:
  template <class F>
  int64_t removed(const char* what, std::vector<int32_t>* coords, std::vector<dyn_voxel>* voxels,
                  F call) {
    const int64_t cap = (coords || voxels) ? GetNumAllocatedBlocks() : 0;
    if (coords) coords->resize((size_t)cap * 3);
    if (voxels) voxels->resize((size_t)cap * 512);
    int64_t n = 0;
    dyn_throw(what, call(coords ? coords->data() : nullptr, voxels ? voxels->data() : nullptr,
                         cap, &n));
    const int64_t m = n < cap ? n : cap;
    if (coords) coords->resize((size_t)m * 3);
    if (voxels) voxels->resize((size_t)m * 512);
    return n;
  }

  dyn_session* session_ = nullptr;
  rgbdSensor sensor_;
};

}  // namespace tsdf
}  // namespace DynaMap

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

  dyn_session* session() const { return session_; }

 private:
  dyn_session* session_ = nullptr;
  rgbdSensor sensor_;
};

}  // namespace tsdf
}  // namespace DynaMap

// geometry/tsdf/tsdf.h -- C++ drop-in for DynaMap::tsdf::tsdfVolume,
// tsdfProperties (reference include/geometry/tsdf/tsdf.h:19-81) and the
// HashTable it derives from (include/dataStructure/hashTable/hashTable.h:
// 32-142), header-only over the C ABI of dynamap.h.
//
// The reference's calls are kept: init(const tsdfProperties&),
// IntegrateScan(const rgbdImage&, float4x4), GenerateDepth / GenerateRgb
// returning a float* / uchar3* image, ExtractMesh, and HashTable's
// FindHashEntry, AllocateBlock, DeleteBlock, GetNumAllocatedBlocks,
// GetNumEntries.  Differences, all forced by the boundary:
//  - the volume's device state is created at the first call that brings a
//    sensor (IntegrateScan's image, GenerateDepth's sensor), or by the
//    init overload that takes the sensor: the library sizes its image
//    buffers by the sensor;
//  - GenerateDepth / GenerateRgb return host buffers the volume owns, valid
//    until the next call of the same method (the reference returns a new
//    managed buffer per call and never frees it, tsdf.cu:527-550);
//  - HashTable's calls are host calls on the whole table (its device-side
//    AllocateBlock / DeleteBlock run inside the library's kernels).
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

// hashTable.h:20-25: a block's coordinate and its heap index (kFreeEntry
// when the coordinate has no block)
constexpr int kFreeEntry = -1;
struct HashEntry {
  int3 position;
  int pointer;
};

// HashTable (hashTable.h:32-142) over a session's table.  The session is
// created by the derived volume; every call waits for the session's frames.
class HashTable {
 public:
  HashTable() = default;
  HashTable(const HashTable&) = delete;
  HashTable& operator=(const HashTable&) = delete;
  virtual ~HashTable() = default;

  // hashTable.cu:136-150
  HashEntry FindHashEntry(int3 position) {
    HashEntry e{position, kFreeEntry};
    if (!session_) return e;
    const int32_t c[3] = {position.x, position.y, position.z};
    int32_t p = kFreeEntry;
    dyn_throw("HashTable::FindHashEntry", dyn_find_blocks(session_, c, 1, &p));
    e.pointer = p;
    return e;
  }
  // hashTable.cu:80-110: 1 allocated, 0 already present, -1 bucket full
  // (the block's voxels start unobserved; -2: the heap is exhausted)
  int AllocateBlock(const int3& position) {
    require("HashTable::AllocateBlock");
    const int32_t c[3] = {position.x, position.y, position.z};
    std::vector<dyn_voxel> vox(512, dyn_voxel{0, 0, 0, 0, 0.0f});
    int64_t counts[4] = {0, 0, 0, 0};
    dyn_throw("HashTable::AllocateBlock", dyn_upload_blocks(session_, c, vox.data(), 1, counts));
    return counts[0] ? 1 : counts[1] ? 0 : counts[2] ? -1 : -2;
  }
  // hashTable.cu:112-134: true when a block was there and is now removed
  bool DeleteBlock(const int3& position) {
    require("HashTable::DeleteBlock");
    const int32_t c[3] = {position.x, position.y, position.z};
    int64_t n = 0;
    dyn_throw("HashTable::DeleteBlock",
              dyn_delete_blocks(session_, c, 1, nullptr, nullptr, 0, &n));
    return n > 0;
  }
  // hashTable.cu:165
  int64_t GetNumAllocatedBlocks() {
    if (!session_) return 0;
    int64_t n = 0;
    dyn_throw("HashTable::GetNumAllocatedBlocks", dyn_num_blocks(session_, &n));
    return n;
  }
  // hashTable.cu:167 (numBuckets * bucketSize)
  int GetNumEntries() const { return numEntries_; }

 protected:
  void require(const char* what) const {
    if (!session_) dyn_throw(what, DYN_ERR_INVALID_ARG);
  }
  dyn_session* session_ = nullptr;
  int numEntries_ = 0;
};

class tsdfVolume : public HashTable {
 public:
  tsdfProperties Properties;

  tsdfVolume() = default;
  virtual ~tsdfVolume() { Free(); }

  // tsdf.h:45, tsdf.cu:18: the device state follows at the first call that
  // brings a sensor
  void init(const tsdfProperties& _Properties, int device = 0) {
    Free();
    Properties = _Properties;
    device_ = device;
    numEntries_ = _Properties.numBuckets * _Properties.bucketSize;
  }
  // ... or at once, for a known sensor
  void init(const tsdfProperties& props, const rgbdSensor& sensor, int device = 0) {
    init(props, device);
    create(sensor);
  }
  void Free() {
    if (session_) dyn_session_destroy(session_);
    session_ = nullptr;
  }

  // tsdf.cu:454-469: allocate blocks along the rays, integrate the frame.
  void IntegrateScan(const rgbdImage& image, float4x4 camera_pose) {
    if (!session_) create(image.sensor);
    std::vector<uint16_t> units;
    const uint16_t* d = image.sensorDepth(units);
    dyn_throw("tsdfVolume::IntegrateScan",
              dyn_integrate_with_pose(session_, d, image.rgb ? image.rgbBytes() : nullptr,
                                      camera_pose.entries));
  }

  // tsdf.cu:527-538: the model's depth (metres; maxSensorDepth where no
  // surface is hit) seen from camera_pose by 'sensor'
  float* GenerateDepth(float4x4 camera_pose, rgbdSensor sensor) {
    if (!session_) create(sensor);
    depth_out_.resize((size_t)sensor.rows * sensor.cols);
    dyn_sensor s = sensor.to_c();
    dyn_throw("tsdfVolume::GenerateDepth",
              dyn_raycast(session_, camera_pose.entries, &s, depth_out_.data(), nullptr));
    return depth_out_.data();
  }
  // tsdf.cu:539-550: the model's colour at those hits
  uchar3* GenerateRgb(float4x4 camera_pose, rgbdSensor sensor) {
    if (!session_) create(sensor);
    const size_t n = (size_t)sensor.rows * sensor.cols;
    std::vector<float> d(n);
    rgb_out_.resize(n);
    dyn_sensor s = sensor.to_c();
    dyn_throw("tsdfVolume::GenerateRgb",
              dyn_raycast(session_, camera_pose.entries, &s, d.data(),
                          reinterpret_cast<uint8_t*>(rgb_out_.data())));
    return rgb_out_.data();
  }

  // tsdf.cu:551-560: the mesh of the box between the corners
  geometry::Mesh ExtractMesh(const float3& lower_corner, const float3& upper_corner) {
    require("tsdfVolume::ExtractMesh");
    const float lo[3] = {lower_corner.x, lower_corner.y, lower_corner.z};
    const float hi[3] = {upper_corner.x, upper_corner.y, upper_corner.z};
    return geometry::ExtractMesh(session_, lo, hi);
  }
  // tsdf.h:51 (GetProperties)
  tsdfProperties GetProperties() const { return Properties; }
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
  void create(const rgbdSensor& sensor) {
    sensor_ = sensor;
    dyn_gn_params g;
    dyn_bilateral_params b;
    dyn_default_params(nullptr, &g, &b, nullptr);
    dyn_tsdf_params t = Properties.to_c();
    dyn_sensor s = sensor.to_c();
    dyn_throw("tsdfVolume::init", dyn_session_create(&t, &g, &b, &s, DYN_PRECISION_FP32, device_,
                                                     &session_));
  }

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

  rgbdSensor sensor_;
  int device_ = 0;
  std::vector<float> depth_out_;
  std::vector<uchar3> rgb_out_;
};

}  // namespace tsdf
}  // namespace DynaMap

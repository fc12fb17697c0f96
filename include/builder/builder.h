// builder/builder.h -- C++ drop-in for DynaMap::builder (reference
// include/builder/builder.h:49-117, builder.cu), header-only over the C ABI
// of dynamap.h: one session = one RGB-D stream with its own map.
//
// buildModelLS runs the per-frame path in the intended order (track the
// frame against the previous target, integrate it at the new pose, raycast
// the next target); Mode 0 tracks frame to frame, Mode 1 frame to model.
// Frames are the sensor's uint16 depth + optional RGB, passed directly or
// through utils::dataSet (include/utils/dataSet.h) as the reference does.
#pragma once

#include <cstdint>
#include <fstream>
#include <vector>

#include "../dynamap.h"
#include "../dynamap/pose_io.h"
#include "../dynamap/types.h"
#include "../geometry/tsdf/tsdf.h"
#include "../solver/gnSolver/gnSolver.h"

namespace DynaMap {

class builder {
 public:
  rgbdSensor sensor;
  dyn_frame_stats lastStats{};
  int frameNum = 0;
  // builder.h:98-99: the target's and the source's vertex and normal maps
  // (rows*cols each), refreshed after every frame while keepClouds is set:
  // the target is the model seen from the new pose (the next frame's
  // target), the source the frame just tracked (its filtered depth).  The
  // reference fills them inside gnSolver::solve with the target it tracked
  // against; here they cost a device->host copy per frame, so callers that
  // do not read them clear keepClouds.
  geometry::PointCloudXYZ* targetPCL = &target_pcl_;
  geometry::PointCloudXYZ* sourcePCL = &source_pcl_;
  bool keepClouds = true;

  builder() = default;
  builder(const builder&) = delete;
  builder& operator=(const builder&) = delete;
  virtual ~builder() {
    if (session_) dyn_session_destroy(session_);
  }

  // builder.cu:11-49
  void init(const tsdf::tsdfProperties& tsdfProp, const solver::Properties optimizerProp,
            const rgbdSensor& s, const gaussianKernal& kernel, int device = 0,
            int precision = DYN_PRECISION_FP32) {
    sensor = s;
    tsdf_ = tsdfProp.to_c();
    opt_ = optimizerProp;
    bil_.diameter = kernel.diameter;
    bil_.sigma_i = kernel.sigmaI;
    bil_.sigma_s = kernel.sigmaS;
    bil_.enabled = 1;
    device_ = device;
    precision_ = precision;
  }

  // builder.cu:70-139
  void buildModelLS(const uint16_t* depth, const uint8_t* rgb = nullptr, int Mode = 1) {
    ensure(Mode);
    dyn_throw("builder::buildModelLS", dyn_frame_submit(session_, depth, rgb));
    float pose[16];
    dyn_status r = dyn_frame_result(session_, pose, &lastStats);
    if (r != DYN_ERR_HASH_FULL) dyn_throw("builder::buildModelLS", r);
    currentPose_ = Matrix4f::from_row_major(pose);
    ++frameNum;
    if (keepClouds) refresh_clouds();
  }

  // builder.cu:70 / builder.h:58: the frame dataset.image, read by
  // dataSet::invokeNextFrame (any type with that member and frame layout)
  template <class DataSet>
  auto buildModelLS(DataSet& dataset, int Mode = 0) -> decltype(dataset.image.depth.data(), void()) {
    check_frame(dataset.image, "builder::buildModelLS");
    buildModelLS(dataset.image.depth.data(),
                 dataset.image.rgb.empty() ? nullptr : dataset.image.rgb.data(), Mode);
  }
  // builder.cu:140-160 / builder.h:60: integrate dataset.image at the
  // frame's ground-truth pose
  template <class DataSet>
  auto buildModelGT(DataSet& dataset) -> decltype(dataset.image.depth.data(), void()) {
    check_frame(dataset.image, "builder::buildModelGT");
    if (dataset.groundTruthLine.size() < 8)
      dyn_throw("builder::buildModelGT: the frame has no ground truth", DYN_ERR_INVALID_ARG);
    buildModelGT(dataset.image.depth.data(),
                 dataset.image.rgb.empty() ? nullptr : dataset.image.rgb.data(),
                 v2tRef(dataset.groundTruthLine));
  }

  // builder.cu:140-160: integrate at a known pose (no tracking)
  void buildModelGT(const uint16_t* depth, const uint8_t* rgb, const Matrix4f& pose) {
    ensure(mode_ < 0 ? 1 : mode_);
    float4x4 p = pose.to_row_major();
    dyn_throw("builder::buildModelGT", dyn_integrate_with_pose(session_, depth, rgb, p.entries));
    currentPose_ = pose;
    ++frameNum;
  }

  // builder.cu:263-283
  void setInitialPose(const Matrix4f& pose) {
    ensure(mode_ < 0 ? 1 : mode_);
    float4x4 p = pose.to_row_major();
    dyn_throw("builder::setInitialPose", dyn_session_set_pose(session_, p.entries));
    currentPose_ = pose;
  }
  Matrix4f getCurrentPose() const { return currentPose_; }

  // builder.cu:161-196: render the model at the current pose for a virtual
  // sensor of width x height (intrinsics scaled by width/cols, height/rows).
  // The image is the builder's, valid until the next call of the same
  // method (the reference returns a managed buffer it never frees).
  float* GenerateDepth(int width, int height) {
    depth_out_.resize((size_t)width * height);
    dyn_sensor v = virtual_sensor(width, height);
    float4x4 p = currentPose_.to_row_major();
    dyn_throw("builder::GenerateDepth",
              dyn_raycast(session_, p.entries, &v, depth_out_.data(), nullptr));
    return depth_out_.data();
  }
  uchar3* GenerateRgb(int width, int height) {
    std::vector<float> d((size_t)width * height);
    rgb_out_.resize(d.size());
    dyn_sensor v = virtual_sensor(width, height);
    float4x4 p = currentPose_.to_row_major();
    dyn_throw("builder::GenerateRgb",
              dyn_raycast(session_, p.entries, &v, d.data(),
                          reinterpret_cast<uint8_t*>(rgb_out_.data())));
    return rgb_out_.data();
  }

  // builder.cu:66-69: the mesh of the box between the corners
  geometry::Mesh ExtractMesh(const float3& lower_corner, const float3& upper_corner) {
    const float lo[3] = {lower_corner.x, lower_corner.y, lower_corner.z};
    const float hi[3] = {upper_corner.x, upper_corner.y, upper_corner.z};
    return geometry::ExtractMesh(session_, lo, hi);
  }


  dyn_session* session() const { return session_; }

  // builder.cu:222-241: a TUM ground-truth line {stamp, tx, ty, tz, qx, qy,
  // qz, qw} as a pose (quaternion normalised, rotation rounded to float)
  static Matrix4f v2tRef(std::vector<double>& vec) {
    if (vec.size() < 8) dyn_throw("builder::v2tRef", DYN_ERR_INVALID_ARG);
    float p[16];
    pose_io::pose_from_tum(vec.data(), p);
    return Matrix4f::from_row_major(p);
  }

  // builder.cu:243-257: append "stamp tx ty tz qx qy qz qw" (fixed, four
  // decimals; vec[0] is the stamp) for Pose to fileName.  'count' is unused,
  // as in the reference.
  static void writePoseToTxt(const char* fileName, std::vector<double>& vec, const Matrix4f& Pose,
                             int count) {
    (void)count;
    if (vec.empty()) dyn_throw("builder::writePoseToTxt", DYN_ERR_INVALID_ARG);
    std::ofstream file(fileName, std::ios::ate | std::ios::app);
    if (file.is_open()) file << pose_io::tum_line(vec[0], Pose.to_row_major().entries) << "\n";
  }

 private:
  template <class Frame>
  void check_frame(const Frame& f, const char* what) const {
    const size_t n = (size_t)sensor.rows * sensor.cols;
    if ((size_t)f.rows != (size_t)sensor.rows || (size_t)f.cols != (size_t)sensor.cols ||
        f.depth.size() != n || (!f.rgb.empty() && f.rgb.size() != 3 * n))
      dyn_throw(what, DYN_ERR_INVALID_ARG);
  }
  void ensure(int mode) {
    if (session_) {
      if (mode != mode_) dyn_throw("builder: Mode changed after the first frame", DYN_ERR_INVALID_ARG);
      return;
    }
    mode_ = mode;
    dyn_gn_params g = opt_.to_c(mode);
    dyn_sensor s = sensor.to_c();
    dyn_throw("builder::init", dyn_session_create(&tsdf_, &g, &bil_, &s, precision_, device_,
                                                  &session_));
  }
  dyn_sensor virtual_sensor(int width, int height) const {
    dyn_sensor v = sensor.to_c();
    float fx = (float)width / (float)sensor.cols, fy = (float)height / (float)sensor.rows;
    v.rows = (uint32_t)height;
    v.cols = (uint32_t)width;
    v.fx = fx * sensor.f.x;
    v.fy = fy * sensor.f.y;
    v.cx = fx * sensor.c.x;
    v.cy = fy * sensor.c.y;
    return v;
  }

  // the session's level-0 target (which 5) or source (which 2) depth and
  // its vertex and normal maps into the clouds
  void refresh_clouds() {
    const size_t n = (size_t)sensor.rows * sensor.cols;
    std::vector<float> d(n), v(4 * n), nm(4 * n);
    cloud_points_[0].resize(n);
    cloud_normals_[0].resize(n);
    cloud_points_[1].resize(n);
    cloud_normals_[1].resize(n);
    const dyn_sensor s = sensor.to_c();
    for (int k = 0; k < 2; ++k) {
      dyn_throw("builder: clouds", dyn_debug_image(session_, k == 0 ? 5 : 2, 0, d.data(),
                                                   (int64_t)(n * sizeof(float))));
      for (float& z : d)
        if (!(z > 0.0f && z < tsdf_.max_sensor_depth)) z = 0.0f;  // no surface
      dyn_throw("builder: clouds", dyn_depth_to_maps_host(d.data(), &s, v.data(), nm.data()));
      for (size_t i = 0; i < n; ++i) {
        cloud_points_[k][i] = make_float3(v[4 * i], v[4 * i + 1], v[4 * i + 2]);
        cloud_normals_[k][i] = make_float3(nm[4 * i], nm[4 * i + 1], nm[4 * i + 2]);
      }
    }
    target_pcl_.points = cloud_points_[0].data();
    target_pcl_.normals = cloud_normals_[0].data();
    source_pcl_.points = cloud_points_[1].data();
    source_pcl_.normals = cloud_normals_[1].data();
  }

  geometry::PointCloudXYZ target_pcl_, source_pcl_;
  std::vector<float3> cloud_points_[2], cloud_normals_[2];
  std::vector<float> depth_out_;
  std::vector<uchar3> rgb_out_;
  dyn_session* session_ = nullptr;
  dyn_tsdf_params tsdf_{};
  solver::Properties opt_;
  dyn_bilateral_params bil_{};
  int device_ = 0;
  int precision_ = DYN_PRECISION_FP32;
  int mode_ = -1;
  Matrix4f currentPose_;
};

}  // namespace DynaMap

// solver/gnSolver/gnSolver.h -- C++ drop-in for DynaMap::solver::gnSolver and
// solver::Properties (reference include/solver/gnSolver/gnSolver.h:45-100),
// header-only over the C ABI of dynamap.h.
//
// solve() keeps the reference's contract (gnSolver.cu:317-438): coarse-to-
// fine point-to-plane (+photometric) Gauss-Newton of the source frame
// against the target frame, then pose <- exp(xi) pose (or pose exp(xi)).
// The images are float depth in metres (what the reference's rgbdImage
// holds) on the host; the normal equations, the 6x6 solve and the SE(3)
// exponential run on the device.  Eigen::Matrix4f / Vector6d become the
// column-major Matrix4f and double[6] of dynamap/types.h.
#pragma once

#include <cstdint>
#include <utility>
#include <vector>

#include "../../dynamap.h"
#include "../../dynamap/types.h"
#include "../../geometry/geom_Types.h"
#include "../../image/sensor/rgbdImage.h"

namespace DynaMap {
namespace solver {

// gnSolver.h:47-55 plus the values the reference hard-codes
struct Properties {
  int lvlIterationNum[3] = {0, 0, 20};
  int lvlScale[3] = {4, 2, 1};
  int maxIteration = 20;
  float minIncrement = 0.001f;
  float maxIncrement = 0.3f;
  float regularization = 0.02f;
  float huberConstant = 0.3f;
  // additive (gnSolver.cu:108,180; pyramid.h:15-16)
  float colorWeight = 0.0f;
  float icpMinDepth = 0.15f;
  float icpMaxDepth = 2.0f;
  float normalCosThresh = 0.95105651629515357f;
  // 1: pose <- exp(xi) * pose as gnSolver.cu:429 writes it; 0 (default):
  // pose <- pose * exp(xi), the composition that matches xi's frame
  int composeLeft = 0;

  dyn_gn_params to_c(int mode) const {
    dyn_gn_params g;
    for (int i = 0; i < 3; ++i) {
      g.lvl_iteration_num[i] = lvlIterationNum[i];
      g.lvl_scale[i] = lvlScale[i];
    }
    g.max_iteration = maxIteration;
    g.min_increment = minIncrement;
    g.max_increment = maxIncrement;
    g.regularization = regularization;
    g.huber_constant = huberConstant;
    g.color_weight = colorWeight;
    g.icp_min_depth = icpMinDepth;
    g.icp_max_depth = icpMaxDepth;
    g.normal_cos_thresh = normalCosThresh;
    g.mode = mode;
    g.compose_left = composeLeft;
    return g;
  }
};

class gnSolver {
 public:
  Properties OptProp;
  int iterationNum = 1;
  dyn_frame_stats lastStats{};

  gnSolver() = default;
  gnSolver(const gnSolver&) = delete;
  gnSolver& operator=(const gnSolver&) = delete;
  ~gnSolver() { Free(); }

  // gnSolver.cu:12-21
  void init(Properties props, const rgbdSensor& sensor, int device = 0) {
    Free();
    OptProp = props;
    sensor_ = sensor;
    dyn_tsdf_params t;
    dyn_bilateral_params b;
    dyn_default_params(&t, nullptr, &b, nullptr);
    t.num_buckets = 1;  // the solver uses no map
    t.num_blocks = 1;
    b.enabled = 0;
    dyn_gn_params g = props.to_c(0);
    dyn_sensor s = sensor.to_c();
    dyn_throw("gnSolver::init",
              dyn_session_create(&t, &g, &b, &s, DYN_PRECISION_FP32, device, &session_));
  }
  void Free() {
    if (session_) dyn_session_destroy(session_);
    session_ = nullptr;
  }

  // gnSolver.cu:317-438
  void solve(Matrix4f& pose, Vector6d& prev_increment, const std::vector<float>& target_depth,
             const std::vector<float>& source_depth, const uint8_t* target_rgb = nullptr,
             const uint8_t* source_rgb = nullptr) {
    size_t n = (size_t)sensor_.rows * sensor_.cols;
    if (target_depth.size() != n || source_depth.size() != n)
      dyn_throw("gnSolver::solve", DYN_ERR_INVALID_ARG);
    float4x4 p = pose.to_row_major();
    dyn_throw("gnSolver::solve",
              dyn_solver_solve(session_, target_depth.data(), target_rgb, source_depth.data(),
                               source_rgb, p.entries, prev_increment, &lastStats));
    pose = Matrix4f::from_row_major(p.entries);
    iterationNum = lastStats.icp_iterations[2];
  }

  // gnSolver.h:72-76, the reference's own signature: the images' depth
  // (metres) and colour; the clouds, where their arrays are given, receive
  // the full-resolution vertex and normal maps of the two images, as the
  // reference's solve leaves them (the solver itself derives the pyramid's
  // maps from the depths on the device).
  void solve(Matrix4f& pose, Vector6d& prev_increment, rgbdImage& targetImage,
             rgbdImage& sourceImage, geometry::PointCloudXYZ& targetCloud,
             geometry::PointCloudXYZ& sourceCloud) {
    const size_t n = (size_t)sensor_.rows * sensor_.cols;
    if (!targetImage.depth || !sourceImage.depth || targetImage.size() != n ||
        sourceImage.size() != n)
      dyn_throw("gnSolver::solve", DYN_ERR_INVALID_ARG);
    float4x4 p = pose.to_row_major();
    const bool col = OptProp.colorWeight != 0.0f && targetImage.rgb && sourceImage.rgb;
    dyn_throw("gnSolver::solve",
              dyn_solver_solve(session_, targetImage.depth, col ? targetImage.rgbBytes() : nullptr,
                               sourceImage.depth, col ? sourceImage.rgbBytes() : nullptr,
                               p.entries, prev_increment, &lastStats));
    pose = Matrix4f::from_row_major(p.entries);
    iterationNum = lastStats.icp_iterations[2];
    for (auto c : {std::make_pair(&targetImage, &targetCloud),
                    std::make_pair(&sourceImage, &sourceCloud)}) {
      if (c.second->points) c.first->getPointCloudXYZ(*c.second);
      if (c.second->normals) c.first->getNormalsfromVertices(*c.second);
    }
  }

 private:
  dyn_session* session_ = nullptr;
  rgbdSensor sensor_;
};

}  // namespace solver
}  // namespace DynaMap

// config.cpp -- defaults and the reference's flat YAML parameter files.
//
// The reference loads config/*.yaml only through ROS rosparam
// (launch/dynamap_node.launch:12-15) and hard-codes the same values in its
// standalone driver (src/dynaMap.cpp:124-208).  The files are lists of
// "- key: value" lines under one top-level name; this parser reads exactly
// that shape with no external library.  Keys are the reference's own
// (tsdfParams.yaml, gnOptimParams.yaml, bilateralFParams.yaml,
// cameraParams.yaml) plus additive keys for values the reference hard-codes.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>

#include "../../include/dynamap.h"

namespace {

std::string trim(const std::string& s) {
  size_t a = s.find_first_not_of(" \t\r\n");
  if (a == std::string::npos) return "";
  size_t b = s.find_last_not_of(" \t\r\n");
  return s.substr(a, b - a + 1);
}

bool parse_num(const std::string& v, double* out) {
  std::string t = trim(v);
  if (t.empty()) return false;
  if (t == "True" || t == "true") {
    *out = 1;
    return true;
  }
  if (t == "False" || t == "false") {
    *out = 0;
    return true;
  }
  char* end = nullptr;
  double d = std::strtod(t.c_str(), &end);
  if (end == t.c_str()) return false;
  *out = d;
  return true;
}

}  // namespace

extern "C" {

dyn_status dyn_default_params(dyn_tsdf_params* tsdf, dyn_gn_params* gn, dyn_bilateral_params* bil,
                              dyn_sensor* sensor) {
  if (tsdf) {  // config/tsdfParams.yaml:1-10
    tsdf->voxel_size = 0.01f;
    tsdf->num_buckets = 2500;
    tsdf->bucket_size = 10;
    tsdf->num_blocks = 25000;
    tsdf->block_size = 8;
    tsdf->max_sdf_weight = 64;
    tsdf->truncation_distance = 0.05f;
    tsdf->max_sensor_depth = 5.0f;
    tsdf->min_sensor_depth = 0.3f;
  }
  if (gn) {  // config/gnOptimParams.yaml:1-11
    gn->lvl_iteration_num[0] = 0;
    gn->lvl_iteration_num[1] = 0;
    gn->lvl_iteration_num[2] = 20;
    gn->lvl_scale[0] = 4;
    gn->lvl_scale[1] = 2;
    gn->lvl_scale[2] = 1;
    gn->max_iteration = 20;
    gn->min_increment = 0.001f;
    gn->max_increment = 0.3f;
    gn->regularization = 0.02f;
    gn->huber_constant = 0.3f;
    gn->color_weight = 0.0f;             // gnSolver.cu:180
    gn->icp_min_depth = 0.15f;           // pyramid.h:16 DEPTH_MIN
    gn->icp_max_depth = 2.0f;            // pyramid.h:15 DEPTH_MAX
    gn->normal_cos_thresh = (float)std::cos(3.14159265358979323846 / 10);  // gnSolver.cu:108
    gn->mode = 1;                        // frame-to-model (builder Mode 1)
    gn->compose_left = 0;
  }
  if (bil) {  // config/bilateralFParams.yaml:1-4
    bil->diameter = 8;
    bil->sigma_i = 10.0f;
    bil->sigma_s = 1.0f;
    bil->enabled = 1;
  }
  if (sensor) {  // config/cameraParams.yaml:1-10 (TUM)
    sensor->fx = 525.0f;
    sensor->fy = 525.0f;
    sensor->cx = 319.5f;
    sensor->cy = 239.5f;
    sensor->depth_scaler = 5000.0f;
    sensor->rows = 480;
    sensor->cols = 640;
  }
  return DYN_OK;
}

dyn_status dyn_load_yaml(const char* path, dyn_tsdf_params* tsdf, dyn_gn_params* gn,
                         dyn_bilateral_params* bil, dyn_sensor* sensor) {
  if (!path) return DYN_ERR_INVALID_ARG;
  FILE* f = std::fopen(path, "r");
  if (!f) return DYN_ERR_INVALID_ARG;
  char buf[1024];
  while (std::fgets(buf, sizeof(buf), f)) {
    std::string line(buf);
    size_t hash = line.find('#');
    if (hash != std::string::npos) line = line.substr(0, hash);
    line = trim(line);
    if (line.empty()) continue;
    if (line[0] == '-') line = trim(line.substr(1));
    size_t colon = line.find(':');
    if (colon == std::string::npos) continue;
    std::string key = trim(line.substr(0, colon));
    double v = 0;
    if (!parse_num(line.substr(colon + 1), &v)) continue;  // section headers
    if (tsdf) {
      if (key == "voxelSize") tsdf->voxel_size = (float)v;
      else if (key == "numBuckets") tsdf->num_buckets = (int)v;
      else if (key == "bucketSize") tsdf->bucket_size = (int)v;
      else if (key == "numBlocks") tsdf->num_blocks = (int)v;
      else if (key == "blockSize") tsdf->block_size = (int)v;
      else if (key == "maxSDFWeight") tsdf->max_sdf_weight = (int)v;
      else if (key == "truncationDistance") tsdf->truncation_distance = (float)v;
      else if (key == "maxSensorDepth") tsdf->max_sensor_depth = (float)v;
      else if (key == "minSensorDepth") tsdf->min_sensor_depth = (float)v;
    }
    if (gn) {
      if (key.rfind("lvlIterationNum[", 0) == 0 || key.rfind("lvlScale[", 0) == 0) {
        size_t lb = key.find('['), rb = key.find(']');
        if (rb != std::string::npos && rb > lb + 1) {
          int i = std::atoi(key.substr(lb + 1, rb - lb - 1).c_str());
          if (i >= 0 && i < 3) {
            if (key[3] == 'I') gn->lvl_iteration_num[i] = (int)v;
            else gn->lvl_scale[i] = (int)v;
          }
        }
      } else if (key == "maxIteration") gn->max_iteration = (int)v;
      else if (key == "minIncrement") gn->min_increment = (float)v;
      else if (key == "maxIncrement") gn->max_increment = (float)v;
      else if (key == "regularization") gn->regularization = (float)v;
      else if (key == "huberConstant") gn->huber_constant = (float)v;
      else if (key == "colorWeight") gn->color_weight = (float)v;
      else if (key == "icpMinDepth") gn->icp_min_depth = (float)v;
      else if (key == "icpMaxDepth") gn->icp_max_depth = (float)v;
      else if (key == "normalCosThresh") gn->normal_cos_thresh = (float)v;
      else if (key == "mode") gn->mode = (int)v;
      else if (key == "composeLeft") gn->compose_left = (int)v;
    }
    if (bil) {
      if (key == "diameter") bil->diameter = (int)v;
      else if (key == "sigmaI") bil->sigma_i = (float)v;
      else if (key == "sigmaS") bil->sigma_s = (float)v;
      else if (key == "bilateralEnabled") bil->enabled = (int)v;
    }
    if (sensor) {
      if (key == "f.x") sensor->fx = (float)v;
      else if (key == "f.y") sensor->fy = (float)v;
      else if (key == "c.x") sensor->cx = (float)v;
      else if (key == "c.y") sensor->cy = (float)v;
      else if (key == "depthScale") sensor->depth_scaler = (float)v;
      else if (key == "height") sensor->rows = (uint32_t)v;
      else if (key == "width") sensor->cols = (uint32_t)v;
    }
  }
  std::fclose(f);
  return DYN_OK;
}

}  // extern "C"

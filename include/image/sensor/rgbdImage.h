// image/sensor/rgbdImage.h -- C++ drop-in for DynaMap::rgbdImage (reference
// include/image/sensor/rgbdImage.h:37-66, rgbdImage.cu), header-only over
// the C ABI of dynamap.h.
//
// The same members as the reference: depth in metres (float, rows*cols),
// rgb as uchar3 (R, G, B), the sensor; init allocates both, zeroed.  The
// reference's buffers are managed memory the host writes directly; these
// are host memory owned by the image (copies are deep: the reference's
// `targetImage = sourceImage` clones the frame).  getPointCloudXYZ and
// getNormalsfromVertices run on the GPU through dyn_depth_to_maps_host.
//
// One addition: rawDepth, the sensor's uint16 frame (metres * depthScaler).
// When it is set the library reads it as-is; otherwise depth is turned back
// into sensor units by rounding depth * depthScaler, which gives the
// original values exactly for depths that came from the sensor's units
// (the reference's loader divides them by depthScaler, utils_Dataset.cpp:
// 233-235).
#pragma once

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "../../dynamap.h"
#include "../../dynamap/types.h"
#include "../../geometry/geom_Types.h"

namespace DynaMap {

static_assert(sizeof(uchar3) == 3, "uchar3 is three bytes: RGB triplets");

class rgbdImage {
 public:
  rgbdImage() = default;
  rgbdImage(const rgbdImage& o) { *this = o; }
  rgbdImage& operator=(const rgbdImage& o) {
    if (this == &o) return *this;
    sensor = o.sensor;
    rawDepth = o.rawDepth;
    if (o.depth || o.rgb) {
      init(o.sensor);
      const size_t n = size();
      if (o.depth) std::memcpy(depth, o.depth, n * sizeof(float));
      if (o.rgb) std::memcpy(rgb, o.rgb, n * sizeof(uchar3));
    } else {
      release();
    }
    return *this;
  }
  ~rgbdImage() { release(); }

  // rgbdImage.cu:16-21
  void init(const rgbdSensor& _sensor) {
    release();
    sensor = _sensor;
    depth_buf_.assign(size(), 0.0f);
    rgb_buf_.assign(size(), make_uchar3(0, 0, 0));
    depth = depth_buf_.data();
    rgb = rgb_buf_.data();
  }

  // the pixel's point (getPoint3d, utils.h:104-112) and colour
  geometry::PointXYZ getPointXYZ(int u, int v) const {
    const float z = depth[(size_t)v * sensor.cols + u];
    return make_float3(((float)u - sensor.c.x) * z / sensor.f.x,
                       ((float)v - sensor.c.y) * z / sensor.f.y, z);
  }
  geometry::PointXYZRGB getPointXYZRGB(int u, int v) const {
    geometry::PointXYZRGB p;
    p.point = getPointXYZ(u, v);
    p.rgb = rgb[(size_t)v * sensor.cols + u];
    return p;
  }

  // rgbdImage.cu:22-49: cloud.points[i] = getPoint3d(i, depth[i], sensor,
  // scale) where depth[i] > 0 (other points are left as they are).
  void getPointCloudXYZ(geometry::PointCloudXYZ& cloud, int scale = 1) {
    if (!cloud.points) dyn_throw("rgbdImage::getPointCloudXYZ", DYN_ERR_INVALID_ARG);
    dyn_sensor s = sensor.to_c();
    s.fx = sensor.f.x / (float)scale;
    s.fy = sensor.f.y / (float)scale;
    std::vector<float> v(size() * 4), nrm(size() * 4);
    dyn_throw("rgbdImage::getPointCloudXYZ",
              dyn_depth_to_maps_host(depth, &s, v.data(), nrm.data()));
    for (size_t i = 0; i < size(); ++i)
      if (depth[i] > 0.0f) cloud.points[i] = make_float3(v[4 * i], v[4 * i + 1], v[4 * i + 2]);
  }

  // rgbdImage.cu:126-167: the normal of every pixel from the vertices two
  // columns and one row either side, normalised cross product.  The
  // vertices are this image's (what getPointCloudXYZ gives at scale 1),
  // recomputed from its depth; a normal is 0 where its pixel or one of
  // those neighbours has no depth or lies outside the image (the reference
  // reads across row ends and past invalid pixels).
  void getNormalsfromVertices(geometry::PointCloudXYZ& cloud) {
    if (!cloud.normals) dyn_throw("rgbdImage::getNormalsfromVertices", DYN_ERR_INVALID_ARG);
    dyn_sensor s = sensor.to_c();
    std::vector<float> nrm(size() * 4);
    dyn_throw("rgbdImage::getNormalsfromVertices",
              dyn_depth_to_maps_host(depth, &s, nullptr, nrm.data()));
    for (size_t i = 0; i < size(); ++i)
      cloud.normals[i] = make_float3(nrm[4 * i], nrm[4 * i + 1], nrm[4 * i + 2]);
  }

  // The frame in sensor units for the library: rawDepth when set, else
  // depth * depthScaler rounded (0 where depth is not a positive finite
  // value; clamped to 65535).
  const uint16_t* sensorDepth(std::vector<uint16_t>& scratch) const {
    if (rawDepth) return rawDepth;
    if (!depth) dyn_throw("rgbdImage: no depth", DYN_ERR_INVALID_ARG);
    scratch.resize(size());
    for (size_t i = 0; i < size(); ++i) {
      const float d = depth[i];
      const float u = d * sensor.depthScaler;
      scratch[i] = (d > 0.0f && std::isfinite(u))
                       ? (uint16_t)std::min(65535.0f, std::nearbyint(u)) : (uint16_t)0;
    }
    return scratch.data();
  }
  const uint8_t* rgbBytes() const { return reinterpret_cast<const uint8_t*>(rgb); }
  size_t size() const { return (size_t)sensor.rows * sensor.cols; }

  float* depth = nullptr;
  uchar3* rgb = nullptr;
  rgbdSensor sensor;
  const uint16_t* rawDepth = nullptr;  // addition (see above); not owned

 private:
  void release() {
    depth_buf_.clear();
    depth_buf_.shrink_to_fit();
    rgb_buf_.clear();
    rgb_buf_.shrink_to_fit();
    depth = nullptr;
    rgb = nullptr;
  }
  std::vector<float> depth_buf_;
  std::vector<uchar3> rgb_buf_;
};

}  // namespace DynaMap

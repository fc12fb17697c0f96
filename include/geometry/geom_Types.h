// geometry/geom_Types.h -- the point types of the reference's
// include/geometry/geom_Types.h:26-35 that its rgbdImage and gnSolver
// interfaces take: points and normals are float3, a cloud is two arrays of
// rows*cols of them (owned by the caller, as in the reference).
#pragma once

#include "../dynamap/types.h"

namespace DynaMap {
namespace geometry {

typedef float3 PointXYZ;
typedef float3 NormalXYZ;

struct PointXYZRGB {
  PointXYZ point;
  uchar3 rgb;
};

struct PointCloudXYZ {
  PointXYZ* points = nullptr;
  NormalXYZ* normals = nullptr;
};

struct PointCloudXYZRGB {
  PointXYZ* points = nullptr;
  NormalXYZ* normals = nullptr;
  uchar3* colors = nullptr;
};

}  // namespace geometry
}  // namespace DynaMap

// geometry/mesh/mesh.h -- C++ drop-in for DynaMap::geometry::Mesh (reference
// include/geometry/mesh/mesh.h:25-70, mesh.cu) and its Vertex / Triangle
// (include/geometry/geom_Types.h:40-60): the triangle soup that
// tsdfVolume::ExtractMesh returns, held in host memory.
//
// ExtractMesh (dynamap.h: dyn_extract_mesh) fills it in one call; the
// reference's device-side AppendTriangle and its managed buffer are not
// needed, and there is no triangle limit to reach.  Vertex normals are zero,
// as the reference leaves them unset.
#pragma once

#include <cstdint>
#include <fstream>
#include <string>
#include <vector>

#include "../../dynamap.h"
#include "../../dynamap/types.h"

namespace DynaMap {
namespace geometry {

// the reference's float3 (CUDA's, or the host stand-in of dynamap/types.h)
typedef float3 float3_;

struct Vertex {
  float3_ position{0.0f, 0.0f, 0.0f};
  float3_ normal{0.0f, 0.0f, 0.0f};
  float3_ color{0.0f, 0.0f, 0.0f};  // 0..1
};

struct Triangle {
  Vertex v0, v1, v2;
};

class Mesh {
 public:
  std::vector<Triangle> triangles_;
  unsigned int num_triangles_ = 0;

  // mesh.cu:7-12 (the capacity is the vector's)
  void Init(unsigned int max_triangles) {
    triangles_.clear();
    triangles_.reserve(max_triangles);
    num_triangles_ = 0;
  }
  void Free() {
    triangles_.clear();
    triangles_.shrink_to_fit();
    num_triangles_ = 0;
  }

  // The triangles of dyn_extract_mesh's output: 18 floats each, three
  // vertices of {x, y, z, r, g, b}.
  void Assign(const float* tri, size_t n) {
    triangles_.resize(n);
    for (size_t i = 0; i < n; ++i) {
      Vertex* v[3] = {&triangles_[i].v0, &triangles_[i].v1, &triangles_[i].v2};
      for (int k = 0; k < 3; ++k) {
        const float* p = tri + 18 * i + 6 * k;
        v[k]->position = {p[0], p[1], p[2]};
        v[k]->normal = {};
        v[k]->color = {p[3], p[4], p[5]};
      }
    }
    num_triangles_ = (unsigned int)n;
  }

  // mesh.cu:39-64: "v x y z r g b" per vertex, then "f i i+1 i+2" per
  // triangle (1-based); returns the triangle count.
  int SaveToFile(const std::string& filename) const {
    std::ofstream fout(filename.c_str(), std::ofstream::out);
    for (const Triangle& t : triangles_)
      for (const Vertex* v : {&t.v0, &t.v1, &t.v2})
        fout << "v " << v->position.x << " " << v->position.y << " " << v->position.z << " "
             << v->color.x << " " << v->color.y << " " << v->color.z << "\n";
    for (size_t i = 1; i <= triangles_.size() * 3; i += 3)
      fout << "f " << i << " " << i + 1 << " " << i + 2 << "\n";
    return (int)num_triangles_;
  }
};

// tsdfVolume::ExtractMesh (tsdf.cu:551-560) on a session's volume.
inline Mesh ExtractMesh(dyn_session* s, const float lower[3], const float upper[3]) {
  int64_t n = 0;
  dyn_throw("ExtractMesh", dyn_extract_mesh(s, lower, upper, nullptr, 0, &n));
  std::vector<float> tri((size_t)n * 18);
  int64_t got = 0;
  dyn_throw("ExtractMesh", dyn_extract_mesh(s, lower, upper, tri.data(), n, &got));
  Mesh m;
  m.Assign(tri.data(), (size_t)(got < n ? got : n));
  return m;
}

}  // namespace geometry
}  // namespace DynaMap

// geometry::Mesh on the host (no GPU): triangles from dyn_extract_mesh's
// layout written by SaveToFile; and, compiled only, the volume's mesh and
// eviction calls with the types callers pass.
//   mesh_io_example OBJ   reads 18*n floats (text) from stdin
#include <cstdio>
#include <iostream>
#include <vector>

#include "builder/builder.h"
#include "geometry/mesh/mesh.h"
#include "geometry/tsdf/tsdf.h"

using namespace DynaMap;

// Never called: instantiates the templates behind the calls.
void uses(tsdf::tsdfVolume& v, builder& b) {
  std::vector<int32_t> coords, outc;
  std::vector<dyn_voxel> outv;
  v.DeleteBlocks(coords, &outc, &outv);
  v.DeleteBlocks(coords, nullptr, nullptr);
  v.EvictBlocks(30, &outc, &outv);
  v.UploadBlocks(outc, outv);
  geometry::Mesh m1 = v.ExtractMesh({-1, -1, 0}, {1, 1, 2});
  geometry::Mesh m2 = b.ExtractMesh({-3, -3, 0}, {3, 3, 4});
  (void)m1;
  (void)m2;
}

int main(int argc, char** argv) {
  if (argc != 2) return 2;
  std::vector<float> tri;
  float x;
  while (std::cin >> x) tri.push_back(x);
  geometry::Mesh m;
  m.Init(4);
  m.Assign(tri.data(), tri.size() / 18);
  std::printf("%d\n", m.SaveToFile(argv[1]));
  return 0;
}

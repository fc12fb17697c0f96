// Reads "stamp m00 .. m33" (row-major float 4x4) lines from stdin, appends
// each pose to argv[1] with builder::writePoseToTxt, and prints the pose
// that builder::v2tRef rebuilds from the written values (row-major, %.9g).
#include <cstdio>
#include <vector>

#include "builder/builder.h"

int main(int argc, char** argv) {
  if (argc < 2) return 2;
  double stamp;
  float m[16];
  while (std::scanf("%lf", &stamp) == 1) {
    for (int i = 0; i < 16; ++i)
      if (std::scanf("%f", &m[i]) != 1) return 3;
    std::vector<double> v{stamp};
    DynaMap::builder::writePoseToTxt(argv[1], v, DynaMap::Matrix4f::from_row_major(m), 0);
  }
  std::FILE* f = std::fopen(argv[1], "r");
  if (!f) return 4;
  double t[8];
  while (std::fscanf(f, "%lf %lf %lf %lf %lf %lf %lf %lf", &t[0], &t[1], &t[2], &t[3], &t[4], &t[5],
                     &t[6], &t[7]) == 8) {
    std::vector<double> v(t, t + 8);
    const DynaMap::float4x4 p = DynaMap::builder::v2tRef(v).to_row_major();
    for (int i = 0; i < 16; ++i) std::printf(i ? " %.9g" : "%.9g", (double)p.entries[i]);
    std::printf("\n");
  }
  std::fclose(f);
  return 0;
}

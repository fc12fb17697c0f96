// Streams through the front end (include/nodeHandler/nodeHandler.h): one
// served session per line of a spec file, each fed by a TUM-layout
// directory replayed at a frame rate or by frames on standard input.
//   stream_example SPEC OUT [--evict HIGH_WATER MAX_AGE MARGIN] [--park BUDGET_BYTES]
//                           [--sequential]
// SPEC, one stream per line:
//   SOURCE rows cols fx fy cx cy scaler voxel buckets blocks trunc maxdepth
//   colour_weight precision rate_hz p00 .. p33 (first pose, row-major)
// SOURCE: a directory, several directories separated by commas (replayed
// into the stream in turn), or "-" for frames on standard input (the pipe
// format of PipeReader).  OUT, one line per frame as the pose callback
// reports it: "stream stamp status it0 it1 it2 p00 .. p33 blocks".  With
// --evict every stream gets the front end's eviction policy; with --evict
// or --park stdout ends with one line per stream: "counts stream evictions
// evicted uploaded stored parks resumes restored".  --park gives the server
// that budget and turns parking on (streams beyond the budget take turns);
// --sequential feeds one directory at a time, each replayed to its end and
// processed before the next starts: round r replays the r-th directory of
// every stream, streams in spec order.
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <memory>
#include <mutex>
#include <sstream>
#include <string>
#include <vector>

#include "nodeHandler/nodeHandler.h"

using namespace DynaMap;

int main(int argc, char** argv) {
  if (argc < 3) return 2;
  DynaMapNodeHandler::StreamConfig::EvictPolicy ev;
  size_t budget = size_t(24) << 30;
  bool park = false, sequential = false;
  for (int a = 3; a < argc; ++a) {
    const std::string opt = argv[a];
    if (opt == "--evict" && a + 3 < argc) {
      ev.enabled = true;
      ev.highWater = (float)std::atof(argv[a + 1]);
      ev.maxAge = std::atoi(argv[a + 2]);
      ev.margin = (float)std::atof(argv[a + 3]);
      a += 3;
    } else if (opt == "--park" && a + 1 < argc) {
      park = true;
      budget = (size_t)std::atoll(argv[++a]);
    } else if (opt == "--sequential") {
      sequential = true;
    } else {
      return 2;
    }
  }
  std::ifstream spec(argv[1]);
  std::vector<std::string> sources;
  std::vector<DynaMapNodeHandler::StreamConfig> cfgs;
  std::vector<double> rates;
  std::string line;
  while (std::getline(spec, line)) {
    if (line.empty()) continue;
    std::istringstream ss(line);
    std::string src;
    DynaMapNodeHandler::StreamConfig c;
    int log2b = 0;
    float pose[16];
    double rate = 0;
    ss >> src >> c.sensor.rows >> c.sensor.cols >> c.sensor.f.x >> c.sensor.f.y >> c.sensor.c.x >>
        c.sensor.c.y >> c.sensor.depthScaler >> c.tsdf.voxelSize >> log2b >> c.tsdf.numBlocks >>
        c.tsdf.truncationDistance >> c.tsdf.maxSensorDepth >> c.solver.colorWeight >>
        c.precision >> rate;
    for (float& v : pose) ss >> v;
    if (!ss) return 2;
    c.tsdf.numBuckets = 1 << log2b;
    c.tsdf.bucketSize = 10;
    c.tsdf.minSensorDepth = 0.15f;
    c.solver.lvlIterationNum[0] = 10;
    c.solver.lvlIterationNum[1] = 5;
    c.solver.lvlIterationNum[2] = 4;
    c.solver.icpMaxDepth = c.tsdf.maxSensorDepth;
    c.solver.huberConstant = 0.3f;
    c.pose0 = Matrix4f::from_row_major(pose);
    c.evict = ev;
    sources.push_back(src);
    cfgs.push_back(c);
    rates.push_back(rate);
  }
  std::FILE* out = std::fopen(argv[2], "w");
  if (!out) return 2;
  std::mutex out_mu;
  DynaMapNodeHandler node(budget);
  node.setParking(park);
  node.setPoseCallback([&](int stream, double stamp, const Matrix4f& P, const dyn_frame_stats& st,
                           dyn_status status) {
    std::lock_guard<std::mutex> lk(out_mu);
    std::fprintf(out, "%d %.6f %d %d %d %d", stream, stamp, (int)status, st.icp_iterations[0],
                 st.icp_iterations[1], st.icp_iterations[2]);
    for (int r = 0; r < 4; ++r)
      for (int k = 0; k < 4; ++k) std::fprintf(out, " %.9g", P(r, k));
    std::fprintf(out, " %lld\n", (long long)st.blocks_total);
  });
  std::vector<int> ids;
  for (auto& c : cfgs) ids.push_back(node.addStream(c));
  node.spin();
  std::vector<std::unique_ptr<TumReplayer>> replay;
  std::unique_ptr<PipeReader> pipe;
  std::vector<std::vector<std::string>> dirs(sources.size());
  size_t rounds = 0;
  for (size_t i = 0; i < sources.size(); ++i) {
    std::stringstream ss(sources[i]);
    std::string d;
    while (std::getline(ss, d, ','))
      if (!d.empty()) dirs[i].push_back(d);
    rounds = std::max(rounds, dirs[i].size());
  }
  for (size_t i = 0; i < sources.size(); ++i)
    if (sources[i] == "-") {
      pipe.reset(new PipeReader(node, ids[i], 0, cfgs[i].sensor.rows, cfgs[i].sensor.cols));
      pipe->start();
    }
  for (size_t r = 0; r < rounds; ++r)
    for (size_t i = 0; i < sources.size(); ++i) {
      if (sources[i] == "-" || r >= dirs[i].size()) continue;
      replay.emplace_back(new TumReplayer(node, ids[i], dirs[i][r], rates[i]));
      replay.back()->start();
      if (sequential || r + 1 < dirs[i].size()) {
        replay.back()->join();
        node.waitIdle();
      }
    }
  int sent = 0;
  for (auto& r : replay) {
    r->join();
    sent += r->sent();
  }
  if (pipe) {
    pipe->join();
    sent += pipe->sent();
    if (pipe->malformed()) return 3;
  }
  node.waitIdle();
  std::vector<DynaMapNodeHandler::StreamCounts> counts;
  for (int id : ids) counts.push_back(node.counts(id));
  for (int id : ids) node.removeStream(id);
  node.shutdown();
  std::fclose(out);
  std::printf("frames %d done %lld steps %lld\n", sent, (long long)node.framesDone(),
              (long long)node.steps());
  if (ev.enabled || park)
    for (size_t i = 0; i < ids.size(); ++i)
      std::printf("counts %d %lld %lld %lld %lld %lld %lld %lld\n", ids[i],
                  (long long)counts[i].evictions, (long long)counts[i].evicted,
                  (long long)counts[i].uploaded, (long long)counts[i].stored,
                  (long long)counts[i].parks, (long long)counts[i].resumes,
                  (long long)counts[i].restored);
  return node.framesDone() == sent ? 0 : 1;
}

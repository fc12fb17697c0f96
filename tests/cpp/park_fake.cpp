// Streams beyond the budget through the front end's parking policy
// (DynaMapNodeHandler::setParking), against the stand-in server of
// fake_server.cpp: a budget that holds one session, stream A fed frames
// 1-5, then stream B frames 1-5, then A frames 6-10, then B again while A
// keeps a frame queued; then the eviction policy on a stream whose map
// outgrows its pool.  Prints "ok" and returns 0 when every check holds,
// else prints what failed and returns 1.
#include <cstdio>
#include <map>
#include <mutex>
#include <vector>

#include "nodeHandler/nodeHandler.h"

using namespace DynaMap;

extern "C" const int64_t* fake_calls();

struct Row {
  double stamp;
  float x;
  int blocks;
  dyn_status status;
};

static int failures = 0;
#define CHECK(c)                                                   \
  do {                                                             \
    if (!(c)) {                                                    \
      std::printf("check failed (line %d): %s\n", __LINE__, #c);   \
      ++failures;                                                  \
    }                                                              \
  } while (0)

int main() {
  std::mutex mu;
  std::map<int, std::vector<Row>> rows;
  // the fake charges num_blocks * 100 bytes: one session of 4 blocks fits
  // in 600 bytes, two do not
  DynaMapNodeHandler node(600, 0, 8);
  node.setParking(true);
  node.setPoseCallback([&](int stream, double stamp, const Matrix4f& P, const dyn_frame_stats& st,
                           dyn_status status) {
    std::lock_guard<std::mutex> lk(mu);
    rows[stream].push_back({stamp, P(0, 3), st.blocks_total, status});
  });
  DynaMapNodeHandler::StreamConfig c;
  c.sensor.rows = 2;
  c.sensor.cols = 2;
  c.tsdf.numBlocks = 4;
  c.pose0 = Matrix4f::from_row_major(
      std::vector<float>{1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1}.data());
  const int a = node.addStream(c);
  const int b = node.addStream(c);  // beyond the budget: starts parked
  node.spin();
  auto feed = [&](int stream, int k0, int k1) {
    for (int k = k0; k <= k1; ++k) {
      uint16_t depth[4] = {(uint16_t)k, 0, 0, 0};
      node.kinect_callback(stream, depth, nullptr, (double)k);
      node.waitIdle();
    }
  };
  feed(a, 1, 5);
  const auto after_a = node.counts(a);
  feed(b, 1, 5);
  feed(a, 6, 10);
  // A parked again by B's return, then A's frame queued while B runs
  feed(b, 6, 7);
  {
    uint16_t d1[4] = {8, 0, 0, 0}, d2[4] = {11, 0, 0, 0};
    node.kinect_callback(b, d1, nullptr, 8.0);
    node.kinect_callback(a, d2, nullptr, 11.0);
    node.waitIdle();
  }
  const auto ca = node.counts(a), cb = node.counts(b);
  node.removeStream(a);
  node.removeStream(b);
  node.shutdown();

  std::lock_guard<std::mutex> lk(mu);
  CHECK(after_a.parks == 0 && after_a.resumes == 0);
  CHECK(rows[a].size() == 11 && rows[b].size() == 8);
  for (auto& kv : rows)
    for (size_t i = 0; i < kv.second.size(); ++i) {
      CHECK(kv.second[i].status == DYN_OK);
      if (i) CHECK(kv.second[i].stamp > kv.second[i - 1].stamp);  // in frame order
    }
  // A: 5 frames of 3 blocks each, parked, resumed with its 15 blocks back;
  // its first frame after the resume keeps the pose, later ones move on
  CHECK(rows[a][4].blocks == 15 && rows[a][5].blocks == 18);
  CHECK(rows[a][5].x == rows[a][4].x);
  CHECK(rows[a][9].blocks == 30 && rows[a][10].blocks == 33);
  CHECK(ca.parks == 2 && ca.resumes == 2 && ca.restored == 15 + 30);
  // B: started parked (no session yet), admitted, parked when A came back,
  // resumed with its 15 blocks, parked again for A's last frame once its
  // own frame 8 was done (A's frame waited while B had one queued)
  CHECK(cb.parks == 2 && cb.resumes == 2 && cb.restored == 15);
  CHECK(rows[b][4].blocks == 15 && rows[b][5].blocks == 18 && rows[b][7].blocks == 24);
  const int64_t* calls = fake_calls();
  // admissions: A at addStream, then B, A, B, A; releases: the four parks
  // (and A's removal, if the serving thread ran once more before shutdown)
  std::printf("admissions %lld releases %lld\n", (long long)calls[0], (long long)calls[1]);
  CHECK(calls[0] == 5 && calls[1] >= 4);

  // the eviction policy on a stream whose map outgrows 60 % of a 10-block
  // pool: blocks of frames more than one frame old go to the host store;
  // every evicted block is stored or was uploaded back, and eviction
  // repeats as the map grows (its buffers reused)
  {
    DynaMapNodeHandler ev(1 << 20, 0, 8);
    DynaMapNodeHandler::StreamConfig e = c;
    e.tsdf.numBlocks = 10;
    e.evict.enabled = true;
    e.evict.highWater = 0.6f;
    e.evict.maxAge = 1;
    int done = 0;
    ev.setPoseCallback([&](int, double, const Matrix4f&, const dyn_frame_stats&,
                           dyn_status status) {
      if (status == DYN_OK) ++done;
    });
    const int id = ev.addStream(e);
    ev.spin();
    for (int k = 1; k <= 12; ++k) {
      uint16_t depth[4] = {(uint16_t)k, 0, 0, 0};
      ev.kinect_callback(id, depth, nullptr, (double)k);
      ev.waitIdle();
    }
    const auto ce = ev.counts(id);
    ev.removeStream(id);
    ev.shutdown();
    std::printf("evictions %lld evicted %lld uploaded %lld stored %lld\n",
                (long long)ce.evictions, (long long)ce.evicted, (long long)ce.uploaded,
                (long long)ce.stored);
    CHECK(done == 12);
    CHECK(ce.evictions >= 5 && ce.evicted >= 15);
    CHECK(ce.stored + ce.uploaded == ce.evicted);
  }
  if (failures) return 1;
  std::printf("ok\n");
  return 0;
}

// nodeHandler/nodeHandler.h -- the streaming front end: RGB-D streams in,
// one pose per frame out, through the serving loop (dyn_server).
//
// It takes the place of the reference's ROS node
// (include/nodeHandler/nodeHandler.h:50-90, nodeHandler.cpp): there each
// synchronised depth + colour message pair reaches kinect_callback
// (nodeHandler.cpp:170), which converts the images and runs the mapper, and
// tf_publisher (:139-153) broadcasts the estimated camera pose.  ROS is not
// part of this build, so a stream is fed in-process: kinect_callback may be
// called from any thread (a camera driver's, a decoder's, one of the
// replayers below) and copies the frame into the stream's queue; one
// serving thread steps the server whenever frames wait -- all streams'
// waiting frames fused into one launch per stage (continuous batching) --
// and hands each result to the pose callback, in each stream's frame order.
// Every frame is processed; a stream has at most one frame on the device at
// a time, so its results equal the same frames stepped alone.
//
// Sources: TumReplayer replays a TUM-layout directory (utils::dataSet) at a
// frame rate; PipeReader reads frames from a file descriptor (a pipe from a
// capture process) in a small binary format (see PipeReader).
//
// A stream's block pool is fixed when it is admitted.  With an eviction
// policy (StreamConfig::evict) the front end keeps it from filling: after a
// frame whose map holds more than highWater of the pool, the blocks the
// allocation has not touched for more than maxAge frames move to a host
// store (dyn_evict_blocks, the reference's unused HashTable::DeleteBlock
// applied by age); before each frame, stored blocks that the camera at its
// last pose can see -- within the sensor's range and image, widened by a
// margin -- go back (dyn_upload_blocks), so a revisited place keeps what
// was fused into it.
//
// Streams beyond the HBM budget (setParking(true)): a stream that does not
// fit when it is added starts parked, and a parked stream with a frame
// waiting is admitted in place of the admitted stream idle the longest (no
// frame queued or on the device), which is parked: its blocks go to host
// memory (dyn_download_blocks) and its slot and device bytes are released.
// A resumed stream gets a new session at its last pose with its blocks
// uploaded back (dyn_upload_blocks); its first frame is integrated at that
// pose without tracking (the new session has no target yet), the frames
// after it track against the restored map.
//
// Header-only over the C ABI of dynamap.h; needs C++17 and threads.
#pragma once

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstdint>
#include <cstring>
#include <deque>
#include <functional>
#include <cmath>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include <unistd.h>

#include "../builder/builder.h"
#include "../dynamap.h"
#include "../dynamap/types.h"
#include "../utils/dataSet.h"

namespace DynaMap {

class DynaMapNodeHandler {
 public:
  // one stream: the builder's init arguments (builder.h:51-54) plus the
  // voxel form and the first pose
  struct StreamConfig {
    tsdf::tsdfProperties tsdf;
    solver::Properties solver;
    rgbdSensor sensor;
    gaussianKernal kernel;
    int mode = 1;  // 0 frame-to-frame, 1 frame-to-model
    int precision = DYN_PRECISION_FP32;
    Matrix4f pose0;
    bool bilateral = true;
    struct EvictPolicy {
      bool enabled = false;
      float highWater = 0.85f;  // share of the pool that triggers an eviction
      int maxAge = 4;           // blocks untouched for more frames leave
      float margin = 0.1f;      // metres the upload's view test is widened by
    } evict;
  };
  struct StreamCounts {
    int64_t evictions = 0, evicted = 0, uploaded = 0, stored = 0;
    int64_t parks = 0, resumes = 0;  // times parked / resumed (setParking)
    int64_t restored = 0;            // blocks uploaded back at resumes
  };
  // tf_publisher's role: the frame's time stamp, its camera pose and the
  // frame's statistics (status: the frame's dyn_status, e.g. a full heap)
  using PoseCallback = std::function<void(int stream, double stamp, const Matrix4f& pose,
                                          const dyn_frame_stats& stats, dyn_status status)>;

  explicit DynaMapNodeHandler(size_t budget_bytes = 0, int device = 0, int max_sessions = 64) {
    dyn_server_params p;
    p.budget_bytes = budget_bytes;
    p.max_sessions = max_sessions;
    p.device = device;
    dyn_throw("DynaMapNodeHandler", dyn_server_create(&p, &server_));
  }
  DynaMapNodeHandler(const DynaMapNodeHandler&) = delete;
  DynaMapNodeHandler& operator=(const DynaMapNodeHandler&) = delete;
  virtual ~DynaMapNodeHandler() {
    shutdown();
    if (server_) dyn_server_destroy(server_);
  }

  void setPoseCallback(PoseCallback cb) {
    std::lock_guard<std::mutex> lk(mu_);
    on_pose_ = std::move(cb);
  }

  // Streams beyond the budget are parked and resumed in turn instead of
  // refused (see the header comment).  Off by default.
  void setParking(bool on) {
    std::lock_guard<std::mutex> lk(server_mu_);
    parking_ = on;
  }

  // Admits a stream; returns its id.  Throws when the budget or the slots
  // are exhausted (DYN_ERR_BUDGET_EXCEEDED: add it after another stream
  // has been removed), unless parking is on: then the stream starts
  // parked and is admitted when it has a frame.
  int addStream(const StreamConfig& c) {
    std::lock_guard<std::mutex> lk(server_mu_);
    int32_t slot = -1;
    const dyn_status r = admit(c, c.pose0, &slot);
    if (!(r == DYN_ERR_BUDGET_EXCEEDED && parking_))
      dyn_throw("DynaMapNodeHandler::addStream", r);
    std::lock_guard<std::mutex> lk2(mu_);
    auto st = std::make_shared<Stream>();
    st->slot = slot;
    st->last_active = steps_;
    st->npx = (size_t)c.sensor.rows * c.sensor.cols;
    st->scaler = c.sensor.depthScaler;
    st->cfg = c;
    st->pose = c.pose0;
    const int id = next_id_++;
    streams_[id] = st;
    return id;
  }

  // nodeHandler.cpp:170: one frame of a stream (uint16 depth in sensor
  // units, rows*cols; RGB triplets or null).  The frame is copied; the call
  // returns at once.
  void kinect_callback(int stream, const uint16_t* depth, const uint8_t* rgb, double stamp) {
    std::unique_lock<std::mutex> lk(mu_);
    auto it = streams_.find(stream);
    if (it == streams_.end() || it->second->closing)
      dyn_throw("DynaMapNodeHandler::kinect_callback", DYN_ERR_INVALID_ARG);
    Stream& s = *it->second;
    Frame f;
    f.stamp = stamp;
    f.depth.assign(depth, depth + s.npx);
    if (rgb) f.rgb.assign(rgb, rgb + 3 * s.npx);
    s.queue.push_back(std::move(f));
    ++queued_;
    cv_.notify_all();
  }
  // the reference's own input: depth in metres (TYPE_32FC1), turned into
  // sensor units (rounded depth * depthScaler, 0 where not positive)
  void kinect_callback(int stream, const float* depth_m, const uint8_t* rgb, double stamp) {
    size_t n = 0;
    float scaler = 1.0f;
    {
      std::lock_guard<std::mutex> lk(mu_);
      auto it = streams_.find(stream);
      if (it == streams_.end()) dyn_throw("DynaMapNodeHandler::kinect_callback", DYN_ERR_INVALID_ARG);
      n = it->second->npx;
      scaler = it->second->scaler;
    }
    std::vector<uint16_t> u(n);
    for (size_t i = 0; i < n; ++i) {
      const float v = depth_m[i] * scaler;
      u[i] = (depth_m[i] > 0.0f && v < 65535.5f) ? (uint16_t)(v + 0.5f) : (uint16_t)0;
    }
    kinect_callback(stream, u.data(), rgb, stamp);
  }

  // Stops taking frames for the stream; it is released once its queued
  // frames have been processed.
  void removeStream(int stream) {
    std::lock_guard<std::mutex> lk(mu_);
    auto it = streams_.find(stream);
    if (it != streams_.end()) it->second->closing = true;
    cv_.notify_all();
  }

  // Starts the serving thread (ros::spin's role).
  void spin() {
    if (worker_.joinable()) return;
    running_ = true;
    worker_ = std::thread([this] { serve(); });
  }
  // Waits until every queued frame has been processed and reported.
  void waitIdle() {
    std::unique_lock<std::mutex> lk(mu_);
    idle_cv_.wait(lk, [this] { return queued_ == 0 || !running_; });
  }
  void shutdown() {
    {
      std::lock_guard<std::mutex> lk(mu_);
      running_ = false;
    }
    cv_.notify_all();
    if (worker_.joinable()) worker_.join();
    idle_cv_.notify_all();
  }
  // eviction and upload counts of a stream (its host store's blocks)
  StreamCounts counts(int stream) {
    std::lock_guard<std::mutex> lk(mu_);
    auto it = streams_.find(stream);
    return it == streams_.end() ? StreamCounts() : it->second->counts;
  }
  // frames processed, steps run (several frames share a step)
  int64_t framesDone() const { return frames_done_; }
  int64_t steps() const { return steps_; }
  dyn_server* server() const { return server_; }
  // the session behind a stream (raycast, mesh, download), only while the
  // stream is idle
  dyn_session* session(int stream) {
    std::lock_guard<std::mutex> slk(server_mu_);  // server first, as everywhere
    std::lock_guard<std::mutex> lk(mu_);
    auto it = streams_.find(stream);
    if (it == streams_.end() || it->second->slot < 0) return nullptr;
    dyn_session* out = nullptr;
    dyn_server_session(server_, it->second->slot, &out);
    return out;
  }

 private:
  struct Frame {
    double stamp = 0.0;
    std::vector<uint16_t> depth;
    std::vector<uint8_t> rgb;
  };
  struct Stream {
    int32_t slot = -1;  // -1 while parked
    size_t npx = 0;
    float scaler = 1.0f;
    std::deque<Frame> queue;
    bool in_flight = false;  // a frame pushed and stepped, result not yet read
    double stamp = 0.0;      // that frame's
    bool closing = false;
    StreamConfig cfg;
    Matrix4f pose;           // after the last reported frame
    // evicted blocks: packed coordinate -> 512 voxels
    std::unordered_map<uint64_t, std::vector<dyn_voxel>> store;
    StreamCounts counts;
    // while parked: the blocks its session held (coordinates, 512 voxels each)
    std::vector<int32_t> park_coords;
    std::vector<dyn_voxel> park_vox;
    int64_t last_active = 0;  // the step of its last admission or result
    // host buffers the eviction hands blocks out into, grown when the map
    // outgrows them and kept (not cleared) between evictions
    std::vector<int32_t> evict_coords;
    std::unique_ptr<dyn_voxel[]> evict_vox;
    int64_t evict_cap = 0;
  };

  dyn_status admit(const StreamConfig& c, const Matrix4f& pose, int32_t* slot) {
    dyn_tsdf_params t = c.tsdf.to_c();
    dyn_gn_params g = c.solver.to_c(c.mode);
    dyn_bilateral_params b;
    b.diameter = c.kernel.diameter;
    b.sigma_i = c.kernel.sigmaI;
    b.sigma_s = c.kernel.sigmaS;
    b.enabled = c.bilateral ? 1 : 0;
    dyn_sensor s = c.sensor.to_c();
    float4x4 p0 = pose.to_row_major();
    return dyn_server_admit(server_, &t, &g, &b, &s, c.precision, p0.entries, slot);
  }

  // Parks an idle stream: its blocks to host memory, its slot released
  // (server lock held; the stream has no frame on the device).
  bool park(Stream& v) {
    dyn_session* sess = nullptr;
    if (dyn_server_session(server_, v.slot, &sess) != DYN_OK || !sess) return false;
    int64_t n = 0, got = 0;
    if (dyn_num_blocks(sess, &n) != DYN_OK) return false;
    v.park_coords.resize((size_t)n * 3);
    v.park_vox.resize((size_t)n * 512);
    if (n > 0 && dyn_download_blocks(sess, v.park_coords.data(), v.park_vox.data(), n, &got) !=
                     DYN_OK)
      return false;
    v.park_coords.resize((size_t)std::min(got, n) * 3);
    v.park_vox.resize((size_t)std::min(got, n) * 512);
    if (dyn_server_release(server_, v.slot) != DYN_OK) return false;
    std::lock_guard<std::mutex> lk(mu_);
    v.slot = -1;
    v.counts.parks++;
    return true;
  }

  // Admits a parked stream that has a frame waiting, parking the admitted
  // streams idle the longest while the budget does not hold it (server
  // lock held).  False when no idle stream is left to park.
  bool resume(Stream& s) {
    int32_t slot = -1;
    while (true) {
      const dyn_status r = admit(s.cfg, s.pose, &slot);
      if (r == DYN_OK) break;
      if (r != DYN_ERR_BUDGET_EXCEEDED) return false;
      Stream* victim = nullptr;
      {
        std::lock_guard<std::mutex> lk(mu_);
        for (auto& kv : streams_) {
          Stream& v = *kv.second;
          if (&v == &s || v.slot < 0 || v.in_flight || !v.queue.empty()) continue;
          if (!victim || v.last_active < victim->last_active) victim = &v;
        }
      }
      if (!victim || !park(*victim)) return false;
    }
    const int64_t n = (int64_t)s.park_coords.size() / 3;
    int64_t counts[4] = {0, 0, 0, 0};
    if (n > 0) {
      dyn_session* sess = nullptr;
      dyn_server_session(server_, slot, &sess);
      if (sess) dyn_upload_blocks(sess, s.park_coords.data(), s.park_vox.data(), n, counts);
    }
    std::vector<int32_t>().swap(s.park_coords);
    std::vector<dyn_voxel>().swap(s.park_vox);
    std::lock_guard<std::mutex> lk(mu_);
    s.slot = slot;
    s.last_active = steps_;
    s.counts.resumes++;
    s.counts.restored += counts[0];
    return true;
  }
  static uint64_t block_key(int x, int y, int z) {
    const uint64_t m = (1ull << 21) - 1;
    return (((uint64_t)x & m) << 42) | (((uint64_t)y & m) << 21) | ((uint64_t)z & m);
  }
  static int key_part(uint64_t k, int shift) {
    return (int)((int64_t)(((k >> shift) & ((1ull << 21) - 1)) << 43) >> 43);
  }

  // Stored blocks the camera at the stream's last pose can see go back into
  // its volume (server lock held; the stream has no frame on the device).
  void upload_visible(Stream& s) {
    if (!s.cfg.evict.enabled || s.store.empty()) return;
    const float bs = s.cfg.tsdf.voxelSize * (float)s.cfg.tsdf.blockSize;
    const float r = bs * 0.8660254f + s.cfg.evict.margin;  // half diagonal + margin
    const rgbdSensor& sn = s.cfg.sensor;
    const Matrix4f& P = s.pose;
    std::vector<int32_t> coords;
    std::vector<dyn_voxel> vox;
    std::vector<uint64_t> taken;
    for (const auto& kv : s.store) {
      const int x = key_part(kv.first, 42), y = key_part(kv.first, 21), z = key_part(kv.first, 0);
      const float c[3] = {((float)x + 0.5f) * bs, ((float)y + 0.5f) * bs, ((float)z + 0.5f) * bs};
      float q[3];  // R^T (c - t)
      for (int i = 0; i < 3; ++i)
        q[i] = P(0, i) * (c[0] - P(0, 3)) + P(1, i) * (c[1] - P(1, 3)) + P(2, i) * (c[2] - P(2, 3));
      if (q[2] < -r || q[2] > s.cfg.tsdf.maxSensorDepth + r) continue;
      bool in = q[2] <= r;  // around the camera: always
      if (!in) {
        const float u = sn.f.x * q[0] / q[2] + sn.c.x, v = sn.f.y * q[1] / q[2] + sn.c.y;
        const float pu = sn.f.x * r / q[2], pv = sn.f.y * r / q[2];
        in = u >= -pu && u <= (float)sn.cols + pu && v >= -pv && v <= (float)sn.rows + pv;
      }
      if (!in) continue;
      coords.insert(coords.end(), {x, y, z});
      vox.insert(vox.end(), kv.second.begin(), kv.second.end());
      taken.push_back(kv.first);
    }
    if (taken.empty()) return;
    dyn_session* sess = nullptr;
    dyn_server_session(server_, s.slot, &sess);
    int64_t counts[4] = {0, 0, 0, 0};
    if (sess && dyn_upload_blocks(sess, coords.data(), vox.data(), (int64_t)taken.size(), counts) ==
                    DYN_OK) {
      for (uint64_t k : taken) s.store.erase(k);
      std::lock_guard<std::mutex> lk(mu_);
      s.counts.uploaded += counts[0];
      s.counts.stored = (int64_t)s.store.size();
    }
  }

  // After a frame: the pool past its high-water mark sends the blocks the
  // allocation has not touched for maxAge frames to the host store.
  void evict_old(Stream& s, const dyn_frame_stats& st) {
    const auto& e = s.cfg.evict;
    if (!e.enabled || (double)st.blocks_total <= (double)e.highWater * s.cfg.tsdf.numBlocks) return;
    dyn_session* sess = nullptr;
    dyn_server_session(server_, s.slot, &sess);
    if (!sess) return;
    // every allocated block may leave, so the buffers hold them all
    const int64_t cap = st.blocks_total;
    if (cap > s.evict_cap) {
      s.evict_coords.resize((size_t)cap * 3);
      s.evict_vox.reset(new dyn_voxel[(size_t)cap * 512]);
      s.evict_cap = cap;
    }
    const int32_t* coords = s.evict_coords.data();
    const dyn_voxel* vox = s.evict_vox.get();
    int64_t n = 0;
    if (dyn_evict_blocks(sess, e.maxAge, s.evict_coords.data(), s.evict_vox.get(), cap, &n) !=
        DYN_OK)
      return;
    const int64_t m = n < cap ? n : cap;
    for (int64_t i = 0; i < m; ++i)
      s.store[block_key(coords[3 * i], coords[3 * i + 1], coords[3 * i + 2])] =
          std::vector<dyn_voxel>(vox + i * 512, vox + (i + 1) * 512);
    std::lock_guard<std::mutex> lk(mu_);
    s.counts.evictions++;
    s.counts.evicted += m;
    s.counts.stored = (int64_t)s.store.size();
  }

  // One pass: push the next frame of every stream without a frame on the
  // device, step once, then report the results that are ready.
  struct Refused {
    int id;
    double stamp;
    dyn_status status;
  };
  void serve() {
    std::vector<std::pair<int, std::shared_ptr<Stream>>> ready;
    std::vector<Refused> refused;
    while (true) {
      ready.clear();
      {
        std::unique_lock<std::mutex> lk(mu_);
        cv_.wait_for(lk, std::chrono::milliseconds(1), [this] {
          if (!running_) return true;
          for (auto& kv : streams_)
            if (!kv.second->in_flight && !kv.second->queue.empty()) return true;
          return in_flight_ > 0;
        });
        if (!running_ && in_flight_ == 0) break;
        for (auto& kv : streams_) ready.push_back(kv);
      }
      int pushed = 0;
      bool waiting_parked = false;  // a parked stream found no idle stream to replace
      {
        std::lock_guard<std::mutex> slk(server_mu_);
        for (auto& [id, s] : ready) {
          Frame f;
          bool parked;
          {
            std::lock_guard<std::mutex> lk(mu_);
            if (s->in_flight || s->queue.empty()) continue;
            parked = s->slot < 0;
          }
          if (parked && !resume(*s)) {  // waits for an idle stream
            waiting_parked = true;
            continue;
          }
          {
            std::lock_guard<std::mutex> lk(mu_);
            f = std::move(s->queue.front());
            s->queue.pop_front();
          }
          upload_visible(*s);
          const dyn_status r = dyn_server_push(server_, s->slot, f.depth.data(),
                                               f.rgb.empty() ? nullptr : f.rgb.data());
          if (r == DYN_ERR_NOT_READY) {  // not stepped yet: put it back
            std::lock_guard<std::mutex> lk(mu_);
            s->queue.push_front(std::move(f));
            continue;
          }
          if (r != DYN_OK) {  // refused (a malformed frame): reported below, dropped
            refused.push_back({id, f.stamp, r});
            continue;
          }
          std::lock_guard<std::mutex> lk(mu_);
          s->in_flight = true;
          s->stamp = f.stamp;
          ++in_flight_;
          ++pushed;
        }
        if (pushed) {
          int32_t n = 0;
          dyn_throw("DynaMapNodeHandler: step", dyn_server_step(server_, &n));
          ++steps_;
        }
      }
      // nothing to step while a parked stream waits: back off instead of
      // spinning (its wake-up condition stays true until a stream idles)
      if (!pushed && waiting_parked) {
        bool none;
        {
          std::lock_guard<std::mutex> lk(mu_);
          none = in_flight_ == 0;
        }
        if (none) std::this_thread::sleep_for(std::chrono::microseconds(200));
      }
      for (const Refused& x : refused) report(x.id, x.stamp, nullptr, nullptr, x.status);
      refused.clear();
      // results, in each stream's order (one frame per stream in flight)
      for (auto& [id, s] : ready) {
        bool fl;
        {
          std::lock_guard<std::mutex> lk(mu_);
          fl = s->in_flight;
        }
        if (!fl) continue;
        float pose[16];
        dyn_frame_stats st;
        dyn_status r;
        {
          std::lock_guard<std::mutex> slk(server_mu_);
          int32_t done = 0;
          dyn_throw("DynaMapNodeHandler: poll", dyn_server_poll(server_, s->slot, &done));
          if (!done) continue;
          r = dyn_server_result(server_, s->slot, pose, &st);
          s->pose = Matrix4f::from_row_major(pose);
          s->last_active = steps_;
          evict_old(*s, st);
        }
        {
          std::lock_guard<std::mutex> lk(mu_);
          s->in_flight = false;
          --in_flight_;
        }
        report(id, s->stamp, pose, &st, r);
      }
      // streams that were removed and have nothing left
      std::lock_guard<std::mutex> slk(server_mu_);
      std::lock_guard<std::mutex> lk(mu_);
      for (auto it = streams_.begin(); it != streams_.end();) {
        Stream& s = *it->second;
        if (s.closing && s.queue.empty() && !s.in_flight) {
          if (s.slot >= 0) dyn_server_release(server_, s.slot);
          it = streams_.erase(it);
        } else {
          ++it;
        }
      }
    }
  }

  // the pose callback for one handed-over frame (pose null: the frame was
  // refused), then the frame counts as done
  void report(int id, double stamp, const float* pose, const dyn_frame_stats* st, dyn_status r) {
    PoseCallback cb;
    {
      std::lock_guard<std::mutex> lk(mu_);
      cb = on_pose_;
    }
    dyn_frame_stats none{};
    if (cb)
      cb(id, stamp, pose ? Matrix4f::from_row_major(pose) : Matrix4f(), st ? *st : none, r);
    std::lock_guard<std::mutex> lk(mu_);
    --queued_;
    ++frames_done_;
    if (queued_ == 0) idle_cv_.notify_all();
  }

  dyn_server* server_ = nullptr;
  std::mutex mu_;         // streams, queues, counters, callback
  std::mutex server_mu_;  // calls on the server (not thread-safe)
  std::condition_variable cv_, idle_cv_;
  std::map<int, std::shared_ptr<Stream>> streams_;
  PoseCallback on_pose_;
  std::thread worker_;
  bool running_ = false;
  int next_id_ = 0;
  bool parking_ = false;
  int64_t queued_ = 0;  // frames handed over and not yet reported
  int in_flight_ = 0;
  std::atomic<int64_t> frames_done_{0}, steps_{0};
};

// Replays a TUM-layout directory into a stream at 'rate_hz' frames per
// second (0: as fast as the stream takes them), stamps from the files.
class TumReplayer {
 public:
  TumReplayer(DynaMapNodeHandler& h, int stream, std::string dir, double rate_hz)
      : h_(h), stream_(stream), dir_(std::move(dir)), rate_(rate_hz) {}
  ~TumReplayer() { join(); }
  void start() {
    th_ = std::thread([this] {
      utils::dataSet ds(dir_);
      const auto t0 = std::chrono::steady_clock::now();
      for (size_t k = 0; k < ds.size(); ++k) {
        if (rate_ > 0)
          std::this_thread::sleep_until(t0 + std::chrono::duration<double>((double)k / rate_));
        ds.invokeNextFrame();
        h_.kinect_callback(stream_, ds.image.depth.data(),
                           ds.image.rgb.empty() ? nullptr : ds.image.rgb.data(), ds.stamp);
        ++sent_;
      }
    });
  }
  void join() {
    if (th_.joinable()) th_.join();
  }
  int sent() const { return sent_; }

 private:
  DynaMapNodeHandler& h_;
  int stream_;
  std::string dir_;
  double rate_;
  std::thread th_;
  std::atomic<int> sent_{0};
};

// Frames from a file descriptor (a pipe): per frame a 32-byte header
//   char magic[4] = "DYNF"; uint32 rows, cols, flags (bit 0: RGB follows);
//   double stamp; uint64 reserved (0)
// then rows*cols uint16 depth (sensor units, little-endian) and, with
// bit 0, rows*cols*3 bytes RGB.  End of file ends the stream.
class PipeReader {
 public:
  PipeReader(DynaMapNodeHandler& h, int stream, int fd, uint32_t rows, uint32_t cols)
      : h_(h), stream_(stream), fd_(fd), rows_(rows), cols_(cols) {}
  ~PipeReader() { join(); }
  void start() {
    th_ = std::thread([this] {
      const size_t n = (size_t)rows_ * cols_;
      std::vector<uint16_t> d(n);
      std::vector<uint8_t> c(3 * n);
      while (true) {
        unsigned char hdr[32];
        if (!read_all(hdr, sizeof hdr)) break;
        uint32_t rows, cols, flags;
        double stamp;
        std::memcpy(&rows, hdr + 4, 4);
        std::memcpy(&cols, hdr + 8, 4);
        std::memcpy(&flags, hdr + 12, 4);
        std::memcpy(&stamp, hdr + 16, 8);
        if (std::memcmp(hdr, "DYNF", 4) != 0 || rows != rows_ || cols != cols_) {
          bad_ = true;
          break;
        }
        if (!read_all(d.data(), 2 * n)) break;
        if ((flags & 1) && !read_all(c.data(), 3 * n)) break;
        h_.kinect_callback(stream_, d.data(), (flags & 1) ? c.data() : nullptr, stamp);
        ++sent_;
      }
    });
  }
  void join() {
    if (th_.joinable()) th_.join();
  }
  int sent() const { return sent_; }
  bool malformed() const { return bad_; }

 private:
  bool read_all(void* p, size_t n) {
    char* q = static_cast<char*>(p);
    while (n > 0) {
      const ssize_t r = ::read(fd_, q, n);
      if (r <= 0) return false;
      q += r;
      n -= (size_t)r;
    }
    return true;
  }
  DynaMapNodeHandler& h_;
  int stream_, fd_;
  uint32_t rows_, cols_;
  std::thread th_;
  std::atomic<int> sent_{0};
  std::atomic<bool> bad_{false};
};

}  // namespace DynaMap

// serving.cu -- many sessions on one device: dyn_batch (a fixed set stepped
// together, one CUDA graph per frame) and dyn_server (sessions admitted and
// released at any time under an HBM budget, every step fusing the frames
// that are waiting into one launch per stage).  No counterpart in the
// reference, whose builder drives one stream.
#include <algorithm>
#include <cstdio>
#include <map>
#include <mutex>
#include <new>

#include "session_impl.cuh"

using namespace dyn;
using namespace dyn::host;

extern "C" {

// ---------------------------------------------------------------- batches

// Resident blocks of group g's persistent ICP out of 'cap': in proportion
// to the group's level-0 pixel tiles among all groups' (at least one).
static int group_budget(const std::vector<dyn_session*>& sorted, const std::vector<int>& start,
                        int g, int cap) {
  long long all = 0, mine = 0;
  const int k = (int)start.size() - 1;
  for (int h = 0; h < k; ++h)
    for (int j = start[h]; j < start[h + 1]; ++j) {
      const long long t = icp_tiles((int)sorted[j]->npx);
      all += t;
      if (h == g) mine += t;
    }
  if (all <= 0) return 0;
  return std::max(1, (int)((long long)cap * mine / all));
}

dyn_status dyn_batch_create(dyn_session* const* sessions, int32_t n, dyn_batch** out) {
  if (!out) return DYN_ERR_INVALID_ARG;
  *out = nullptr;
  if (!sessions || n < 1 || n > 65535) return DYN_ERR_INVALID_ARG;
  for (int i = 0; i < n; ++i) {
    if (!sessions[i] || sessions[i]->batch || sessions[i]->device != sessions[0]->device)
      return DYN_ERR_INVALID_ARG;
    for (int j = 0; j < i; ++j)
      if (sessions[j] == sessions[i]) return DYN_ERR_INVALID_ARG;
  }
  DeviceGuard dg(sessions[0]->device);
  dyn_batch* b = new (std::nothrow) dyn_batch();
  if (!b) return DYN_ERR_OOM;
  b->device = sessions[0]->device;
  b->n = n;
  b->ss.assign(sessions, sessions + n);
  int64_t cap = 0;
  for (int i = 0; i < n; ++i) {
    if (cudaStreamSynchronize(sessions[i]->stream) != cudaSuccess) {
      delete b;
      return DYN_ERR_CUDA;
    }
    cap += sessions[i]->tp.num_blocks;
  }
  if (cap > INT32_MAX) {
    delete b;
    return DYN_ERR_INVALID_ARG;
  }
  auto dalloc = [&](void** p, size_t bytes) -> dyn_status {
    cudaError_t e = cudaMalloc(p, bytes < 256 ? 256 : bytes);
    if (e != cudaSuccess) {
      cudaGetLastError();
      return e == cudaErrorMemoryAllocation ? DYN_ERR_OOM : DYN_ERR_CUDA;
    }
    b->allocs.push_back(*p);
    return DYN_OK;
  };
  dyn_status r = DYN_OK;
  if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&b->h2d_done, cudaEventDisableTiming) != cudaSuccess ||
      cudaMallocHost(&b->h_res, sizeof(ResultBlock) * (size_t)n) != cudaSuccess)
    r = DYN_ERR_CUDA;
  // members in decreasing image size, split into runs of about equal pixel
  // count (one run per 4 members, at most kMaxGroups): sessions of a group
  // have similar grids, and the groups' streams overlap each other's tails
  // (32 mixed-size members: 8 groups 2.2 % faster than 4)
  std::vector<int> order((size_t)n);
  for (int i = 0; i < n; ++i) order[i] = i;
  std::stable_sort(order.begin(), order.end(),
                   [&](int a, int c) { return sessions[a]->npx > sessions[c]->npx; });
  const int k = std::max(1, std::min(kMaxGroups, n / 4));
  std::vector<int> start(k + 1, n);
  {
    double total = 0.0, acc = 0.0;
    for (int i = 0; i < n; ++i) total += (double)sessions[i]->npx;
    int g = 1;
    start[0] = 0;
    for (int j = 0; j < n && g < k; ++j) {
      acc += (double)sessions[order[j]]->npx;
      // close group g-1 once it holds its share (leaving a member per later group)
      if (acc >= total * g / k && j + 1 <= n - (k - g)) start[g++] = j + 1;
    }
    for (; g < k; ++g) start[g] = std::max(start[g - 1] + 1, n - (k - g));
    start[k] = n;
  }
  if (r == DYN_OK) r = dalloc((void**)&b->d_tab, sizeof(SessDev) * (size_t)n);
  if (r == DYN_OK) r = dalloc((void**)&b->d_map, sizeof(int) * (size_t)n);
  if (r == DYN_OK) r = dalloc((void**)&b->d_gvis, sizeof(int2) * (size_t)cap);
  if (r == DYN_OK) r = dalloc((void**)&b->d_gcount, sizeof(int) * kMaxGroups);
  if (r == DYN_OK) r = dalloc((void**)&b->d_icp_bar, kIcpBarWords * sizeof(unsigned) * kMaxGroups);
  if (r == DYN_OK) r = dalloc((void**)&b->d_res, sizeof(ResultBlock) * (size_t)n);
  for (int g = 1; g < k && r == DYN_OK; ++g)
    if (cudaStreamCreateWithFlags(&b->groups.st[g], cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&b->groups.join[g], cudaEventDisableTiming) != cudaSuccess)
      r = DYN_ERR_CUDA;
  if (r == DYN_OK &&
      cudaEventCreateWithFlags(&b->groups.fork, cudaEventDisableTiming) != cudaSuccess)
    r = DYN_ERR_CUDA;
  std::vector<dyn_session*> sorted((size_t)n);
  if (r == DYN_OK) {
    std::vector<SessDev> tab((size_t)n);
    std::vector<int> map((size_t)n);
    for (int j = 0; j < n; ++j) {
      sorted[j] = sessions[order[j]];
      tab[j] = sorted[j]->hsd;
      map[j] = order[j];
    }
    if (cudaMemcpyAsync(b->d_tab, tab.data(), sizeof(SessDev) * (size_t)n,
                        cudaMemcpyHostToDevice, b->stream) != cudaSuccess ||
        cudaMemcpyAsync(b->d_map, map.data(), sizeof(int) * (size_t)n, cudaMemcpyHostToDevice,
                        b->stream) != cudaSuccess ||
        cudaEventRecord(b->h2d_done, b->stream) != cudaSuccess ||
        cudaStreamSynchronize(b->stream) != cudaSuccess)
      r = DYN_ERR_CUDA;
  }
  if (r != DYN_OK) {
    cudaGetLastError();
    release(b);
    return r;
  }
  FrameGroups& G = b->groups;
  G.k = k;
  G.st[0] = b->stream;
  int64_t voff = 0;
  for (int g = 0; g < k; ++g) {
    const int n_g = start[g + 1] - start[g];
    int64_t cap_g = 0;
    for (int j = start[g]; j < start[g + 1]; ++j) cap_g += sorted[j]->tp.num_blocks;
    G.tab[g] = b->d_tab + start[g];
    G.map[g] = b->d_map + start[g];
    G.shape[g] = make_shape(sorted.data() + start[g], n_g, b->d_gvis + voff, b->d_gcount + g,
                            (int)cap_g);
    // the groups' persistent ICP launches may run at once: each takes a
    // share of the resident blocks in proportion to its pixel tiles
    set_icp_persistent(G.shape[g], sorted.data() + start[g], n_g, b->d_icp_bar + kIcpBarWords * g,
                       group_budget(sorted, start, g, icp_persistent_capacity(b->device)));
    voff += cap_g;
  }
  FrameGroups& one = b->single;
  one.k = 1;
  one.st[0] = b->stream;
  one.tab[0] = b->d_tab;
  one.map[0] = b->d_map;
  b->sorted = sorted;
  b->gstart.assign(start.begin(), start.end());
  one.shape[0] = make_shape(sorted.data(), n, b->d_gvis, b->d_gcount, (int)cap);
  set_icp_persistent(one.shape[0], sorted.data(), n, b->d_icp_bar, icp_persistent_capacity(b->device));
  b->shape = one.shape[0];
  for (int i = 0; i < n; ++i) sessions[i]->batch = b;
  *out = b;
  return DYN_OK;
}

dyn_status dyn_batch_destroy(dyn_batch* b) {
  if (!b) return DYN_ERR_INVALID_ARG;
  release(b);
  return DYN_OK;
}

static dyn_status batch_ready(dyn_batch* b) {
  for (dyn_session* s : b->ss)
    if (!s) return DYN_ERR_INVALID_ARG;  // a member was destroyed
  return DYN_OK;
}

// Autotuner candidates: launch shapes that change no result (integration
// CTAs, raycast tile), so they can be timed on live frames.
struct TuneCandidate {
  int integrate_ctas;
  int ray_tile;
  int icp;  // 0: persistent ICP on the group's full share of the resident
            // blocks, 1: on half of it, 2: the chained kernels
};
// Phase 1: the integration grid x the raycast tile (persistent ICP); phase
// 2: the ICP's shape with phase 1's best.  Every candidate gives the same
// results (the batch test steps through all of them).
constexpr TuneCandidate kTune[] = {{148 * 8, 0, 0}, {148 * 4, 0, 0}, {148 * 16, 0, 0},
                                   {148 * 8, 1, 0}, {148 * 4, 1, 0}, {148 * 16, 1, 0},
                                   {148 * 8, 2, 0}, {148 * 4, 2, 0}, {148 * 16, 2, 0}};
constexpr int kNumTune = (int)(sizeof(kTune) / sizeof(kTune[0]));
constexpr int kNumIcpShapes = 3;

static void apply_shape(dyn_batch* b, const TuneCandidate& c) {
  const int cap = icp_persistent_capacity(b->device);
  const int k = b->groups.k;
  for (int g = 0; g < k; ++g) {
    BatchShape& sh = b->groups.shape[g];
    sh.integrate_ctas = c.integrate_ctas;
    sh.ray_tile = c.ray_tile;
    const int share = group_budget(b->sorted, b->gstart, g, cap);
    const int budget = c.icp == 2 ? 0 : (c.icp == 1 ? share / 2 : share);
    set_icp_persistent(sh, b->sorted.data() + b->gstart[g], b->gstart[g + 1] - b->gstart[g],
                       sh.icp_bar, budget);
  }
  b->single.shape[0].integrate_ctas = c.integrate_ctas;
  b->single.shape[0].ray_tile = c.ray_tile;
  if (b->exec) {
    cudaGraphExecDestroy(b->exec);
    b->exec = nullptr;
  }
}

// The candidate measured in position i of the run: phase 1's shapes, then
// the ICP shapes 1 and 2 with phase 1's best.
static TuneCandidate tune_candidate(const dyn_batch* b, int i) {
  if (i < kNumTune) return kTune[i];
  TuneCandidate c = kTune[b->tune_best1];
  c.icp = 1 + (i - kNumTune);
  return c;
}

// Reads the last timed frame and moves through the candidates: each runs
// tune_frames frames, its first (graph capture and upload) not counted;
// after the last one the fastest is kept.
static dyn_status tune_step(dyn_batch* b) {
  if (b->tune_pending) {
    DYN_CUDA(cudaEventSynchronize(b->tune_ev[1]));
    float ms = 0.0f;
    DYN_CUDA(cudaEventElapsedTime(&ms, b->tune_ev[0], b->tune_ev[1]));
    b->tune_pending = false;
    if (b->tune_count > 0) b->tune_ms[b->tune_idx] += ms;
    if (++b->tune_count >= b->tune_frames) {
      b->tune_count = 0;
      ++b->tune_idx;
      if (b->tune_idx == kNumTune) {  // phase 1 done: its best, then the ICP shapes
        int best = 0;
        for (int i = 1; i < kNumTune; ++i)
          if (b->tune_ms[i] < b->tune_ms[best]) best = i;
        b->tune_best1 = best;
      }
      if (b->tune_idx == kNumTune + kNumIcpShapes - 1) {
        int best = 0;
        for (int i = 1; i < b->tune_idx; ++i)
          if (b->tune_ms[i] < b->tune_ms[best]) best = i;
        b->tune_best = best;
        const TuneCandidate c = tune_candidate(b, best);
        b->tune_icp = c.icp;
        apply_shape(b, c);
        return DYN_OK;
      }
      apply_shape(b, tune_candidate(b, b->tune_idx));
    }
  }
  return DYN_OK;
}

static dyn_status batch_launch(dyn_batch* b) {
  const bool tuning = b->tune_frames > 0 && b->tune_best < 0;
  if (tuning) DYN_TRY(tune_step(b));
  const bool timed = b->tune_frames > 0 && b->tune_best < 0;
  if (!b->exec) {
    Marks m;
    m.on = b->profile;
    m.ev = b->ev;
    m.st = b->stream;
    // a profiled frame runs as one group, so that stage boundaries are
    // those of the whole batch
    dyn_status r = capture_groups(b->profile ? b->single : b->groups, b->d_res, b->h_res, b->n,
                                  m, &b->exec, &b->kernels_per_frame);
    if (r != DYN_OK) return r;
  }
  if (timed) DYN_CUDA(cudaEventRecord(b->tune_ev[0], b->stream));
  DYN_CUDA(cudaGraphLaunch(b->exec, b->stream));
  if (timed) {
    DYN_CUDA(cudaEventRecord(b->tune_ev[1], b->stream));
    b->tune_pending = true;
  }
  b->pending = true;
  for (dyn_session* s : b->ss) s->frames++;
  return DYN_OK;
}

dyn_status dyn_batch_submit(dyn_batch* b, const uint16_t* const* depth_host,
                            const uint8_t* const* rgb_host) {
  if (!b || !depth_host) return DYN_ERR_INVALID_ARG;
  DYN_TRY(batch_ready(b));
  for (int i = 0; i < b->n; ++i)
    if (!depth_host[i]) return DYN_ERR_INVALID_ARG;
  DeviceGuard dg(b->device);
  // the staging buffers may still feed the previous frame's copies
  DYN_CUDA(cudaEventSynchronize(b->h2d_done));
  for (int i = 0; i < b->n; ++i)
    DYN_TRY(copy_frame_in(b->ss[i], depth_host[i], rgb_host ? rgb_host[i] : nullptr, b->stream));
  DYN_CUDA(cudaEventRecord(b->h2d_done, b->stream));
  return batch_launch(b);
}

dyn_status dyn_batch_submit_device(dyn_batch* b, const uint16_t* const* depth_dev,
                                   const uint8_t* const* rgb_dev) {
  if (!b || !depth_dev) return DYN_ERR_INVALID_ARG;
  DYN_TRY(batch_ready(b));
  for (int i = 0; i < b->n; ++i)
    if (!depth_dev[i]) return DYN_ERR_INVALID_ARG;
  DeviceGuard dg(b->device);
  for (int i = 0; i < b->n; ++i) {
    dyn_session* s = b->ss[i];
    const uint8_t* rgb = rgb_dev ? rgb_dev[i] : nullptr;
    DYN_CUDA(cudaMemcpyAsync(s->d_u16, depth_dev[i], s->npx * 2, cudaMemcpyDeviceToDevice,
                             b->stream));
    if (rgb)
      DYN_CUDA(cudaMemcpyAsync(s->d_rgb, rgb, s->npx * 3, cudaMemcpyDeviceToDevice, b->stream));
    DYN_TRY(set_rgb_flag(s, rgb != nullptr, b->stream));
  }
  return batch_launch(b);
}

dyn_status dyn_batch_result(dyn_batch* b, float* poses_out, dyn_frame_stats* stats_out,
                            dyn_status* status_out) {
  if (!b) return DYN_ERR_INVALID_ARG;
  if (!b->pending) return DYN_ERR_NOT_READY;
  DeviceGuard dg(b->device);
  DYN_CUDA(cudaStreamSynchronize(b->stream));
  b->pending = false;
  if (b->profile) add_stage_times(b->ev, b->stage_ms, &b->prof_frames);
  dyn_status first = DYN_OK;
  for (int i = 0; i < b->n; ++i) {
    const ResultBlock& r = b->h_res[i];
    if (poses_out)
      for (int k = 0; k < 16; ++k) poses_out[16 * i + k] = (float)r.pose.pose[k];
    if (stats_out && b->ss[i]) fill_stats(b->ss[i], r, &stats_out[i]);
    const dyn_status st = counters_status(r.cnt);
    if (status_out) status_out[i] = st;
    if (first == DYN_OK) first = st;
  }
  return first;
}

dyn_status dyn_batch_size(dyn_batch* b, int32_t* n_out) {
  if (!b || !n_out) return DYN_ERR_INVALID_ARG;
  *n_out = b->n;
  return DYN_OK;
}

dyn_status dyn_batch_stream(dyn_batch* b, void** stream_out) {
  if (!b || !stream_out) return DYN_ERR_INVALID_ARG;
  *stream_out = (void*)b->stream;
  return DYN_OK;
}

dyn_status dyn_batch_profile(dyn_batch* b, int32_t enable) {
  if (!b) return DYN_ERR_INVALID_ARG;
  DeviceGuard dg(b->device);
  DYN_CUDA(cudaStreamSynchronize(b->stream));
  bool en = enable != 0;
  if (en && !b->ev[0])
    for (int k = 0; k < DYN_NUM_STAGES; ++k) DYN_CUDA(cudaEventCreate(&b->ev[k]));
  if (en != b->profile) {
    if (b->exec) {
      cudaGraphExecDestroy(b->exec);
      b->exec = nullptr;
    }
    b->profile = en;
  }
  return DYN_OK;
}

dyn_status dyn_batch_stage_times(dyn_batch* b, double ms_out[DYN_NUM_STAGES],
                                 int64_t* frames_out, int32_t reset) {
  if (!b) return DYN_ERR_INVALID_ARG;
  if (ms_out)
    for (int k = 0; k < DYN_NUM_STAGES; ++k) ms_out[k] = b->stage_ms[k];
  if (frames_out) *frames_out = b->prof_frames;
  if (reset) {
    for (int k = 0; k < DYN_NUM_STAGES; ++k) b->stage_ms[k] = 0.0;
    b->prof_frames = 0;
  }
  return DYN_OK;
}

dyn_status dyn_batch_autotune(dyn_batch* b, int32_t frames_per_candidate) {
  if (!b || frames_per_candidate < 0 || frames_per_candidate == 1) return DYN_ERR_INVALID_ARG;
  DeviceGuard dg(b->device);
  DYN_CUDA(cudaStreamSynchronize(b->stream));
  for (int k = 0; k < 2; ++k)
    if (!b->tune_ev[k]) DYN_CUDA(cudaEventCreate(&b->tune_ev[k]));
  b->tune_frames = frames_per_candidate;
  b->tune_idx = 0;
  b->tune_count = 0;
  b->tune_best = -1;
  b->tune_pending = false;
  b->tune_ms.assign(kNumTune + kNumIcpShapes - 1, 0.0f);
  b->tune_best1 = -1;
  apply_shape(b, kTune[0]);  // the default shape, measured first
  return DYN_OK;
}

dyn_status dyn_batch_tuning(dyn_batch* b, int32_t* done, int32_t* integrate_ctas,
                            int32_t* ray_tile) {
  if (!b) return DYN_ERR_INVALID_ARG;
  const BatchShape& sh = b->groups.shape[0];
  if (done) *done = b->tune_best >= 0 ? 1 : 0;
  if (integrate_ctas) *integrate_ctas = sh.integrate_ctas > 0 ? sh.integrate_ctas : 148 * 8;
  if (ray_tile) *ray_tile = sh.ray_tile;
  return DYN_OK;
}

dyn_status dyn_batch_kernels_per_frame(dyn_batch* b, int32_t* n_out) {
  if (!b || !n_out) return DYN_ERR_INVALID_ARG;
  *n_out = b->kernels_per_frame;
  return DYN_OK;
}

}  // extern "C"

// ---------------------------------------------------------------- serving

namespace {

// The server's device budget, reserved once: sessions are carved from it
// and returned to it, so admission and release allocate and free nothing
// on the device (cudaMalloc and cudaFree would stall the steps in flight).
// First fit by address over free ranges; freed ranges merge with their
// neighbours.  All sizes are multiples of 256 bytes.
struct Arena {
  char* base = nullptr;
  size_t size = 0;
  std::map<size_t, size_t> free_;  // offset -> length
  void init(char* b, size_t n) {
    base = b;
    size = n;
    free_.clear();
    if (n) free_[0] = n;
  }
  // offset of 'n' bytes, or SIZE_MAX
  size_t take(size_t n) {
    for (auto it = free_.begin(); it != free_.end(); ++it) {
      if (it->second < n) continue;
      const size_t off = it->first, len = it->second;
      free_.erase(it);
      if (len > n) free_[off + n] = len - n;
      return off;
    }
    return SIZE_MAX;
  }
  void give(size_t off, size_t n) {
    auto it = free_.emplace(off, n).first;
    auto next = std::next(it);
    if (next != free_.end() && it->first + it->second == next->first) {
      it->second += next->second;
      free_.erase(next);
    }
    if (it != free_.begin()) {
      auto prev = std::prev(it);
      if (prev->first + prev->second == it->first) {
        prev->second += it->second;
        free_.erase(it);
      }
    }
  }
};

struct ServerSlot {
  dyn_session* s = nullptr;
  size_t bytes = 0;
  size_t offset = 0;         // of its region in the server's arena
  bool queued = false;       // a frame waits for the next step
  bool queued_rgb = false;
  const uint16_t* src_depth = nullptr;  // pinned caller buffers read at step time
  const uint8_t* src_rgb = nullptr;     // (null: the session's staging buffers)
  int64_t last_step = -1;    // id of the last step that processed the slot
  int last_ring = 0;
};

// One step's device table: descriptors and slot indices of its sessions,
// with pinned host copies (kept until the step has completed).
struct StepBuf {
  SessDev* d_tab = nullptr;
  int* d_map = nullptr;
  SessDev* h_tab = nullptr;
  int* h_map = nullptr;
  cudaEvent_t done = nullptr;
  bool used = false;
};

constexpr int kServerRing = 4;

}  // namespace

struct dyn_server {
  int device = 0;
  size_t budget = 0, used = 0;
  char* d_arena = nullptr;  // the budget, reserved at creation
  size_t sessions_off = 0;  // the sessions' part of it (after the visible list)
  Arena arena;
  int capacity = 0;
  std::vector<ServerSlot> slots;
  cudaStream_t stream = nullptr;
  StepBuf ring[kServerRing];
  int ring_pos = 0;
  int64_t steps = 0;
  int64_t steps_done = 0;  // steps known to have completed (in order)
  int64_t frames = 0;
  int2* d_gvis = nullptr;  // the start of the budget: one entry per block admissible
  int* d_gcount = nullptr;
  unsigned* d_icp_bar = nullptr;  // the persistent ICP's barrier words
  int64_t gvis_cap = 0;
  // streams and events lent to admitted sessions (created ahead of the
  // serving loop: stream creation can block for tens of milliseconds while
  // the device is busy)
  std::vector<std::pair<cudaStream_t, cudaEvent_t>> pool;
  ResultBlock* d_res = nullptr;
  ResultBlock* h_res = nullptr;  // pinned, one entry per slot
  std::vector<dyn_session*> act;
};

namespace {

void release(dyn_server* sv) {
  if (!sv) return;
  int prev = 0;
  cudaGetDevice(&prev);
  cudaSetDevice(sv->device);
  if (sv->stream) cudaStreamSynchronize(sv->stream);
  for (ServerSlot& sl : sv->slots)
    if (sl.s) {
      sl.s->owner_stream = nullptr;
      sv->pool.emplace_back(sl.s->stream, sl.s->h2d_done);
      dyn_session_destroy(sl.s);
    }
  for (StepBuf& r : sv->ring) {
    cudaFree(r.d_tab);
    cudaFree(r.d_map);
    if (r.h_tab) cudaFreeHost(r.h_tab);
    if (r.h_map) cudaFreeHost(r.h_map);
    if (r.done) cudaEventDestroy(r.done);
  }
  for (auto& pe : sv->pool) {
    cudaStreamDestroy(pe.first);
    cudaEventDestroy(pe.second);
  }
  cudaFree(sv->d_arena);
  cudaFree(sv->d_gcount);
  cudaFree(sv->d_icp_bar);
  cudaFree(sv->d_res);
  if (sv->h_res) cudaFreeHost(sv->h_res);
  if (sv->stream) cudaStreamDestroy(sv->stream);
  cudaSetDevice(prev);
  delete sv;
}

// Device bytes every admitted block costs at least (its voxels in the
// smallest form, its heap key and its entry in the session's visible list),
// which bounds the blocks of all admitted sessions by the budget.
constexpr size_t kMinBlockBytes = 4 * kBlockVox + sizeof(unsigned long long) + sizeof(int2);
// Pooled stream/event pairs made at creation (more are made on demand).
constexpr int kServerStreamPool = 64;

dyn_status pool_make(cudaStream_t* st, cudaEvent_t* ev) {
  *st = nullptr;
  *ev = nullptr;
  if (cudaStreamCreateWithFlags(st, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(ev, cudaEventDisableTiming) != cudaSuccess) {
    cudaGetLastError();
    if (*st) cudaStreamDestroy(*st);
    return DYN_ERR_CUDA;
  }
  return DYN_OK;
}
dyn_status pool_take(dyn_server* sv, cudaStream_t* st, cudaEvent_t* ev) {
  if (sv->pool.empty()) return pool_make(st, ev);
  *st = sv->pool.back().first;
  *ev = sv->pool.back().second;
  sv->pool.pop_back();
  return DYN_OK;
}

dyn_status check_slot(dyn_server* sv, int32_t slot) {
  if (!sv || slot < 0 || slot >= sv->capacity || !sv->slots[slot].s) return DYN_ERR_INVALID_ARG;
  return DYN_OK;
}

}  // namespace

extern "C" {

dyn_status dyn_server_create(const dyn_server_params* p, dyn_server** out) {
  if (!out || !p) return DYN_ERR_INVALID_ARG;
  *out = nullptr;
  const int cap = p->max_sessions > 0 ? p->max_sessions : 256;
  if (cap > 65535) return DYN_ERR_INVALID_ARG;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return DYN_ERR_NO_DEVICE;
  }
  if (p->device < 0 || p->device >= ndev) return DYN_ERR_INVALID_ARG;
  DeviceGuard dg(p->device);
  dyn_server* sv = new (std::nothrow) dyn_server();
  if (!sv) return DYN_ERR_OOM;
  sv->device = p->device;
  sv->capacity = cap;
  sv->slots.resize((size_t)cap);
  size_t free_b = 0, total_b = 0;
  if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) {
    delete sv;
    return DYN_ERR_CUDA;
  }
  sv->budget = (p->budget_bytes ? p->budget_bytes : free_b / 10 * 9) / 256 * 256;
  // the batch visible list comes first in the budget, sized for every block
  // the rest of the budget can hold, so a step never has to grow it
  sv->gvis_cap = (int64_t)(sv->budget / kMinBlockBytes) + 1;
  sv->sessions_off = ((size_t)sv->gvis_cap * sizeof(int2) + 255) / 256 * 256;
  if (sv->sessions_off >= sv->budget) {
    delete sv;
    return DYN_ERR_BUDGET_EXCEEDED;
  }
  bool ok = cudaMalloc(&sv->d_arena, sv->budget) == cudaSuccess &&
            cudaStreamCreateWithFlags(&sv->stream, cudaStreamNonBlocking) == cudaSuccess &&
            cudaMalloc(&sv->d_gcount, 256) == cudaSuccess &&
            cudaMalloc(&sv->d_icp_bar, kIcpBarWords * sizeof(unsigned)) == cudaSuccess &&
            cudaMalloc(&sv->d_res, sizeof(ResultBlock) * (size_t)cap) == cudaSuccess &&
            cudaMallocHost(&sv->h_res, sizeof(ResultBlock) * (size_t)cap) == cudaSuccess;
  for (StepBuf& r : sv->ring)
    ok = ok && cudaMalloc(&r.d_tab, sizeof(SessDev) * (size_t)cap) == cudaSuccess &&
         cudaMalloc(&r.d_map, sizeof(int) * (size_t)cap) == cudaSuccess &&
         cudaMallocHost(&r.h_tab, sizeof(SessDev) * (size_t)cap) == cudaSuccess &&
         cudaMallocHost(&r.h_map, sizeof(int) * (size_t)cap) == cudaSuccess &&
         cudaEventCreateWithFlags(&r.done, cudaEventDisableTiming) == cudaSuccess;
  if (!ok) {
    cudaGetLastError();
    release(sv);
    return DYN_ERR_OOM;
  }
  sv->d_gvis = reinterpret_cast<int2*>(sv->d_arena);
  for (int i = 0; i < std::min(cap, kServerStreamPool) && ok; ++i) {
    cudaStream_t st = nullptr;
    cudaEvent_t ev = nullptr;
    ok = pool_make(&st, &ev) == DYN_OK;
    if (ok) sv->pool.emplace_back(st, ev);
  }
  if (!ok) {
    release(sv);
    return DYN_ERR_CUDA;
  }
  std::memset(sv->h_res, 0, sizeof(ResultBlock) * (size_t)cap);
  sv->arena.init(sv->d_arena + sv->sessions_off, sv->budget - sv->sessions_off);
  *out = sv;
  return DYN_OK;
}

dyn_status dyn_server_destroy(dyn_server* sv) {
  if (!sv) return DYN_ERR_INVALID_ARG;
  release(sv);
  return DYN_OK;
}

dyn_status dyn_server_admit(dyn_server* sv, const dyn_tsdf_params* tsdf, const dyn_gn_params* gn,
                            const dyn_bilateral_params* bil, const dyn_sensor* sensor,
                            int32_t precision, const float pose0[16], int32_t* slot_out) {
  if (!sv || !slot_out || !tsdf || !gn || !sensor) return DYN_ERR_INVALID_ARG;
  *slot_out = -1;
  int slot = -1;
  for (int i = 0; i < sv->capacity && slot < 0; ++i)
    if (!sv->slots[i].s) slot = i;
  if (slot < 0) return DYN_ERR_BUDGET_EXCEEDED;
  const size_t bytes = session_device_bytes(tsdf, gn, bil, sensor, precision);
  if (bytes == 0) return DYN_ERR_INVALID_ARG;
  const size_t off = sv->arena.take(bytes);
  if (off == SIZE_MAX) return DYN_ERR_BUDGET_EXCEEDED;
  DeviceGuard dg(sv->device);
  // the session's buffers from its region; no pinned staging yet (page-
  // locked frames need none); initialisation enqueued on the session's
  // stream, which the server's stream waits for
  SessionMemory mem;
  mem.region = sv->d_arena + sv->sessions_off + off;
  mem.region_size = bytes;
  mem.host_staging = false;
  mem.sync = false;
  dyn_status r = pool_take(sv, &mem.stream, &mem.h2d_done);
  if (r != DYN_OK) {
    sv->arena.give(off, bytes);
    return r;
  }
  dyn_session* s = nullptr;
  r = create_session(tsdf, gn, bil, sensor, precision, sv->device, mem, &s);
  if (r == DYN_OK && pose0) r = set_pose_async(s, pose0);
  if (r == DYN_OK && (cudaEventRecord(s->h2d_done, s->stream) != cudaSuccess ||
                      cudaStreamWaitEvent(sv->stream, s->h2d_done, 0) != cudaSuccess))
    r = DYN_ERR_CUDA;
  if (r != DYN_OK) {
    if (s) dyn_session_destroy(s);
    sv->pool.emplace_back(mem.stream, mem.h2d_done);
    sv->arena.give(off, bytes);
    return r;
  }
  s->owner_stream = sv->stream;
  ServerSlot& sl = sv->slots[slot];
  sl = ServerSlot();
  sl.s = s;
  sl.bytes = bytes;
  sl.offset = off;
  sv->used += bytes;
  *slot_out = slot;
  return DYN_OK;
}

dyn_status dyn_server_release(dyn_server* sv, int32_t slot) {
  DYN_TRY(check_slot(sv, slot));
  DeviceGuard dg(sv->device);
  ServerSlot& sl = sv->slots[slot];
  // the last step that used the session must have completed (older ring
  // entries were waited for when they were reused)
  if (sl.last_step >= 0 && sl.last_step >= sv->steps - kServerRing)
    DYN_CUDA(cudaEventSynchronize(sv->ring[sl.last_ring].done));
  sl.s->owner_stream = nullptr;
  const std::pair<cudaStream_t, cudaEvent_t> lent(sl.s->stream, sl.s->h2d_done);
  dyn_session_destroy(sl.s);  // its device buffers are the region: nothing freed
  sv->pool.push_back(lent);   // (the destroy synchronised the stream)
  sv->arena.give(sl.offset, sl.bytes);
  sv->used -= sl.bytes;
  sl = ServerSlot();
  return DYN_OK;
}

dyn_status dyn_server_push(dyn_server* sv, int32_t slot, const uint16_t* depth_host,
                           const uint8_t* rgb_host) {
  DYN_TRY(check_slot(sv, slot));
  if (!depth_host) return DYN_ERR_INVALID_ARG;
  ServerSlot& sl = sv->slots[slot];
  if (sl.queued) return DYN_ERR_NOT_READY;  // the previous frame has not been stepped
  dyn_session* s = sl.s;
  DeviceGuard dg(sv->device);
  sl.src_depth = nullptr;
  sl.src_rgb = nullptr;
  if (is_pinned(depth_host) && (!rgb_host || is_pinned(rgb_host))) {
    // page-locked: copied to the device by the step itself
    sl.src_depth = depth_host;
    sl.src_rgb = rgb_host;
  } else {
    DYN_TRY(ensure_staging(s));  // pinned staging on the first pageable frame
    // the staging buffers may still feed the copies of the slot's last step
    DYN_CUDA(cudaEventSynchronize(s->h2d_done));
    std::memcpy(s->h_depth, depth_host, s->npx * sizeof(uint16_t));
    if (rgb_host) std::memcpy(s->h_rgb, rgb_host, s->npx * 3);
  }
  sl.queued = true;
  sl.queued_rgb = rgb_host != nullptr;
  return DYN_OK;
}

dyn_status dyn_server_step(dyn_server* sv, int32_t* n_out) {
  if (!sv) return DYN_ERR_INVALID_ARG;
  if (n_out) *n_out = 0;
  DeviceGuard dg(sv->device);
  StepBuf& rb = sv->ring[sv->ring_pos];
  if (rb.used) DYN_CUDA(cudaEventSynchronize(rb.done));  // its table may still be read
  sv->act.clear();
  int64_t cap = 0;
  for (int i = 0; i < sv->capacity; ++i) {
    ServerSlot& sl = sv->slots[i];
    if (!sl.s || !sl.queued) continue;
    rb.h_tab[sv->act.size()] = sl.s->hsd;
    rb.h_map[sv->act.size()] = i;
    sv->act.push_back(sl.s);
    cap += sl.s->tp.num_blocks;
  }
  const int n = (int)sv->act.size();
  if (n == 0) return DYN_OK;
  // the admitted sessions' blocks fit the list by construction (each block
  // costs at least kMinBlockBytes of the budget)
  if (cap > sv->gvis_cap) return DYN_ERR_BUDGET_EXCEEDED;
  cudaStream_t st = sv->stream;
  DYN_CUDA(cudaMemcpyAsync(rb.d_tab, rb.h_tab, sizeof(SessDev) * (size_t)n,
                           cudaMemcpyHostToDevice, st));
  DYN_CUDA(cudaMemcpyAsync(rb.d_map, rb.h_map, sizeof(int) * (size_t)n, cudaMemcpyHostToDevice,
                           st));
  for (int i = 0; i < n; ++i) {
    dyn_session* s = sv->act[i];
    ServerSlot& sl = sv->slots[rb.h_map[i]];
    DYN_CUDA(cudaMemcpyAsync(s->d_u16, sl.src_depth ? sl.src_depth : s->h_depth, s->npx * 2,
                             cudaMemcpyHostToDevice, st));
    if (sl.queued_rgb)
      DYN_CUDA(cudaMemcpyAsync(s->d_rgb, sl.src_rgb ? sl.src_rgb : s->h_rgb, s->npx * 3,
                               cudaMemcpyHostToDevice, st));
    DYN_TRY(set_rgb_flag(s, sl.queued_rgb, st));
    DYN_CUDA(cudaEventRecord(s->h2d_done, st));
  }
  BatchShape b = make_shape(sv->act.data(), n, sv->d_gvis, sv->d_gcount, (int)cap);
  set_icp_persistent(b, sv->act.data(), n, sv->d_icp_bar, icp_persistent_capacity(sv->device));
  enqueue_frame(rb.d_tab, b, rb.d_map, sv->d_res, sv->h_res, sv->capacity, st, Marks());
  DYN_CUDA(cudaGetLastError());
  DYN_CUDA(cudaEventRecord(rb.done, st));
  rb.used = true;
  for (int i = 0; i < n; ++i) {
    ServerSlot& sl = sv->slots[rb.h_map[i]];
    sl.queued = false;
    sl.last_step = sv->steps;
    sl.last_ring = sv->ring_pos;
    sl.s->frames++;
  }
  sv->ring_pos = (sv->ring_pos + 1) % kServerRing;
  sv->steps++;
  sv->frames += n;
  if (n_out) *n_out = n;
  return DYN_OK;
}

dyn_status dyn_server_poll(dyn_server* sv, int32_t slot, int32_t* ready_out) {
  DYN_TRY(check_slot(sv, slot));
  if (!ready_out) return DYN_ERR_INVALID_ARG;
  const ServerSlot& sl = sv->slots[slot];
  *ready_out = 0;
  if (sl.last_step < 0) return DYN_OK;
  DeviceGuard dg(sv->device);
  cudaError_t e = cudaEventQuery(sv->ring[sl.last_ring].done);
  if (e == cudaSuccess) *ready_out = 1;
  else if (e != cudaErrorNotReady) return DYN_ERR_CUDA;
  else cudaGetLastError();
  return DYN_OK;
}

dyn_status dyn_server_result(dyn_server* sv, int32_t slot, float pose_out[16],
                             dyn_frame_stats* stats) {
  DYN_TRY(check_slot(sv, slot));
  const ServerSlot& sl = sv->slots[slot];
  if (sl.last_step < 0) return DYN_ERR_NOT_READY;
  DeviceGuard dg(sv->device);
  // a later step reusing the ring entry completes after this slot's step
  DYN_CUDA(cudaEventSynchronize(sv->ring[sl.last_ring].done));
  const ResultBlock& r = sv->h_res[slot];
  if (pose_out)
    for (int k = 0; k < 16; ++k) pose_out[k] = (float)r.pose.pose[k];
  if (stats) fill_stats(sl.s, r, stats);
  return counters_status(r.cnt);
}

dyn_status dyn_server_sync(dyn_server* sv) {
  if (!sv) return DYN_ERR_INVALID_ARG;
  DeviceGuard dg(sv->device);
  DYN_CUDA(cudaStreamSynchronize(sv->stream));
  return DYN_OK;
}

dyn_status dyn_server_session(dyn_server* sv, int32_t slot, dyn_session** out) {
  DYN_TRY(check_slot(sv, slot));
  if (!out) return DYN_ERR_INVALID_ARG;
  *out = sv->slots[slot].s;
  return DYN_OK;
}

dyn_status dyn_server_info(dyn_server* sv, dyn_server_usage* out) {
  if (!sv || !out) return DYN_ERR_INVALID_ARG;
  std::memset(out, 0, sizeof(*out));
  out->budget_bytes = sv->budget;
  out->used_bytes = sv->used;
  out->capacity = sv->capacity;
  for (const ServerSlot& sl : sv->slots)
    if (sl.s) out->sessions++;
  out->steps = sv->steps;
  out->frames = sv->frames;
  DeviceGuard dg(sv->device);
  // steps complete in order; those a ring length back are known complete
  int64_t id = std::max(sv->steps_done, sv->steps - (int64_t)kServerRing);
  for (; id < sv->steps; ++id) {
    const cudaError_t e = cudaEventQuery(sv->ring[id % kServerRing].done);
    if (e == cudaErrorNotReady) {
      cudaGetLastError();
      break;
    }
    if (e != cudaSuccess) return DYN_ERR_CUDA;
  }
  sv->steps_done = id;
  out->steps_done = id;
  return DYN_OK;
}

}  // extern "C"

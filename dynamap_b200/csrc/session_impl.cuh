// session_impl.cuh -- internal definitions shared by session.cu (sessions,
// the per-frame pipeline, stage entry points) and serving.cu (batches and
// the serving loop).  Not part of the public interface.
#pragma once
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "common.cuh"
#include "icp.cuh"
#include "image.cuh"
#include "sessdev.cuh"
#include "tsdf.cuh"

namespace dyn {
namespace host {

struct ResultBlock {
  PoseState pose;
  IcpState icp;
  Counters cnt;
};
static_assert(sizeof(PoseState) % 4 == 0 && sizeof(IcpState) % 4 == 0 &&
                  sizeof(Counters) % 4 == 0,
              "result parts are copied as 32-bit words");

inline int level_of_scale(int scale) {
  int l = 0;
  while ((1 << l) < scale && l < kLevels - 1) ++l;
  return l;
}

inline DSensor dsensor(const dyn_sensor& s) {
  DSensor d;
  d.rows = (int)s.rows;
  d.cols = (int)s.cols;
  d.fx = s.fx;
  d.fy = s.fy;
  d.cx = s.cx;
  d.cy = s.cy;
  return d;
}

// Level sensor for scale 2^l: f/s, (c+0.5)/s-0.5, dims floor(dim/s).
inline dyn_sensor level_sensor(const dyn_sensor& s, int scale) {
  dyn_sensor o = s;
  o.rows = s.rows / (uint32_t)scale;
  o.cols = s.cols / (uint32_t)scale;
  o.fx = s.fx / (float)scale;
  o.fy = s.fy / (float)scale;
  o.cx = (s.cx + 0.5f) / (float)scale - 0.5f;
  o.cy = (s.cy + 0.5f) / (float)scale - 0.5f;
  return o;
}

inline DTsdf dtsdf(const dyn_tsdf_params& p, int precision) {
  DTsdf t;
  t.vs = p.voxel_size;
  t.bsm = (float)p.block_size * p.voxel_size;  // tsdf.cu:437-438
  t.trunc = p.truncation_distance;
  t.dmin = p.min_sensor_depth;
  t.dmax = p.max_sensor_depth;
  t.num_buckets = p.num_buckets;
  t.nb_mask = (p.num_buckets & (p.num_buckets - 1)) == 0 ? p.num_buckets - 1 : -1;
  t.bucket_size = p.bucket_size;
  t.num_blocks = p.num_blocks;
  t.max_w = p.max_sdf_weight;
  double bs = (double)p.block_size * (double)p.voxel_size;
  t.dda_cap = 3 * (int)std::ceil(((double)p.max_sensor_depth + (double)p.truncation_distance) / bs) + 8;
  double step = std::min((double)p.voxel_size, (double)p.truncation_distance);
  t.rc_cap = (int)std::ceil((double)p.max_sensor_depth / step) + 4;
  t.band = precision == DYN_PRECISION_MIXED_BAND ? 1 : 0;
  return t;
}

#define DYN_CUDA(x)                                  \
  do {                                               \
    cudaError_t e_ = (x);                            \
    if (e_ != cudaSuccess) {                         \
      if (e_ == cudaErrorMemoryAllocation) return DYN_ERR_OOM; \
      return DYN_ERR_CUDA;                           \
    }                                                \
  } while (0)

#define DYN_TRY(x)                 \
  do {                             \
    dyn_status r_ = (x);           \
    if (r_ != DYN_OK) return r_;   \
  } while (0)

inline bool valid_sensor(const dyn_sensor* s) {
  return s && s->rows > 0 && s->cols > 0 && s->rows <= 8192 && s->cols <= 8192 &&
         s->fx > 0 && s->fy > 0 && s->depth_scaler > 0;
}

}  // namespace host
}  // namespace dyn

// The opaque handle types of the C ABI (global names), built from dyn:: parts.
using namespace dyn;
using dyn::host::ResultBlock;

struct dyn_session {
  int device = 0;
  dyn_tsdf_params tp;
  dyn_gn_params gp;
  dyn_bilateral_params bp;
  dyn_sensor sensor;
  int precision = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t h2d_done = nullptr;
  DSensor ls[kLevels];
  int nlev = 1;
  size_t npx = 0;
  // device buffers
  std::vector<void*> allocs;
  uint16_t* d_u16 = nullptr;
  uint8_t* d_rgb = nullptr;
  float* d_raw = nullptr;
  float* d_sdist = nullptr;
  float* d_filt = nullptr;
  float* d_sdep[kLevels] = {};
  float4* d_snrm[kLevels] = {};
  float4* d_svtx[kLevels] = {};
  float* d_sint[kLevels] = {};
  float* d_tdep[kLevels] = {};
  float4* d_tnrm[kLevels] = {};
  float4* d_tvtx[kLevels] = {};
  float* d_tint[kLevels] = {};
  float* d_ray = nullptr;
  uint8_t* d_trgb = nullptr;
  float* d_pose_override = nullptr;
  double* d_pose_in = nullptr;
  double* d_partials = nullptr;
  unsigned* d_icp_bar = nullptr;  // the persistent ICP's barrier words
  IcpState* d_icp = nullptr;
  PoseState* d_pose = nullptr;
  VolumeDev vol;
  // fused-launch descriptor (host copy and its device table of one)
  SessDev hsd;
  SessDev* d_sd = nullptr;
  BilateralTable* d_btab = nullptr;
  int* d_rgb_flag = nullptr;   // nonzero: the current frame carries RGB
  int rgb_flag_host = -1;      // last value written (-1: unknown)
  unsigned* d_rbound = nullptr;  // ray depth bounds per 8x8 pixel tile (near, then far)
  unsigned* d_ftile = nullptr;   // free-space tile map (depth-only frames)
  int rb_tx = 0, rb_ty = 0;
  int2* d_gvis = nullptr;      // visible list of the table of one
  int* d_gcount = nullptr;
  ResultBlock* d_res = nullptr;
  BatchShape shape;
  dyn_batch* batch = nullptr;  // member of this batch (frames go through it)
  cudaStream_t owner_stream = nullptr;  // a server's stream when it owns the session
  bool borrowed_stream = false;  // 'stream' and 'h2d_done' belong to the server's pool
  // host
  uint16_t* h_depth = nullptr;
  uint8_t* h_rgb = nullptr;
  ResultBlock* h_res = nullptr;
  cudaGraphExec_t exec = nullptr;
  BilateralTable btab;
  // profiling: ev[i] ends stage i (DYN_STAGE_*), ev[DYN_STAGE_FRAME] starts the frame
  bool profile = false;
  cudaEvent_t ev[DYN_NUM_STAGES] = {};
  double stage_ms[DYN_NUM_STAGES] = {};
  int64_t prof_frames = 0;
  int kernels_per_frame = 0;
  bool debug_maps = false;
  int frames = 0;
  bool pending = false;  // a frame submitted whose result has not been read
  // Two frames in flight (dyn_frame_submit before the previous frame's
  // dyn_frame_result): input slot 0 is d_u16 / d_rgb / d_rgb_flag with
  // h_depth / h_rgb, h_res, exec and d_sd above; slot 1 has its own.  A
  // frame's host->device copy runs on copy_stream and overlaps the previous
  // frame's graph on 'stream'; ev_h2d[k] marks slot k's copy done (the
  // graph waits for it, the next copy into slot k's staging waits for it),
  // ev_done[k] slot k's graph done (the next copy into slot k's device
  // buffers waits for it).  Results are read in submission order.
  cudaStream_t copy_stream = nullptr;
  cudaEvent_t ev_h2d[2] = {};
  cudaEvent_t ev_done[2] = {};
  uint16_t* d_u16_1 = nullptr;
  uint8_t* d_rgb_1 = nullptr;
  int* d_rgb_flag_1 = nullptr;
  int rgb_flag_host_1 = -1;
  SessDev* d_sd_1 = nullptr;
  SessDev hsd_1;
  uint16_t* h_depth_1 = nullptr;
  uint8_t* h_rgb_1 = nullptr;
  ResultBlock* h_res_1 = nullptr;
  cudaGraphExec_t exec_1 = nullptr;
  ResultBlock* h_res_aux = nullptr;  // results of the calls outside the frame graphs
  int inflight[2] = {0, 0};          // slots of the frames in flight, oldest first
  int n_inflight = 0;
  int next_slot = 0;

  // device memory: cudaMalloc per buffer, or carved from a region a server
  // reserved (region != null), or only counted (measure)
  char* region = nullptr;
  size_t region_size = 0, region_used = 0;
  bool measure = false;
  size_t measured = 0;

  template <class T>
  dyn_status dalloc(T** p, size_t bytes) {
    void* q = nullptr;
    bytes = (bytes + 255) / 256 * 256;  // whole 16-byte vectors at the tail
    if (bytes < 256) bytes = 256;
    if (measure) {
      measured += bytes;
      *p = nullptr;
      return DYN_OK;
    }
    if (region) {
      if (region_used + bytes > region_size) return DYN_ERR_OOM;
      *p = (T*)(region + region_used);
      region_used += bytes;
      return DYN_OK;
    }
    cudaError_t e = cudaMalloc(&q, bytes);
    if (e != cudaSuccess) {
      cudaGetLastError();
      return e == cudaErrorMemoryAllocation ? DYN_ERR_OOM : DYN_ERR_CUDA;
    }
    allocs.push_back(q);
    *p = (T*)q;
    return DYN_OK;
  }
  bool use_color() const { return gp.color_weight != 0.0f; }
  IcpParams icp_params() const {
    IcpParams P;
    P.dmin = gp.icp_min_depth;
    P.dmax = gp.icp_max_depth;
    P.cos_thr = gp.normal_cos_thresh;
    P.cw = gp.color_weight;
    P.min_inc = gp.min_increment;
    P.max_inc = gp.max_increment;
    P.reg = gp.regularization;
    P.compose_left = gp.compose_left;
    P.kahan = precision != DYN_PRECISION_FP32 ? 1 : 0;
    return P;
  }
};

// A fixed set of sessions on one device whose frames run together: each
// stage is one launch over the members' descriptor table and the whole frame
// one CUDA graph on the batch's stream.
// A table of sessions split into groups, each group's fused stage chain on
// its own stream (group 0 on the caller's stream): groups overlap the
// tails of each other's launches.
constexpr int kMaxGroups = 8;
struct FrameGroups {
  int k = 1;
  const SessDev* tab[kMaxGroups] = {};  // group sub-tables (device)
  const int* map[kMaxGroups] = {};      // group-local index -> result index (device)
  BatchShape shape[kMaxGroups];
  cudaStream_t st[kMaxGroups] = {};     // st[0]: the caller's stream
  cudaEvent_t fork = nullptr;
  cudaEvent_t join[kMaxGroups] = {};
};

struct dyn_batch {
  int device = 0;
  int n = 0;
  std::vector<dyn_session*> ss;
  cudaStream_t stream = nullptr;
  FrameGroups groups;     // members in size order, split into groups
  FrameGroups single;     // all members as one group (profiled frames)
  int* d_map = nullptr;   // table position -> member index
  cudaEvent_t h2d_done = nullptr;
  std::vector<void*> allocs;
  SessDev* d_tab = nullptr;
  int2* d_gvis = nullptr;
  int* d_gcount = nullptr;
  unsigned* d_icp_bar = nullptr;  // kIcpBarWords per group (persistent ICP barrier)
  ResultBlock* d_res = nullptr;
  ResultBlock* h_res = nullptr;  // pinned, n entries
  BatchShape shape;
  cudaGraphExec_t exec = nullptr;
  int kernels_per_frame = 0;
  bool profile = false;
  cudaEvent_t ev[DYN_NUM_STAGES] = {};
  double stage_ms[DYN_NUM_STAGES] = {};
  int64_t prof_frames = 0;
  // autotuner: result-invariant launch shapes timed on the batch's own
  // frames (tune_frames per candidate; tune_idx the candidate measured)
  int tune_frames = 0;
  int tune_idx = -1;
  int tune_count = 0;
  int tune_best = -1;
  bool tune_pending = false;
  cudaEvent_t tune_ev[2] = {nullptr, nullptr};
  std::vector<float> tune_ms;
  int tune_best1 = -1;          // phase 1's best candidate
  int tune_icp = 0;             // the ICP shape kept (0 persistent, 1 half budget, 2 chained)
  // members in table order and the first member of each group (for the
  // ICP's launch shape)
  std::vector<dyn_session*> sorted;
  std::vector<int> gstart;
  bool pending = false;
};

namespace dyn {
namespace host {

struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int dev) {
    cudaGetDevice(&prev);
    if (prev != dev) cudaSetDevice(dev);
  }
  ~DeviceGuard() {
    int cur = -1;
    cudaGetDevice(&cur);
    if (prev >= 0 && cur != prev) cudaSetDevice(prev);
  }
};

// Stage boundary events (profiling only; captured into the frame graph):
// ev[i] ends stage i, ev[DYN_STAGE_FRAME] starts the frame.
struct Marks {
  bool on = false;
  cudaEvent_t* ev = nullptr;
  cudaStream_t st = nullptr;
  void operator()(int stage) const {
    // External: during capture this becomes an event-record node of the graph
    if (on) cudaEventRecordWithFlags(ev[stage], st, cudaEventRecordExternal);
  }
};

void release(dyn_session* s);
void release(dyn_batch* b);
// Session calls that read device state wait for the batch or server that
// runs its frames.
dyn_status quiesce(dyn_session* s);
// The launch shape of a table of sessions (the largest member bounds every
// grid).
BatchShape make_shape(dyn_session* const* ss, int n, int2* gvis, int* gcount, int gvis_cap);
// The persistent ICP of a table: its grid within 'budget' blocks (0 when it
// does not fit: the chained kernels, same results) and its barrier words.
void set_icp_persistent(BatchShape& b, dyn_session* const* ss, int n, unsigned* bar, int budget);
// Marks whether this frame of 's' carries RGB (stream-ordered).
dyn_status set_rgb_flag(dyn_session* s, bool has_rgb, cudaStream_t st);
// Host frame into the session's device input buffers on 'st'.
dyn_status copy_frame_in(dyn_session* s, const uint16_t* depth, const uint8_t* rgb,
                         cudaStream_t st);
// One frame of every session of 'tab' on 'st', then every session's results
// into res_dev[slot_map ? slot_map[i] : i] and n_results entries of res_dev
// back into res_host (pinned).
void enqueue_frame(const SessDev* tab, const BatchShape& b, const int* slot_map,
                   ResultBlock* res_dev, ResultBlock* res_host, int n_results, cudaStream_t st,
                   const Marks& m);
// The same captured into an executable graph.
dyn_status capture_frame(const SessDev* tab, const BatchShape& b, ResultBlock* res_dev,
                         ResultBlock* res_host, cudaStream_t st, const Marks& m,
                         cudaGraphExec_t* exec_out, int* kernels_out);
// One frame of every group (fork from and join back into G.st[0]), then
// n_results entries of res_dev back into res_host; marks on group 0 only.
void enqueue_groups(const FrameGroups& G, ResultBlock* res_dev, ResultBlock* res_host,
                    int n_results, const Marks& m);
dyn_status capture_groups(const FrameGroups& G, ResultBlock* res_dev, ResultBlock* res_host,
                          int n_results, const Marks& m, cudaGraphExec_t* exec_out,
                          int* kernels_out);
void add_stage_times(cudaEvent_t* ev, double* ms_acc, int64_t* frames);
// Page-locked host memory (read by the copy engines without staging).
bool is_pinned(const void* p);
// Device bytes a session with these parameters allocates (colour: a mixed
// session keeps per-voxel colour).
size_t session_bytes(const dyn_tsdf_params& t, const dyn_sensor& s, int precision, bool colour);

// Where a session's memory comes from (dyn_session_create: cudaMalloc per
// buffer, pinned staging now, initialisation waited for).
struct SessionMemory {
  char* region = nullptr;    // carve the device buffers from [region, region + size)
  size_t region_size = 0;
  bool host_staging = true;  // pinned staging and result buffers now (else on first use)
  bool sync = true;          // return after the initialisation has run
  // a stream and event the session uses instead of creating its own (a
  // server's pool); such a session has no copy stream and no second input
  // slot events (frames reach it only through its server)
  cudaStream_t stream = nullptr;
  cudaEvent_t h2d_done = nullptr;
};
// Exact device bytes of a session with these parameters (no CUDA calls);
// 0 when the parameters are invalid.
size_t session_device_bytes(const dyn_tsdf_params* tsdf, const dyn_gn_params* gn,
                            const dyn_bilateral_params* bil, const dyn_sensor* sensor,
                            int precision);
dyn_status create_session(const dyn_tsdf_params* tsdf, const dyn_gn_params* gn,
                          const dyn_bilateral_params* bil, const dyn_sensor* sensor,
                          int precision, int device, const SessionMemory& mem,
                          dyn_session** out);
// The pose from the host without waiting (stream-ordered on the session).
dyn_status set_pose_async(dyn_session* s, const float pose[16]);
// Pinned staging buffers of a session created without them.
dyn_status ensure_staging(dyn_session* s);
bool mixed_colour(const dyn_gn_params* gn);
dyn_status counters_status(const Counters& c);
void fill_stats(const dyn_session* s, const ResultBlock& r, dyn_frame_stats* st);

}  // namespace host
}  // namespace dyn

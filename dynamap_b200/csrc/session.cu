// session.cu -- the C ABI of include/dynamap.h: sessions (the reference's
// builder, include/builder/builder.cu), the per-frame pipeline and the stage
// entry points.
//
// One session = one RGB-D stream.  All of its device memory (hash entries,
// voxel blocks, image pyramids, solver state) is allocated once in
// dyn_session_create and sized from its parameters; frames allocate nothing.
// The per-frame kernel sequence is captured once into a CUDA graph and
// replayed per frame on the session's own stream; tracking state, pose and
// counters stay on the device, so a frame needs no host synchronisation
// between stages (the reference synchronises after every launch and solves
// each GN iteration on the host).
//
// Every stage is a fused launch over a device table of session descriptors
// (SessDev): a session alone runs a table of one, a dyn_batch runs the
// table of its members, one launch per stage for all of them and the whole
// frame as one graph.
#include <cstdio>
#include <cstdlib>
#include <mutex>
#include <new>

#include "session_impl.cuh"

using namespace dyn;
using namespace dyn::host;

namespace dyn {
namespace host {

void release(dyn_batch* b) {
  if (!b) return;
  int prev = 0;
  cudaGetDevice(&prev);
  cudaSetDevice(b->device);
  if (b->stream) cudaStreamSynchronize(b->stream);
  for (dyn_session* s : b->ss)
    if (s && s->batch == b) s->batch = nullptr;
  if (b->exec) cudaGraphExecDestroy(b->exec);
  for (int g = 1; g < kMaxGroups; ++g) {
    if (b->groups.st[g]) cudaStreamDestroy(b->groups.st[g]);
    if (b->groups.join[g]) cudaEventDestroy(b->groups.join[g]);
  }
  if (b->groups.fork) cudaEventDestroy(b->groups.fork);
  for (cudaEvent_t e : b->tune_ev)
    if (e) cudaEventDestroy(e);
  for (void* p : b->allocs) cudaFree(p);
  if (b->h_res) cudaFreeHost(b->h_res);
  if (b->h2d_done) cudaEventDestroy(b->h2d_done);
  for (int k = 0; k < DYN_NUM_STAGES; ++k)
    if (b->ev[k]) cudaEventDestroy(b->ev[k]);
  if (b->stream) cudaStreamDestroy(b->stream);
  cudaSetDevice(prev);
  delete b;
}

void release(dyn_session* s) {
  if (!s) return;
  int prev = 0;
  cudaGetDevice(&prev);
  cudaSetDevice(s->device);
  if (s->batch) {  // a destroyed member leaves its batch unusable
    cudaStreamSynchronize(s->batch->stream);
    for (auto& m : s->batch->ss)
      if (m == s) m = nullptr;
  }
  if (s->copy_stream) cudaStreamSynchronize(s->copy_stream);
  if (s->stream) cudaStreamSynchronize(s->stream);
  if (s->exec) cudaGraphExecDestroy(s->exec);
  if (s->exec_1) cudaGraphExecDestroy(s->exec_1);
  for (void* p : s->allocs) cudaFree(p);
  for (void* p : {(void*)s->h_depth, (void*)s->h_rgb, (void*)s->h_res, (void*)s->h_depth_1,
                  (void*)s->h_rgb_1, (void*)s->h_res_1, (void*)s->h_res_aux})
    if (p) cudaFreeHost(p);
  if (s->h2d_done && !s->borrowed_stream) cudaEventDestroy(s->h2d_done);
  for (int k = 0; k < 2; ++k) {
    if (s->ev_h2d[k]) cudaEventDestroy(s->ev_h2d[k]);
    if (s->ev_done[k]) cudaEventDestroy(s->ev_done[k]);
  }
  if (s->copy_stream) cudaStreamDestroy(s->copy_stream);
  for (int k = 0; k < DYN_NUM_STAGES; ++k)
    if (s->ev[k]) cudaEventDestroy(s->ev[k]);
  if (s->stream && !s->borrowed_stream) cudaStreamDestroy(s->stream);
  cudaSetDevice(prev);
  delete s;
}

MapsArgs maps_args(dyn_session* s, bool target) {
  MapsArgs a;
  int off = 0;
  for (int l = 0; l < s->nlev; ++l) {
    a.lv[l].depth = target ? s->d_tdep[l] : s->d_sdep[l];
    a.lv[l].normal = target ? s->d_tnrm[l] : s->d_snrm[l];
    a.lv[l].vertex = s->debug_maps ? (target ? s->d_tvtx[l] : s->d_svtx[l]) : nullptr;
    a.lv[l].s = s->ls[l];
    a.lv[l].offset = off;
    off += s->ls[l].rows * s->ls[l].cols;
  }
  a.nlev = s->nlev;
  a.total = off;
  return a;
}

__global__ void mark_target_kernel(IcpState* st) {
  if (threadIdx.x == 0 && blockIdx.x == 0) st->have_target = 1;
}
__global__ void bump_frame_kernel(PoseState* ps) {
  if (threadIdx.x == 0 && blockIdx.x == 0) ps->frame += 1;
}

__device__ inline void copy_words(void* dst, const void* src, int bytes) {
  for (int k = threadIdx.x; k < bytes / 4; k += blockDim.x)
    static_cast<unsigned*>(dst)[k] = static_cast<const unsigned*>(src)[k];
}
// pose, solver state and counters of every session into one array, read
// back by one copy (entry slot_map[i] when a map is given)
__global__ void gather_results_kernel(const SessDev* __restrict__ tab, int n,
                                      const int* __restrict__ slot_map,
                                      ResultBlock* __restrict__ out) {
  const int i = blockIdx.x;
  if (i >= n) return;
  const SessDev& S = tab[i];
  ResultBlock& o = out[slot_map ? slot_map[i] : i];
  copy_words(&o.pose, S.pose, (int)sizeof(PoseState));
  copy_words(&o.icp, S.icp, (int)sizeof(IcpState));
  copy_words(&o.cnt, S.vol.cnt, (int)sizeof(Counters));
}

// Source side of a frame: ingest, bilateral filter, pyramid, normal maps.
void enqueue_source(const SessDev* tab, const BatchShape& b, cudaStream_t st, const Marks& m) {
  m(DYN_STAGE_FRAME);
  fused_reset_counters(tab, b, st);
  fused_ingest(tab, b, st);
  m(DYN_STAGE_INGEST);
  fused_bilateral(tab, b, st);
  m(DYN_STAGE_BILATERAL);
  fused_pyramid(tab, b, 0, st);
  m(DYN_STAGE_SOURCE_MAPS);
}

// gnSolver::solve's level loop (gnSolver.cu:340-431): iterations 1 .. N-1
// of each level slot; every launch after the first overlaps its
// predecessor's tail (programmatic dependent launch).
void enqueue_icp(const SessDev* tab, const BatchShape& b, cudaStream_t st) {
  if (b.icp_grid > 0) {  // one persistent launch for every level and iteration
    fused_icp_persistent(tab, b, st);
    return;
  }
  bool chained = false;
  for (int pl = 0; pl < 3; ++pl)
    for (int it = 1; it < b.max_slot_iters[pl]; ++it) {
      fused_icp_iteration(tab, b, pl, it, chained, st);
      chained = true;
    }
}

// Integration at the session pose, then the next frame's target.
void enqueue_map_update(const SessDev* tab, const BatchShape& b, cudaStream_t st,
                        const Marks& m) {
  fused_allocate(tab, b, st);
  m(DYN_STAGE_ALLOCATE);
  fused_visible(tab, b, st);
  m(DYN_STAGE_VISIBLE);
  fused_integrate(tab, b, st);
  fused_free_cells(tab, b, st);
  m(DYN_STAGE_INTEGRATE);
  fused_raycast(tab, b, st);
  m(DYN_STAGE_RAYCAST);
  fused_target_prepare(tab, b, st);
  fused_pyramid(tab, b, 1, st);
  m(DYN_STAGE_TARGET_MAPS);
}

// builder::buildModelLS with the intended order: track frame k against the
// target of frame k-1, integrate frame k at the new pose, raycast the target
// for frame k+1; then the results into 'res_host' (pinned).
void enqueue_frame(const SessDev* tab, const BatchShape& b, const int* slot_map,
                   ResultBlock* res_dev, ResultBlock* res_host, int n_results, cudaStream_t st,
                   const Marks& m) {
  enqueue_source(tab, b, st, m);
  enqueue_icp(tab, b, st);
  fused_pose_finalize(tab, b, 1, st);
  m(DYN_STAGE_ICP);
  enqueue_map_update(tab, b, st, m);
  gather_results_kernel<<<b.n, 128, 0, st>>>(tab, b.n, slot_map, res_dev);
  if (res_host)
    cudaMemcpyAsync(res_host, res_dev, sizeof(ResultBlock) * (size_t)n_results,
                    cudaMemcpyDeviceToHost, st);
}

void enqueue_groups(const FrameGroups& G, ResultBlock* res_dev, ResultBlock* res_host,
                    int n_results, const Marks& m) {
  cudaStream_t main = G.st[0];
  if (G.k > 1) {
    cudaEventRecord(G.fork, main);
    for (int g = 1; g < G.k; ++g) cudaStreamWaitEvent(G.st[g], G.fork, 0);
  }
  for (int g = 0; g < G.k; ++g)
    enqueue_frame(G.tab[g], G.shape[g], G.map[g], res_dev, nullptr, 0, G.st[g],
                  g == 0 ? m : Marks());
  for (int g = 1; g < G.k; ++g) {
    cudaEventRecord(G.join[g], G.st[g]);
    cudaStreamWaitEvent(main, G.join[g], 0);
  }
  cudaMemcpyAsync(res_host, res_dev, sizeof(ResultBlock) * (size_t)n_results,
                  cudaMemcpyDeviceToHost, main);
}

// Kernel nodes of a captured graph, then its executable form.
static dyn_status instantiate(cudaGraph_t g, cudaGraphExec_t* exec_out, int* kernels_out) {
  size_t nn = 0;
  cudaGraphGetNodes(g, nullptr, &nn);
  std::vector<cudaGraphNode_t> nodes(nn);
  if (nn) cudaGraphGetNodes(g, nodes.data(), &nn);
  int nk = 0;
  for (size_t i = 0; i < nn; ++i) {
    cudaGraphNodeType ty;
    if (cudaGraphNodeGetType(nodes[i], &ty) == cudaSuccess && ty == cudaGraphNodeTypeKernel) ++nk;
  }
  *kernels_out = nk;
  cudaGraphExec_t ex = nullptr;
  const cudaError_t e = cudaGraphInstantiate(&ex, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) return DYN_ERR_CUDA;
  *exec_out = ex;
  return DYN_OK;
}

dyn_status capture_groups(const FrameGroups& G, ResultBlock* res_dev, ResultBlock* res_host,
                          int n_results, const Marks& m, cudaGraphExec_t* exec_out,
                          int* kernels_out) {
  cudaGraph_t g = nullptr;
  DYN_CUDA(cudaStreamBeginCapture(G.st[0], cudaStreamCaptureModeThreadLocal));
  enqueue_groups(G, res_dev, res_host, n_results, m);
  if (cudaStreamEndCapture(G.st[0], &g) != cudaSuccess) return DYN_ERR_CUDA;
  return instantiate(g, exec_out, kernels_out);
}

// Captures one frame of 'tab' on 'st' into an executable graph.
dyn_status capture_frame(const SessDev* tab, const BatchShape& b, ResultBlock* res_dev,
                         ResultBlock* res_host, cudaStream_t st, const Marks& m,
                         cudaGraphExec_t* exec_out, int* kernels_out) {
  cudaGraph_t g = nullptr;
  DYN_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
  enqueue_frame(tab, b, nullptr, res_dev, res_host, b.n, st, m);
  if (cudaStreamEndCapture(st, &g) != cudaSuccess) return DYN_ERR_CUDA;
  return instantiate(g, exec_out, kernels_out);
}

// The launch shape of a table of sessions: the largest image, level and
// heap of its members bound every grid.
BatchShape make_shape(dyn_session* const* ss, int n, int2* gvis, int* gcount, int gvis_cap) {
  BatchShape b;
  std::memset(&b, 0, sizeof(b));
  b.n = n;
  b.gvis = gvis;
  b.gcount = gcount;
  b.gvis_cap = gvis_cap;
  for (int i = 0; i < n; ++i) {
    const dyn_session* s = ss[i];
    b.max_rows = std::max(b.max_rows, s->ls[0].rows);
    b.max_cols = std::max(b.max_cols, s->ls[0].cols);
    b.max_npx = std::max(b.max_npx, (int)s->npx);
    b.max_nlev = std::max(b.max_nlev, s->nlev);
    b.max_blocks = std::max(b.max_blocks, s->tp.num_blocks);
    for (int l = 0; l < s->nlev; ++l)
      b.max_level_px[l] = std::max(b.max_level_px[l], s->ls[l].rows * s->ls[l].cols);
    for (int pl = 0; pl < 3; ++pl) {
      const int l = level_of_scale(s->gp.lvl_scale[pl]);
      b.max_slot_px[pl] = std::max(b.max_slot_px[pl], s->ls[l].rows * s->ls[l].cols);
      b.max_slot_iters[pl] = std::max(b.max_slot_iters[pl], s->gp.lvl_iteration_num[pl]);
    }
    if (s->bp.enabled) b.max_bil_radius = std::max(b.max_bil_radius, s->btab.radius);
    b.max_rb_tiles = std::max(b.max_rb_tiles, std::max(1, s->rb_tx * s->rb_ty));
    b.kahan_mask |= s->icp_params().kahan ? 2 : 1;
    b.fp16_mask |= s->vol.fp16 ? 2 : 1;
  }
  return b;
}

// The persistent ICP for a table of sessions: its grid within 'budget'
// blocks (0: chained kernels) and its barrier words.  DYN_ICP_CHAINED=1 in
// the environment keeps every table on the chained kernels (the same
// results; for comparisons).
void set_icp_persistent(BatchShape& b, dyn_session* const* ss, int n, unsigned* bar, int budget) {
  static const bool chained_only = [] {
    const char* e = std::getenv("DYN_ICP_CHAINED");
    return e && e[0] == '1';
  }();
  std::vector<int> npx((size_t)n), kahan((size_t)n);
  for (int i = 0; i < n; ++i) {
    npx[i] = (int)ss[i]->npx;
    kahan[i] = ss[i]->icp_params().kahan;
  }
  b.icp_budget = budget;
  b.icp_grid_k[0] = b.icp_grid_k[1] = 0;
  b.icp_grid = (chained_only || !bar)
                   ? 0
                   : icp_persistent_grid(npx.data(), kahan.data(), n, budget, b.icp_grid_k);
  b.icp_bar = bar;
}

// The session's descriptor (device buffers, sensor levels, parameters).
void fill_sessdev(dyn_session* s) {
  SessDev& d = s->hsd;
  std::memset(&d, 0, sizeof(d));
  for (int l = 0; l < kLevels; ++l) d.ls[l] = s->ls[l];
  d.nlev = s->nlev;
  d.npx = (int)s->npx;
  d.depth_scaler = s->sensor.depth_scaler;
  d.rgb_flag = s->d_rgb_flag;
  d.use_color = s->use_color() ? 1 : 0;
  d.bil_enabled = s->bp.enabled ? 1 : 0;
  d.mode = s->gp.mode;
  d.debug_maps = 0;
  d.u16 = s->d_u16;
  d.rgb = s->d_rgb;
  d.raw = s->d_raw;
  d.sdist = s->d_sdist;
  d.filt = s->d_filt;
  for (int l = 0; l < s->nlev; ++l) {
    d.sdep[l] = s->d_sdep[l];
    d.snrm[l] = s->d_snrm[l];
    d.svtx[l] = s->d_svtx[l];
    d.sint[l] = s->d_sint[l];
    d.tdep[l] = s->d_tdep[l];
    d.tnrm[l] = s->d_tnrm[l];
    d.tvtx[l] = s->d_tvtx[l];
    d.tint[l] = s->d_tint[l];
  }
  d.ray = s->d_ray;
  d.trgb = s->d_trgb;
  d.rbound = s->d_rbound;
  d.ftile = s->d_ftile;
  d.rb_tx = s->rb_tx;
  d.rb_ty = s->rb_ty;
  d.btab = s->d_btab;
  d.icp = s->d_icp;
  d.pose = s->d_pose;
  d.partials = s->d_partials;
  d.icpp = s->icp_params();
  for (int pl = 0; pl < 3; ++pl) {
    d.slot_level[pl] = level_of_scale(s->gp.lvl_scale[pl]);
    d.slot_iters[pl] = s->gp.lvl_iteration_num[pl];
  }
  d.vol = s->vol;
}

// Marks whether this frame of 's' carries RGB (stream-ordered; written only
// when it changes).  The memset writes 0x01 into every byte: any nonzero
// value means "RGB present".
dyn_status set_rgb_flag(dyn_session* s, bool has_rgb, cudaStream_t st) {
  const int v = has_rgb ? 1 : 0;
  if (s->rgb_flag_host != v) {
    DYN_CUDA(cudaMemsetAsync(s->d_rgb_flag, v, sizeof(int), st));
    s->rgb_flag_host = v;
  }
  return DYN_OK;
}

// Session calls that read device state wait for the batch it belongs to.
dyn_status quiesce(dyn_session* s) {
  if (s->batch) DYN_CUDA(cudaStreamSynchronize(s->batch->stream));
  if (s->owner_stream) DYN_CUDA(cudaStreamSynchronize(s->owner_stream));
  return DYN_OK;
}

bool is_pinned(const void* p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeHost;
}

// Host frame into the session's device input buffers on 'st' (pinned
// sources directly, others through the session's pinned staging buffers).
dyn_status copy_frame_in(dyn_session* s, const uint16_t* depth, const uint8_t* rgb,
                         cudaStream_t st) {
  size_t nd = s->npx * sizeof(uint16_t), nc = s->npx * 3;
  if (is_pinned(depth)) {
    DYN_CUDA(cudaMemcpyAsync(s->d_u16, depth, nd, cudaMemcpyHostToDevice, st));
  } else {
    std::memcpy(s->h_depth, depth, nd);
    DYN_CUDA(cudaMemcpyAsync(s->d_u16, s->h_depth, nd, cudaMemcpyHostToDevice, st));
  }
  if (rgb) {
    if (is_pinned(rgb)) {
      DYN_CUDA(cudaMemcpyAsync(s->d_rgb, rgb, nc, cudaMemcpyHostToDevice, st));
    } else {
      std::memcpy(s->h_rgb, rgb, nc);
      DYN_CUDA(cudaMemcpyAsync(s->d_rgb, s->h_rgb, nc, cudaMemcpyHostToDevice, st));
    }
  }
  return set_rgb_flag(s, rgb != nullptr, st);
}

dyn_status upload_frame(dyn_session* s, const uint16_t* depth, const uint8_t* rgb) {
  // no pipelined copy may still read slot 0's staging buffers
  if (s->copy_stream) DYN_CUDA(cudaStreamSynchronize(s->copy_stream));
  // the staging buffers may still feed the previous frame's copies
  DYN_CUDA(cudaEventSynchronize(s->h2d_done));
  dyn_status r = copy_frame_in(s, depth, rgb, s->stream);
  if (r != DYN_OK) return r;
  DYN_CUDA(cudaEventRecord(s->h2d_done, s->stream));
  return DYN_OK;
}

Marks session_marks(dyn_session* s) {
  Marks m;
  m.on = s->profile;
  m.ev = s->ev;
  m.st = s->stream;
  return m;
}

// ---- frames through the session's graphs, up to two in flight
struct SlotIO {
  uint16_t* d_u16;
  uint8_t* d_rgb;
  int* d_flag;
  int* flag_host;
  uint16_t** h_depth;
  uint8_t** h_rgb;
  ResultBlock* h_res;
  cudaGraphExec_t* exec;
  SessDev* d_sd;
};
SlotIO slot_io(dyn_session* s, int k) {
  if (k == 0)
    return {s->d_u16, s->d_rgb, s->d_rgb_flag, &s->rgb_flag_host, &s->h_depth, &s->h_rgb,
            s->h_res, &s->exec, s->d_sd};
  return {s->d_u16_1, s->d_rgb_1, s->d_rgb_flag_1, &s->rgb_flag_host_1, &s->h_depth_1,
          &s->h_rgb_1, s->h_res_1, &s->exec_1, s->d_sd_1};
}

// The frame's inputs into slot k on the copy stream: host pointers (pinned
// ones read directly, others through the slot's pinned staging) or device
// pointers.
dyn_status stage_slot(dyn_session* s, int k, const uint16_t* depth, const uint8_t* rgb,
                      bool device_src) {
  SlotIO io = slot_io(s, k);
  cudaStream_t cs = s->copy_stream;
  const size_t nd = s->npx * sizeof(uint16_t), nc = s->npx * 3;
  // the slot's staging may still feed its last copy; its device inputs may
  // still be read by the frame two back
  DYN_CUDA(cudaEventSynchronize(s->ev_h2d[k]));
  DYN_CUDA(cudaStreamWaitEvent(cs, s->ev_done[k], 0));
  auto put = [&](void* dst, const void* src, size_t n, void** stage) -> dyn_status {
    if (device_src) {
      DYN_CUDA(cudaMemcpyAsync(dst, src, n, cudaMemcpyDeviceToDevice, cs));
    } else if (is_pinned(src)) {
      DYN_CUDA(cudaMemcpyAsync(dst, src, n, cudaMemcpyHostToDevice, cs));
    } else {
      if (!*stage) {
        if (cudaMallocHost(stage, n) != cudaSuccess) {
          cudaGetLastError();
          return DYN_ERR_OOM;
        }
      }
      std::memcpy(*stage, src, n);
      DYN_CUDA(cudaMemcpyAsync(dst, *stage, n, cudaMemcpyHostToDevice, cs));
    }
    return DYN_OK;
  };
  DYN_TRY(put(io.d_u16, depth, nd, reinterpret_cast<void**>(io.h_depth)));
  if (rgb) DYN_TRY(put(io.d_rgb, rgb, nc, reinterpret_cast<void**>(io.h_rgb)));
  const int v = rgb ? 1 : 0;
  if (*io.flag_host != v) {
    DYN_CUDA(cudaMemsetAsync(io.d_flag, v, sizeof(int), cs));
    *io.flag_host = v;
  }
  DYN_CUDA(cudaEventRecord(s->ev_h2d[k], cs));
  return DYN_OK;
}

// Slot k's frame graph on the session stream once its inputs are in.
dyn_status launch_slot(dyn_session* s, int k) {
  SlotIO io = slot_io(s, k);
  if (!*io.exec) {
    dyn_status r = capture_frame(io.d_sd, s->shape, s->d_res, io.h_res, s->stream,
                                 session_marks(s), io.exec, &s->kernels_per_frame);
    if (r != DYN_OK) return r;
  }
  DYN_CUDA(cudaStreamWaitEvent(s->stream, s->ev_h2d[k], 0));
  DYN_CUDA(cudaGraphLaunch(*io.exec, s->stream));
  DYN_CUDA(cudaEventRecord(s->ev_done[k], s->stream));
  return DYN_OK;
}

// One frame: optional pose hint (stream-ordered after the frames in
// flight), inputs into the next slot, the graph.  With two frames in
// flight the older one's result is given up (its slot is reused).
dyn_status submit_frame(dyn_session* s, const uint16_t* depth, const uint8_t* rgb,
                        bool device_src, const float* hint) {
  if (s->n_inflight == 2) {
    s->inflight[0] = s->inflight[1];
    s->n_inflight = 1;
  }
  if (hint) {
    double H[16];
    for (int k = 0; k < 16; ++k) H[k] = (double)hint[k];
    // pageable source: staged before the call returns
    DYN_CUDA(cudaMemcpyAsync(s->d_pose_in, H, sizeof(H), cudaMemcpyHostToDevice, s->stream));
    launch_pose_hint(s->d_pose, s->d_icp, s->d_pose_in, s->gp.compose_left, s->stream);
    DYN_CUDA(cudaGetLastError());
  }
  const int k = s->next_slot;
  DYN_TRY(stage_slot(s, k, depth, rgb, device_src));
  DYN_TRY(launch_slot(s, k));
  s->inflight[s->n_inflight++] = k;
  s->next_slot = k ^ 1;
  s->pending = true;
  s->frames++;
  return DYN_OK;
}

// Stage times of one profiled frame added to 'ms'.
void add_stage_times(cudaEvent_t* ev, double* ms_acc, int64_t* frames) {
  float ms = 0.0f;
  int prev = DYN_STAGE_FRAME;
  for (int k = 0; k <= DYN_STAGE_TARGET_MAPS; ++k) {
    if (cudaEventElapsedTime(&ms, ev[prev], ev[k]) == cudaSuccess) ms_acc[k] += ms;
    prev = k;
  }
  if (cudaEventElapsedTime(&ms, ev[DYN_STAGE_FRAME], ev[DYN_STAGE_TARGET_MAPS]) == cudaSuccess)
    ms_acc[DYN_STAGE_FRAME] += ms;
  cudaGetLastError();
  ++*frames;
}

dyn_status counters_status(const Counters& c) {
  if (c.icp_timeout) return DYN_ERR_TIMEOUT;
  if (c.heap_exhausted) return DYN_ERR_HEAP_EXHAUSTED;
  if (c.bucket_full) return DYN_ERR_HASH_FULL;
  return DYN_OK;
}

void fill_stats(const dyn_session* s, const ResultBlock& r, dyn_frame_stats* st) {
  std::memset(st, 0, sizeof(*st));
  st->frame_index = r.pose.frame - 1;
  for (int k = 0; k < 3; ++k) {
    st->icp_iterations[k] = r.icp.iters[k];
    st->icp_inliers[k] = r.icp.inliers[k];
    st->icp_rms[k] = r.icp.rms[k];
  }
  st->icp_reset = r.pose.reset;
  st->blocks_total = std::min(r.cnt.nalloc, s->tp.num_blocks);
  st->blocks_new = r.cnt.new_blocks;
  st->blocks_visible = r.cnt.visible;
  st->unique_blocks_probed = r.cnt.unique_probed;
  st->bucket_full = r.cnt.bucket_full;
  st->heap_exhausted = r.cnt.heap_exhausted;
  st->dda_overruns = r.cnt.dda_overruns;
  st->raycast_overruns = r.cnt.raycast_overruns;
  for (int k = 0; k < 6; ++k) st->pose_increment[k] = r.pose.last_inc[k];
}

dyn_status reset_state(dyn_session* s, bool sync = true) {
  cudaStream_t st = s->stream;
  launch_volume_clear(s->vol, st);
  IcpState z;
  std::memset(&z, 0, sizeof(z));
  for (int k = 0; k < 16; ++k) z.T[k] = (k % 5 == 0) ? 1.0f : 0.0f;
  DYN_CUDA(cudaMemcpyAsync(s->d_icp, &z, sizeof(z), cudaMemcpyHostToDevice, st));
  PoseState p;
  std::memset(&p, 0, sizeof(p));
  DYN_CUDA(cudaMemcpyAsync(s->d_pose, &p, sizeof(p), cudaMemcpyHostToDevice, st));
  double I[16];
  for (int k = 0; k < 16; ++k) I[k] = (k % 5 == 0) ? 1.0 : 0.0;
  DYN_CUDA(cudaMemcpyAsync(s->d_pose_in, I, sizeof(I), cudaMemcpyHostToDevice, st));
  launch_pose_set(s->d_pose, s->d_pose_in, st);
  if (sync) DYN_CUDA(cudaStreamSynchronize(st));
  s->frames = 0;
  s->pending = false;
  s->n_inflight = 0;
  return DYN_OK;
}

// Mixed-precision sessions keep per-voxel colour only when the photometric
// term needs the model's colour.
bool mixed_colour(const dyn_gn_params* gn) { return gn && gn->color_weight != 0.0f; }

size_t session_bytes(const dyn_tsdf_params& t, const dyn_sensor& s, int precision, bool colour) {
  size_t n = (size_t)s.rows * s.cols;
  size_t b = 0;
  b += sizeof(Entry) * (size_t)t.num_buckets * t.bucket_size;
  b += sizeof(unsigned long long) * (size_t)t.num_blocks;
  if (precision != DYN_PRECISION_FP32)
    b += (4 + (colour ? 4 : 0)) * (size_t)t.num_blocks * kBlockVox;
  else
    b += sizeof(dyn_voxel) * (size_t)t.num_blocks * kBlockVox;
  b += sizeof(int2) * (size_t)t.num_blocks;  // visible list
  if (precision == DYN_PRECISION_MIXED)
    b += (sizeof(int) + 1) * (size_t)t.num_blocks;  // free-space summaries
  b += n * (2 + 3 + 4 + 4 + 4 + 3);  // inputs, raw, filtered, ray depth, target rgb
  {  // ray depth bounds and the free-space tile map
    const int tx = ((int)s.cols + 7) / 8, ty = ((int)s.rows + 7) / 8;
    b += 4 * (size_t)(ray_bounds_words(tx, ty) + free_tile_words(tx, ty)) + 512;
  }
  b += 2 * n * (4 + 16 + 16 + 4) * 4 / 3;  // source + target pyramids
  b += icp_frame_scratch_bytes(n) + sizeof(SessDev) + sizeof(BilateralTable) + sizeof(ResultBlock) +
       8192;
  return b;
}

// Per-device scratch of the stage entry points (allocated on first use).
struct StageScratch {
  double* partials = nullptr;
  unsigned int* ticket = nullptr;
  double* out = nullptr;
  float* T = nullptr;
};
std::mutex g_stage_mu;
StageScratch g_stage[64];

dyn_status validate_params(const dyn_tsdf_params* tsdf, const dyn_gn_params* gn,
                           const dyn_bilateral_params* bil, const dyn_sensor* sensor,
                           int precision) {
  if (!tsdf || !gn || !bil || !valid_sensor(sensor)) return DYN_ERR_INVALID_ARG;
  if (tsdf->block_size != kBlockSize || tsdf->bucket_size < 1 || tsdf->num_buckets < 1 ||
      tsdf->num_blocks < 1 || tsdf->max_sdf_weight < 1 ||
      tsdf->max_sdf_weight > (precision != DYN_PRECISION_FP32 ? 65535 : 255) ||
      !(tsdf->voxel_size > 0) || !(tsdf->truncation_distance > 0) ||
      !(tsdf->max_sensor_depth > 0))
    return DYN_ERR_INVALID_ARG;
  if ((int64_t)tsdf->num_buckets * tsdf->bucket_size > (int64_t)1 << 30) return DYN_ERR_INVALID_ARG;
  for (int k = 0; k < 3; ++k) {
    int sc = gn->lvl_scale[k];
    if (sc != 1 && sc != 2 && sc != 4 && sc != 8) return DYN_ERR_INVALID_ARG;
    if (gn->lvl_iteration_num[k] < 0 || gn->lvl_iteration_num[k] > 1000) return DYN_ERR_INVALID_ARG;
    if ((int)(sensor->rows / sc) < 3 || (int)(sensor->cols / sc) < 5) return DYN_ERR_INVALID_ARG;
  }
  if (bil->enabled && (bil->diameter < 1 || bil->diameter > 16 || !(bil->sigma_s > 0) ||
                       !(bil->sigma_i > 0)))
    return DYN_ERR_INVALID_ARG;
  if (gn->mode != 0 && gn->mode != 1) return DYN_ERR_INVALID_ARG;
  if (precision != DYN_PRECISION_FP32 && precision != DYN_PRECISION_MIXED &&
      precision != DYN_PRECISION_MIXED_BAND)
    return DYN_ERR_INVALID_ARG;
  return DYN_OK;
}

// Parameters and derived sizes of a session (no CUDA calls).
void init_fields(dyn_session* s, const dyn_tsdf_params* tsdf, const dyn_gn_params* gn,
                 const dyn_bilateral_params* bil, const dyn_sensor* sensor, int precision,
                 int device) {
  s->device = device;
  s->tp = *tsdf;
  s->gp = *gn;
  s->bp = *bil;
  s->sensor = *sensor;
  s->precision = precision;
  s->npx = (size_t)sensor->rows * sensor->cols;
  int maxl = 0;
  for (int k = 0; k < 3; ++k) maxl = std::max(maxl, level_of_scale(gn->lvl_scale[k]));
  s->nlev = maxl + 1;
  for (int l = 0; l < kLevels; ++l) s->ls[l] = dsensor(level_sensor(*sensor, 1 << l));
  std::memset(&s->btab, 0, sizeof(s->btab));
  if (bil->enabled) s->btab = make_bilateral_table(bil->diameter, bil->sigma_i, bil->sigma_s);
}

// Every device buffer of a session (counted only when s->measure).
dyn_status alloc_device_buffers(dyn_session* s) {
  const dyn_tsdf_params* tsdf = &s->tp;
  const int precision = s->precision;
  const size_t n = s->npx;
  DYN_TRY(s->dalloc(&s->d_u16, n * 2));
  DYN_TRY(s->dalloc(&s->d_rgb, n * 3));
  DYN_TRY(s->dalloc(&s->d_raw, n * 4));
  DYN_TRY(s->dalloc(&s->d_sdist, n * 4));
  DYN_TRY(s->dalloc(&s->d_filt, n * 4));
  DYN_TRY(s->dalloc(&s->d_ray, n * 4));
  DYN_TRY(s->dalloc(&s->d_trgb, n * 3));
  for (int l = 0; l < s->nlev; ++l) {
    size_t m = (size_t)s->ls[l].rows * s->ls[l].cols;
    size_t m4 = (m + 3) / 4 * 4;
    if (l == 0) s->d_sdep[0] = s->d_filt;
    else DYN_TRY(s->dalloc(&s->d_sdep[l], m4 * 4));
    DYN_TRY(s->dalloc(&s->d_snrm[l], m * 16));
    DYN_TRY(s->dalloc(&s->d_svtx[l], m * 16));
    DYN_TRY(s->dalloc(&s->d_sint[l], m4 * 4));
    DYN_TRY(s->dalloc(&s->d_tdep[l], m4 * 4));
    DYN_TRY(s->dalloc(&s->d_tnrm[l], m * 16));
    DYN_TRY(s->dalloc(&s->d_tvtx[l], m * 16));
    DYN_TRY(s->dalloc(&s->d_tint[l], m4 * 4));
  }
  DYN_TRY(s->dalloc(&s->d_pose_override, 64));
  DYN_TRY(s->dalloc(&s->d_pose_in, 128));
  DYN_TRY(s->dalloc(&s->d_partials, icp_frame_scratch_bytes(s->npx)));
  DYN_TRY(s->dalloc(&s->d_icp_bar, kIcpBarWords * sizeof(unsigned)));
  DYN_TRY(s->dalloc(&s->d_icp, sizeof(IcpState)));
  DYN_TRY(s->dalloc(&s->d_pose, sizeof(PoseState)));
  s->vol.t = dtsdf(*tsdf, precision);
  s->vol.sat_lo = (float)((double)tsdf->truncation_distance * (1.0 - 1e-6));
  s->vol.free_ok = (double)s->vol.sat_lo >= (double)tsdf->voxel_size ? 1 : 0;
  DYN_TRY(s->dalloc(&s->vol.entries, sizeof(Entry) * (size_t)tsdf->num_buckets * tsdf->bucket_size));
  DYN_TRY(s->dalloc(&s->vol.block_keys, sizeof(unsigned long long) * (size_t)tsdf->num_blocks));
  const size_t nvox = (size_t)tsdf->num_blocks * kBlockVox;
  s->vol.voxels = nullptr;
  s->vol.vox16 = nullptr;
  s->vol.colors = nullptr;
  s->vol.fp16 = precision != DYN_PRECISION_FP32 ? 1 : 0;
  if (s->vol.fp16) {
    DYN_TRY(s->dalloc(&s->vol.vox16, sizeof(unsigned) * nvox));
    if (mixed_colour(&s->gp)) DYN_TRY(s->dalloc(&s->vol.colors, sizeof(uchar4) * nvox));
  } else {
    DYN_TRY(s->dalloc(&s->vol.voxels, sizeof(dyn_voxel) * nvox));
  }
  s->vol.nonsat = nullptr;
  s->vol.freecell = nullptr;
  if (s->vol.fp16 && !s->vol.t.band) {  // the mixed form's raycast steps through free cells
    DYN_TRY(s->dalloc(&s->vol.nonsat, sizeof(int) * (size_t)tsdf->num_blocks));
    DYN_TRY(s->dalloc(&s->vol.freecell, (size_t)tsdf->num_blocks));
  }
  DYN_TRY(s->dalloc(&s->vol.cnt, sizeof(Counters)));
  DYN_TRY(s->dalloc(&s->d_gvis, sizeof(int2) * (size_t)tsdf->num_blocks));
  s->rb_tx = ((int)s->sensor.cols + 7) / 8;
  s->rb_ty = ((int)s->sensor.rows + 7) / 8;
  DYN_TRY(s->dalloc(&s->d_rbound, sizeof(unsigned) * (size_t)ray_bounds_words(s->rb_tx, s->rb_ty)));
  DYN_TRY(s->dalloc(&s->d_ftile, sizeof(unsigned) * (size_t)free_tile_words(s->rb_tx, s->rb_ty)));
  DYN_TRY(s->dalloc(&s->d_gcount, sizeof(int)));
  DYN_TRY(s->dalloc(&s->d_rgb_flag, sizeof(int)));
  DYN_TRY(s->dalloc(&s->d_res, sizeof(ResultBlock)));
  DYN_TRY(s->dalloc(&s->d_btab, sizeof(BilateralTable)));
  DYN_TRY(s->dalloc(&s->d_sd, sizeof(SessDev)));
  // the second input slot of pipelined frames
  DYN_TRY(s->dalloc(&s->d_u16_1, s->npx * 2));
  DYN_TRY(s->dalloc(&s->d_rgb_1, s->npx * 3));
  DYN_TRY(s->dalloc(&s->d_rgb_flag_1, sizeof(int)));
  DYN_TRY(s->dalloc(&s->d_sd_1, sizeof(SessDev)));
  return DYN_OK;
}

size_t session_device_bytes(const dyn_tsdf_params* tsdf, const dyn_gn_params* gn,
                            const dyn_bilateral_params* bil, const dyn_sensor* sensor,
                            int precision) {
  if (validate_params(tsdf, gn, bil, sensor, precision) != DYN_OK) return 0;
  dyn_session* s = new (std::nothrow) dyn_session();
  if (!s) return 0;
  init_fields(s, tsdf, gn, bil, sensor, precision, 0);
  s->measure = true;
  alloc_device_buffers(s);
  const size_t b = s->measured;
  delete s;
  return b;
}

dyn_status ensure_staging(dyn_session* s) {
  if (s->h_depth) return DYN_OK;
  if (cudaMallocHost(&s->h_depth, s->npx * 2) != cudaSuccess ||
      cudaMallocHost(&s->h_rgb, s->npx * 3) != cudaSuccess) {
    cudaGetLastError();
    return DYN_ERR_OOM;
  }
  return DYN_OK;
}

dyn_status set_pose_async(dyn_session* s, const float pose[16]) {
  double P[16];
  for (int k = 0; k < 16; ++k) P[k] = (double)pose[k];
  // pageable source: the copy is staged before the call returns
  DYN_CUDA(cudaMemcpyAsync(s->d_pose_in, P, sizeof(P), cudaMemcpyHostToDevice, s->stream));
  launch_pose_set(s->d_pose, s->d_pose_in, s->stream);
  return DYN_OK;
}

dyn_status create_session(const dyn_tsdf_params* tsdf, const dyn_gn_params* gn,
                          const dyn_bilateral_params* bil, const dyn_sensor* sensor,
                          int precision, int device, const SessionMemory& mem,
                          dyn_session** out) {
  if (!out) return DYN_ERR_INVALID_ARG;
  *out = nullptr;
  DYN_TRY(validate_params(tsdf, gn, bil, sensor, precision));
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return DYN_ERR_NO_DEVICE;
  }
  if (device < 0 || device >= ndev) return DYN_ERR_INVALID_ARG;
  DeviceGuard dg(device);
  dyn_session* s = new (std::nothrow) dyn_session();
  if (!s) return DYN_ERR_OOM;
  init_fields(s, tsdf, gn, bil, sensor, precision, device);
  s->region = mem.region;
  s->region_size = mem.region_size;
  dyn_status r = DYN_OK;
#define TRY(x)               \
  do {                       \
    r = (x);                 \
    if (r != DYN_OK) {       \
      release(s);            \
      return r;              \
    }                        \
  } while (0)
  bool ok = true;
  if (mem.stream) {
    // a server's pooled stream and event: creating streams while the
    // device is busy can block the caller for tens of milliseconds
    s->stream = mem.stream;
    s->h2d_done = mem.h2d_done;
    s->borrowed_stream = true;
  } else {
    ok = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking) == cudaSuccess &&
         cudaStreamCreateWithFlags(&s->copy_stream, cudaStreamNonBlocking) == cudaSuccess &&
         cudaEventCreateWithFlags(&s->h2d_done, cudaEventDisableTiming) == cudaSuccess;
    for (int k = 0; k < 2 && ok; ++k)
      ok = cudaEventCreateWithFlags(&s->ev_h2d[k], cudaEventDisableTiming) == cudaSuccess &&
           cudaEventCreateWithFlags(&s->ev_done[k], cudaEventDisableTiming) == cudaSuccess;
  }
  if (!ok) {
    cudaGetLastError();
    release(s);
    return DYN_ERR_CUDA;
  }
  TRY(alloc_device_buffers(s));
  if (mem.host_staging) {
    TRY(ensure_staging(s));
    if (cudaMallocHost(&s->h_res, sizeof(ResultBlock)) != cudaSuccess ||
        cudaMallocHost(&s->h_res_1, sizeof(ResultBlock)) != cudaSuccess ||
        cudaMallocHost(&s->h_res_aux, sizeof(ResultBlock)) != cudaSuccess) {
      cudaGetLastError();
      release(s);
      return DYN_ERR_OOM;
    }
  }
  // zero the images so unused levels and borders read as invalid
  for (int l = 0; l < s->nlev; ++l) {
    size_t m = (size_t)s->ls[l].rows * s->ls[l].cols;
    cudaMemsetAsync(s->d_tdep[l], 0, m * 4, s->stream);
    cudaMemsetAsync(s->d_tnrm[l], 0, m * 16, s->stream);
    cudaMemsetAsync(s->d_tint[l], 0, m * 4, s->stream);
    cudaMemsetAsync(s->d_sint[l], 0, m * 4, s->stream);
  }
  cudaMemsetAsync(s->d_rgb_flag, 0, sizeof(int), s->stream);
  cudaMemsetAsync(s->d_rgb_flag_1, 0, sizeof(int), s->stream);
  s->rgb_flag_host = 0;
  s->rgb_flag_host_1 = 0;
  fill_sessdev(s);
  s->hsd_1 = s->hsd;  // slot 1: its own inputs, everything else shared
  s->hsd_1.u16 = s->d_u16_1;
  s->hsd_1.rgb = s->d_rgb_1;
  s->hsd_1.rgb_flag = s->d_rgb_flag_1;
  dyn_session* self = s;
  s->shape = make_shape(&self, 1, s->d_gvis, s->d_gcount, tsdf->num_blocks);
  set_icp_persistent(s->shape, &self, 1, s->d_icp_bar, icp_persistent_capacity(device));
  if (cudaMemcpyAsync(s->d_btab, &s->btab, sizeof(BilateralTable), cudaMemcpyHostToDevice,
                      s->stream) != cudaSuccess ||
      cudaMemcpyAsync(s->d_sd, &s->hsd, sizeof(SessDev), cudaMemcpyHostToDevice, s->stream) !=
          cudaSuccess ||
      cudaMemcpyAsync(s->d_sd_1, &s->hsd_1, sizeof(SessDev), cudaMemcpyHostToDevice,
                      s->stream) != cudaSuccess) {
    release(s);
    return DYN_ERR_CUDA;
  }
  TRY(reset_state(s, mem.sync));
  cudaEventRecord(s->h2d_done, s->stream);  // also: initialisation enqueued
#undef TRY
  *out = s;
  return DYN_OK;
}

}  // namespace host
}  // namespace dyn

extern "C" {

int32_t dyn_abi_version(void) { return DYN_ABI_VERSION; }

const char* dyn_status_string(dyn_status s) {
  switch (s) {
    case DYN_OK: return "ok";
    case DYN_ERR_INVALID_ARG: return "invalid argument";
    case DYN_ERR_OOM: return "out of device memory";
    case DYN_ERR_BUDGET_EXCEEDED: return "memory budget exceeded";
    case DYN_ERR_HASH_FULL: return "hash bucket full";
    case DYN_ERR_HEAP_EXHAUSTED: return "voxel block heap exhausted";
    case DYN_ERR_ICP_DIVERGED: return "icp diverged";
    case DYN_ERR_TIMEOUT: return "timeout";
    case DYN_ERR_CUDA: return "cuda error";
    case DYN_ERR_NOT_READY: return "not ready";
    case DYN_ERR_NO_DEVICE: return "no cuda device";
  }
  return "unknown";
}

dyn_status dyn_session_bytes(const dyn_tsdf_params* tsdf, const dyn_sensor* sensor,
                             int32_t precision, size_t* bytes_out) {
  if (!tsdf || !valid_sensor(sensor) || !bytes_out) return DYN_ERR_INVALID_ARG;
  // colour storage of a mixed session depends on its photometric weight,
  // which is not passed here: count it (upper bound)
  *bytes_out = session_bytes(*tsdf, *sensor, precision, true);
  return DYN_OK;
}

dyn_status dyn_session_create(const dyn_tsdf_params* tsdf, const dyn_gn_params* gn,
                              const dyn_bilateral_params* bil, const dyn_sensor* sensor,
                              int32_t precision, int32_t device, dyn_session** out) {
  return create_session(tsdf, gn, bil, sensor, precision, device, SessionMemory(), out);
}

dyn_status dyn_session_destroy(dyn_session* s) {
  if (!s) return DYN_ERR_INVALID_ARG;
  release(s);
  return DYN_OK;
}

dyn_status dyn_session_reset(dyn_session* s) {
  if (!s) return DYN_ERR_INVALID_ARG;
  DeviceGuard dg(s->device);
  DYN_TRY(quiesce(s));
  DYN_CUDA(cudaStreamSynchronize(s->stream));
  return reset_state(s);
}

dyn_status dyn_session_get_pose(dyn_session* s, float pose_out[16]) {
  if (!s || !pose_out) return DYN_ERR_INVALID_ARG;
  DeviceGuard dg(s->device);
  DYN_TRY(quiesce(s));
  PoseState p;
  DYN_CUDA(cudaMemcpyAsync(&p, s->d_pose, sizeof(p), cudaMemcpyDeviceToHost, s->stream));
  DYN_CUDA(cudaStreamSynchronize(s->stream));
  for (int k = 0; k < 16; ++k) pose_out[k] = (float)p.pose[k];
  return DYN_OK;
}

dyn_status dyn_session_set_pose(dyn_session* s, const float pose[16]) {
  if (!s || !pose) return DYN_ERR_INVALID_ARG;
  DeviceGuard dg(s->device);
  DYN_TRY(quiesce(s));
  double P[16];
  for (int k = 0; k < 16; ++k) P[k] = (double)pose[k];
  DYN_CUDA(cudaMemcpyAsync(s->d_pose_in, P, sizeof(P), cudaMemcpyHostToDevice, s->stream));
  launch_pose_set(s->d_pose, s->d_pose_in, s->stream);
  DYN_CUDA(cudaStreamSynchronize(s->stream));
  return DYN_OK;
}

dyn_status dyn_frame_submit(dyn_session* s, const uint16_t* depth_host, const uint8_t* rgb_host) {
  if (!s || !depth_host || s->batch || s->owner_stream) return DYN_ERR_INVALID_ARG;
  DeviceGuard dg(s->device);
  return submit_frame(s, depth_host, rgb_host, false, nullptr);
}

dyn_status dyn_frame_submit_hint(dyn_session* s, const uint16_t* depth_host,
                                 const uint8_t* rgb_host, const float pose_hint[16]) {
  if (!s || !depth_host || s->batch || s->owner_stream) return DYN_ERR_INVALID_ARG;
  DeviceGuard dg(s->device);
  return submit_frame(s, depth_host, rgb_host, false, pose_hint);
}

dyn_status dyn_frame_submit_device(dyn_session* s, const uint16_t* depth_dev, const uint8_t* rgb_dev) {
  if (!s || !depth_dev || s->batch || s->owner_stream) return DYN_ERR_INVALID_ARG;
  DeviceGuard dg(s->device);
  return submit_frame(s, depth_dev, rgb_dev, true, nullptr);
}

dyn_status dyn_frame_result(dyn_session* s, float pose_out[16], dyn_frame_stats* stats) {
  if (!s) return DYN_ERR_INVALID_ARG;
  if (s->n_inflight == 0) return DYN_ERR_NOT_READY;
  DeviceGuard dg(s->device);
  const int k = s->inflight[0];
  DYN_CUDA(cudaEventSynchronize(s->ev_done[k]));
  s->inflight[0] = s->inflight[1];
  s->n_inflight--;
  s->pending = s->n_inflight > 0;
  // stage events are re-recorded by every frame: read them only when no
  // later frame is in flight
  if (s->profile && s->n_inflight == 0) add_stage_times(s->ev, s->stage_ms, &s->prof_frames);
  const ResultBlock& res = *slot_io(s, k).h_res;
  if (pose_out)
    for (int j = 0; j < 16; ++j) pose_out[j] = (float)res.pose.pose[j];
  if (stats) fill_stats(s, res, stats);
  return counters_status(res.cnt);
}

dyn_status dyn_integrate_with_pose(dyn_session* s, const uint16_t* depth_host,
                                   const uint8_t* rgb_host, const float pose[16]) {
  if (!s || !depth_host || !pose || s->batch || s->owner_stream) return DYN_ERR_INVALID_ARG;
  DeviceGuard dg(s->device);
  dyn_status r = dyn_session_set_pose(s, pose);
  if (r != DYN_OK) return r;
  r = upload_frame(s, depth_host, rgb_host);
  if (r != DYN_OK) return r;
  const Marks none;
  enqueue_source(s->d_sd, s->shape, s->stream, none);
  bump_frame_kernel<<<1, 32, 0, s->stream>>>(s->d_pose);
  enqueue_map_update(s->d_sd, s->shape, s->stream, none);
  gather_results_kernel<<<1, 128, 0, s->stream>>>(s->d_sd, 1, nullptr, s->d_res);
  DYN_CUDA(cudaMemcpyAsync(s->h_res_aux, s->d_res, sizeof(ResultBlock), cudaMemcpyDeviceToHost,
                           s->stream));
  DYN_CUDA(cudaStreamSynchronize(s->stream));
  DYN_CUDA(cudaGetLastError());
  s->frames++;
  return counters_status(s->h_res_aux->cnt);
}

dyn_status dyn_solver_solve(dyn_session* s, const float* target_depth_host,
                            const uint8_t* target_rgb_host, const float* source_depth_host,
                            const uint8_t* source_rgb_host, float pose_inout[16],
                            double increment_out[6], dyn_frame_stats* stats) {
  if (!s || !target_depth_host || !source_depth_host || !pose_inout || s->batch || s->owner_stream)
    return DYN_ERR_INVALID_ARG;
  DeviceGuard dg(s->device);
  cudaStream_t st = s->stream;
  const size_t n = s->npx;
  const bool col = s->use_color();
  const float inf = 3.402823466e+38f;
  dyn_status r = dyn_session_set_pose(s, pose_inout);
  if (r != DYN_OK) return r;
  // target: images as given (the reference solves on raw images,
  // builder.cu:91-99), pyramid + normals
  DYN_CUDA(cudaMemcpyAsync(s->d_ray, target_depth_host, n * 4, cudaMemcpyHostToDevice, st));
  if (col && target_rgb_host)
    DYN_CUDA(cudaMemcpyAsync(s->d_trgb, target_rgb_host, n * 3, cudaMemcpyHostToDevice, st));
  launch_target_prepare(s->d_ray, s->d_tdep[0], inf, (col && target_rgb_host) ? s->d_trgb : nullptr,
                        col ? s->d_tint[0] : nullptr, (int)n, st);
  // source
  DYN_CUDA(cudaMemcpyAsync(s->d_raw, source_depth_host, n * 4, cudaMemcpyHostToDevice, st));
  if (col && source_rgb_host)
    DYN_CUDA(cudaMemcpyAsync(s->d_rgb, source_rgb_host, n * 3, cudaMemcpyHostToDevice, st));
  launch_target_prepare(s->d_raw, s->d_sdep[0], inf, (col && source_rgb_host) ? s->d_rgb : nullptr,
                        col ? s->d_sint[0] : nullptr, (int)n, st);
  for (int l = 1; l < s->nlev; ++l) {
    launch_downsample_depth(s->d_tdep[l - 1], s->ls[l - 1].rows, s->ls[l - 1].cols, s->d_tdep[l], st);
    launch_downsample_depth(s->d_sdep[l - 1], s->ls[l - 1].rows, s->ls[l - 1].cols, s->d_sdep[l], st);
    if (col) {
      launch_downsample_intensity(s->d_tint[l - 1], s->ls[l - 1].rows, s->ls[l - 1].cols,
                                  s->d_tint[l], st);
      launch_downsample_intensity(s->d_sint[l - 1], s->ls[l - 1].rows, s->ls[l - 1].cols,
                                  s->d_sint[l], st);
    }
  }
  launch_maps(maps_args(s, true), st);
  launch_maps(maps_args(s, false), st);
  mark_target_kernel<<<1, 32, 0, st>>>(s->d_icp);
  enqueue_icp(s->d_sd, s->shape, st);
  fused_pose_finalize(s->d_sd, s->shape, 0, st);
  gather_results_kernel<<<1, 128, 0, st>>>(s->d_sd, 1, nullptr, s->d_res);
  DYN_CUDA(cudaMemcpyAsync(s->h_res_aux, s->d_res, sizeof(ResultBlock), cudaMemcpyDeviceToHost,
                           st));
  DYN_CUDA(cudaStreamSynchronize(st));
  DYN_CUDA(cudaGetLastError());
  for (int k = 0; k < 16; ++k) pose_inout[k] = (float)s->h_res_aux->pose.pose[k];
  if (increment_out)
    for (int k = 0; k < 6; ++k) increment_out[k] = s->h_res_aux->pose.last_inc[k];
  if (stats) fill_stats(s, *s->h_res_aux, stats);
  return DYN_OK;
}

dyn_status dyn_raycast(dyn_session* s, const float pose[16], const dyn_sensor* virt,
                       float* depth_host, uint8_t* rgb_host) {
  if (!s || !pose || !depth_host) return DYN_ERR_INVALID_ARG;
  dyn_sensor vs = virt ? *virt : s->sensor;
  if (!valid_sensor(&vs) || (size_t)vs.rows * vs.cols > s->npx) return DYN_ERR_INVALID_ARG;
  DeviceGuard dg(s->device);
  DYN_TRY(quiesce(s));
  DYN_CUDA(cudaMemcpyAsync(s->d_pose_override, pose, 64, cudaMemcpyHostToDevice, s->stream));
  size_t n = (size_t)vs.rows * vs.cols;
  launch_raycast(s->vol, dsensor(vs), s->d_pose, s->d_pose_override, s->d_ray,
                 rgb_host ? s->d_trgb : nullptr, s->stream);
  DYN_CUDA(cudaGetLastError());
  DYN_CUDA(cudaMemcpyAsync(depth_host, s->d_ray, n * 4, cudaMemcpyDeviceToHost, s->stream));
  if (rgb_host)
    DYN_CUDA(cudaMemcpyAsync(rgb_host, s->d_trgb, n * 3, cudaMemcpyDeviceToHost, s->stream));
  DYN_CUDA(cudaStreamSynchronize(s->stream));
  return DYN_OK;
}

dyn_status dyn_raycast_maps(dyn_session* s, const float pose[16], const dyn_sensor* virt,
                            float* depth_host, float* vertex4_host, float* normal4_host,
                            uint8_t* rgb_host) {
  if (!s || !pose) return DYN_ERR_INVALID_ARG;
  dyn_sensor vs = virt ? *virt : s->sensor;
  if (!valid_sensor(&vs) || (size_t)vs.rows * vs.cols > s->npx) return DYN_ERR_INVALID_ARG;
  DeviceGuard dg(s->device);
  DYN_TRY(quiesce(s));
  cudaStream_t st = s->stream;
  DYN_CUDA(cudaMemcpyAsync(s->d_pose_override, pose, 64, cudaMemcpyHostToDevice, st));
  const size_t n = (size_t)vs.rows * vs.cols;
  launch_raycast(s->vol, dsensor(vs), s->d_pose, s->d_pose_override, s->d_ray,
                 rgb_host ? s->d_trgb : nullptr, st);
  // misses (at max_sensor_depth or beyond) become invalid depth, then the
  // maps of that depth in the raycast camera's frame
  launch_target_prepare(s->d_ray, s->d_filt, s->tp.max_sensor_depth, nullptr, nullptr, (int)n,
                        st);
  MapsArgs a;
  std::memset(&a, 0, sizeof(a));
  a.lv[0].depth = s->d_filt;
  a.lv[0].normal = s->d_snrm[0];
  a.lv[0].vertex = s->d_svtx[0];
  a.lv[0].s = dsensor(vs);
  a.nlev = 1;
  a.total = (int)n;
  launch_maps(a, st);
  DYN_CUDA(cudaGetLastError());
  if (depth_host)
    DYN_CUDA(cudaMemcpyAsync(depth_host, s->d_ray, n * 4, cudaMemcpyDeviceToHost, st));
  if (vertex4_host)
    DYN_CUDA(cudaMemcpyAsync(vertex4_host, s->d_svtx[0], n * 16, cudaMemcpyDeviceToHost, st));
  if (normal4_host)
    DYN_CUDA(cudaMemcpyAsync(normal4_host, s->d_snrm[0], n * 16, cudaMemcpyDeviceToHost, st));
  if (rgb_host) DYN_CUDA(cudaMemcpyAsync(rgb_host, s->d_trgb, n * 3, cudaMemcpyDeviceToHost, st));
  DYN_CUDA(cudaStreamSynchronize(st));
  return DYN_OK;
}

dyn_status dyn_num_blocks(dyn_session* s, int64_t* n_out) {
  if (!s || !n_out) return DYN_ERR_INVALID_ARG;
  DeviceGuard dg(s->device);
  DYN_TRY(quiesce(s));
  int n = 0;
  DYN_CUDA(cudaMemcpyAsync(&n, &s->vol.cnt->nalloc, sizeof(int), cudaMemcpyDeviceToHost, s->stream));
  DYN_CUDA(cudaStreamSynchronize(s->stream));
  *n_out = std::min(n, s->tp.num_blocks);
  return DYN_OK;
}

dyn_status dyn_find_blocks(dyn_session* s, const int32_t* coords, int64_t n,
                           int32_t* heap_index_out) {
  if (!s || n < 0 || (n > 0 && (!coords || !heap_index_out))) return DYN_ERR_INVALID_ARG;
  if (n == 0) return DYN_OK;
  if (n > (int64_t)1 << 30) return DYN_ERR_INVALID_ARG;
  DeviceGuard dg(s->device);
  DYN_TRY(quiesce(s));
  cudaStream_t st = s->stream;
  int32_t* dc = nullptr;
  int32_t* dp = nullptr;
  dyn_status r = DYN_OK;
  do {
    if (cudaMallocAsync(&dc, sizeof(int32_t) * 3 * (size_t)n, st) != cudaSuccess ||
        cudaMallocAsync(&dp, sizeof(int32_t) * (size_t)n, st) != cudaSuccess) {
      r = DYN_ERR_OOM;
      break;
    }
    if (cudaMemcpyAsync(dc, coords, sizeof(int32_t) * 3 * (size_t)n, cudaMemcpyHostToDevice,
                        st) != cudaSuccess) {
      r = DYN_ERR_CUDA;
      break;
    }
    launch_find_blocks(s->vol, dc, (int)n, dp, st);
    if (cudaGetLastError() != cudaSuccess ||
        cudaMemcpyAsync(heap_index_out, dp, sizeof(int32_t) * (size_t)n, cudaMemcpyDeviceToHost,
                        st) != cudaSuccess)
      r = DYN_ERR_CUDA;
  } while (false);
  if (r != DYN_OK) cudaGetLastError();
  for (void* p : {(void*)dc, (void*)dp})
    if (p) cudaFreeAsync(p, st);
  if (cudaStreamSynchronize(st) != cudaSuccess && r == DYN_OK) r = DYN_ERR_CUDA;
  return r;
}

dyn_status dyn_download_blocks(dyn_session* s, int32_t* coords_out, dyn_voxel* voxels_out,
                               int64_t capacity, int64_t* n_out) {
  if (!s || !n_out || capacity < 0) return DYN_ERR_INVALID_ARG;
  int64_t n = 0;
  dyn_status r = dyn_num_blocks(s, &n);
  if (r != DYN_OK) return r;
  *n_out = n;
  int64_t m = std::min(n, capacity);
  if (m == 0) return DYN_OK;
  DeviceGuard dg(s->device);
  if (coords_out) {
    std::vector<unsigned long long> keys((size_t)m);
    DYN_CUDA(cudaMemcpyAsync(keys.data(), s->vol.block_keys, sizeof(unsigned long long) * m,
                             cudaMemcpyDeviceToHost, s->stream));
    DYN_CUDA(cudaStreamSynchronize(s->stream));
    for (int64_t i = 0; i < m; ++i) {
      coords_out[3 * i] = key_x(keys[i]);
      coords_out[3 * i + 1] = key_y(keys[i]);
      coords_out[3 * i + 2] = key_z(keys[i]);
    }
  }
  if (voxels_out && !s->vol.fp16) {
    DYN_CUDA(cudaMemcpyAsync(voxels_out, s->vol.voxels, sizeof(dyn_voxel) * kBlockVox * m,
                             cudaMemcpyDeviceToHost, s->stream));
    DYN_CUDA(cudaStreamSynchronize(s->stream));
  } else if (voxels_out) {
    // mixed form: f16 sdf / u16 weight (+ colour) converted to the 8-byte
    // voxel; weights above 255 saturate
    const size_t nv = (size_t)kBlockVox * m;
    std::vector<unsigned> v16(nv);
    std::vector<uchar4> col(s->vol.colors ? nv : 0);
    DYN_CUDA(cudaMemcpyAsync(v16.data(), s->vol.vox16, sizeof(unsigned) * nv,
                             cudaMemcpyDeviceToHost, s->stream));
    if (s->vol.colors)
      DYN_CUDA(cudaMemcpyAsync(col.data(), s->vol.colors, sizeof(uchar4) * nv,
                               cudaMemcpyDeviceToHost, s->stream));
    DYN_CUDA(cudaStreamSynchronize(s->stream));
    for (size_t i = 0; i < nv; ++i) {
      __half_raw hr;
      hr.x = (unsigned short)(v16[i] & 0xffffu);
      dyn_voxel& o = voxels_out[i];
      o.sdf = __half2float(__half(hr)) * s->tp.truncation_distance;  // stored as sdf / trunc
      unsigned w = v16[i] >> 16;
      o.weight = (uint8_t)(w > 255 ? 255 : w);
      o.r = s->vol.colors ? col[i].x : 0;
      o.g = s->vol.colors ? col[i].y : 0;
      o.b = s->vol.colors ? col[i].z : 0;
    }
  }
  return DYN_OK;
}

dyn_status dyn_debug_image(dyn_session* s, int32_t which, int32_t level, void* host_out,
                           size_t bytes) {
  if (!s || !host_out || level < 0 || level >= s->nlev) return DYN_ERR_INVALID_ARG;
  DeviceGuard dg(s->device);
  DYN_TRY(quiesce(s));
  size_t m = (size_t)s->ls[level].rows * s->ls[level].cols;
  const void* src = nullptr;
  size_t nb = 0;
  switch (which) {
    case 0: src = s->d_raw; nb = s->npx * 4; break;
    case 1: src = s->d_filt; nb = s->npx * 4; break;
    case 2: src = s->d_sdep[level]; nb = m * 4; break;
    case 3: src = s->d_svtx[level]; nb = m * 16; break;
    case 4: src = s->d_snrm[level]; nb = m * 16; break;
    case 5: src = s->d_tdep[level]; nb = m * 4; break;
    case 6: src = s->d_tvtx[level]; nb = m * 16; break;
    case 7: src = s->d_tnrm[level]; nb = m * 16; break;
    case 8: src = s->d_trgb; nb = s->npx * 3; break;
    case 9: src = s->d_sint[level]; nb = m * 4; break;
    case 10: src = s->d_tint[level]; nb = m * 4; break;
    default: return DYN_ERR_INVALID_ARG;
  }
  if (bytes < nb) return DYN_ERR_INVALID_ARG;
  if ((which == 3 || which == 6) && !s->debug_maps) {
    // vertex maps are only written in debug mode: recompute them now
    s->debug_maps = true;
    launch_maps(maps_args(s, which == 6), s->stream);
    s->debug_maps = false;
  }
  DYN_CUDA(cudaMemcpyAsync(host_out, src, nb, cudaMemcpyDeviceToHost, s->stream));
  DYN_CUDA(cudaStreamSynchronize(s->stream));
  return DYN_OK;
}

dyn_status dyn_session_stream(dyn_session* s, void** stream_out) {
  if (!s || !stream_out) return DYN_ERR_INVALID_ARG;
  *stream_out = (void*)s->stream;
  return DYN_OK;
}

dyn_status dyn_session_profile(dyn_session* s, int32_t enable) {
  if (!s) return DYN_ERR_INVALID_ARG;
  DeviceGuard dg(s->device);
  DYN_CUDA(cudaStreamSynchronize(s->stream));
  bool en = enable != 0;
  if (en && !s->ev[0])
    for (int k = 0; k < DYN_NUM_STAGES; ++k) DYN_CUDA(cudaEventCreate(&s->ev[k]));
  if (en != s->profile) {
    for (cudaGraphExec_t* e : {&s->exec, &s->exec_1})
      if (*e) {
        cudaGraphExecDestroy(*e);
        *e = nullptr;
      }
    s->profile = en;
  }
  return DYN_OK;
}

dyn_status dyn_session_stage_times(dyn_session* s, double ms_out[DYN_NUM_STAGES],
                                   int64_t* frames_out, int32_t reset) {
  if (!s) return DYN_ERR_INVALID_ARG;
  if (ms_out)
    for (int k = 0; k < DYN_NUM_STAGES; ++k) ms_out[k] = s->stage_ms[k];
  if (frames_out) *frames_out = s->prof_frames;
  if (reset) {
    for (int k = 0; k < DYN_NUM_STAGES; ++k) s->stage_ms[k] = 0.0;
    s->prof_frames = 0;
  }
  return DYN_OK;
}

size_t dyn_frame_d2h_bytes(void) { return sizeof(PoseState) + sizeof(IcpState) + sizeof(Counters); }

dyn_status dyn_session_kernels_per_frame(dyn_session* s, int32_t* n_out) {
  if (!s || !n_out) return DYN_ERR_INVALID_ARG;
  *n_out = s->kernels_per_frame;
  return DYN_OK;
}

dyn_status dyn_bilateral_filter(const float* depth_dev, float* out_dev, uint32_t rows, uint32_t cols,
                                const dyn_bilateral_params* p, void* stream) {
  if (!depth_dev || !out_dev || !p || rows == 0 || cols == 0 || p->diameter < 1 ||
      p->diameter > 16 || !(p->sigma_i > 0) || !(p->sigma_s > 0))
    return DYN_ERR_INVALID_ARG;
  BilateralTable tb = make_bilateral_table(p->diameter, p->sigma_i, p->sigma_s);
  launch_bilateral(depth_dev, out_dev, (int)rows, (int)cols, tb, (cudaStream_t)stream);
  DYN_CUDA(cudaGetLastError());
  return DYN_OK;
}

dyn_status dyn_depth_to_maps_host(const float* depth_host, const dyn_sensor* level,
                                  float* vertex4_host, float* normal4_host) {
  if (!depth_host || !valid_sensor(level) || !normal4_host) return DYN_ERR_INVALID_ARG;
  const size_t n = (size_t)level->rows * level->cols;
  cudaStream_t st = cudaStreamPerThread;
  float* d = nullptr;
  float4* v = nullptr;
  float4* nm = nullptr;
  dyn_status r = DYN_OK;
  do {
    if (cudaMallocAsync(&d, n * 4, st) != cudaSuccess ||
        cudaMallocAsync(&nm, n * 16, st) != cudaSuccess ||
        (vertex4_host && cudaMallocAsync(&v, n * 16, st) != cudaSuccess)) {
      r = DYN_ERR_OOM;
      break;
    }
    if (cudaMemcpyAsync(d, depth_host, n * 4, cudaMemcpyHostToDevice, st) != cudaSuccess) {
      r = DYN_ERR_CUDA;
      break;
    }
    r = dyn_depth_to_maps(d, level, reinterpret_cast<float*>(v), reinterpret_cast<float*>(nm),
                          st);
    if (r != DYN_OK) break;
    if (cudaMemcpyAsync(normal4_host, nm, n * 16, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        (vertex4_host &&
         cudaMemcpyAsync(vertex4_host, v, n * 16, cudaMemcpyDeviceToHost, st) != cudaSuccess))
      r = DYN_ERR_CUDA;
  } while (false);
  if (r != DYN_OK) cudaGetLastError();
  for (void* p : {(void*)d, (void*)v, (void*)nm})
    if (p) cudaFreeAsync(p, st);
  if (cudaStreamSynchronize(st) != cudaSuccess && r == DYN_OK) r = DYN_ERR_CUDA;
  return r;
}

dyn_status dyn_depth_to_maps(const float* depth_dev, const dyn_sensor* level, float* vertex4_dev,
                             float* normal4_dev, void* stream) {
  if (!depth_dev || !valid_sensor(level) || !normal4_dev) return DYN_ERR_INVALID_ARG;
  MapsArgs a;
  std::memset(&a, 0, sizeof(a));
  a.lv[0].depth = depth_dev;
  a.lv[0].normal = reinterpret_cast<float4*>(normal4_dev);
  a.lv[0].vertex = reinterpret_cast<float4*>(vertex4_dev);
  a.lv[0].s = dsensor(*level);
  a.lv[0].offset = 0;
  a.nlev = 1;
  a.total = (int)(level->rows * level->cols);
  launch_maps(a, (cudaStream_t)stream);
  DYN_CUDA(cudaGetLastError());
  return DYN_OK;
}

dyn_status dyn_icp_normal_equations(const float* src_depth_dev, const float* src_normal4_dev,
                                    const float* src_intensity_dev, const float* tgt_depth_dev,
                                    const float* tgt_normal4_dev, const float* tgt_intensity_dev,
                                    const dyn_sensor* level, const dyn_gn_params* gn,
                                    const float T[16], double out_host[29], void* stream) {
  if (!src_depth_dev || !src_normal4_dev || !tgt_depth_dev || !tgt_normal4_dev ||
      !valid_sensor(level) || !gn || !T || !out_host)
    return DYN_ERR_INVALID_ARG;
  if (gn->color_weight != 0.0f && (!src_intensity_dev || !tgt_intensity_dev))
    return DYN_ERR_INVALID_ARG;
  int dev = 0;
  DYN_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) return DYN_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> lk(g_stage_mu);
  StageScratch& sc = g_stage[dev];
  if (!sc.partials) {
    DYN_CUDA(cudaMalloc(&sc.partials, icp_scratch_bytes()));
    DYN_CUDA(cudaMalloc(&sc.ticket, 256));
    DYN_CUDA(cudaMemset(sc.ticket, 0, 256));
    DYN_CUDA(cudaMalloc(&sc.out, 256));
    DYN_CUDA(cudaMalloc(&sc.T, 64));
  }
  cudaStream_t st = (cudaStream_t)stream;
  IcpLevel L;
  L.sd = src_depth_dev;
  L.sn = reinterpret_cast<const float4*>(src_normal4_dev);
  L.si = src_intensity_dev;
  L.td = tgt_depth_dev;
  L.tn = reinterpret_cast<const float4*>(tgt_normal4_dev);
  L.ti = tgt_intensity_dev;
  L.s = dsensor(*level);
  IcpParams P;
  P.dmin = gn->icp_min_depth;
  P.dmax = gn->icp_max_depth;
  P.cos_thr = gn->normal_cos_thresh;
  P.cw = gn->color_weight;
  P.min_inc = gn->min_increment;
  P.max_inc = gn->max_increment;
  P.reg = gn->regularization;
  P.compose_left = gn->compose_left;
  P.kahan = 0;
  DYN_CUDA(cudaMemcpyAsync(sc.T, T, 64, cudaMemcpyHostToDevice, st));
  launch_icp_reduce_only(L, P, sc.T, sc.partials, sc.ticket, sc.out, st);
  DYN_CUDA(cudaGetLastError());
  DYN_CUDA(cudaMemcpyAsync(out_host, sc.out, sizeof(double) * kIcpVals, cudaMemcpyDeviceToHost, st));
  DYN_CUDA(cudaStreamSynchronize(st));
  return DYN_OK;
}

dyn_status dyn_barrier_selftest(int32_t device, int32_t blocks, int32_t missing) {
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return DYN_ERR_NO_DEVICE;
  }
  if (device < 0 || device >= ndev || blocks < 1 || missing < 0) return DYN_ERR_INVALID_ARG;
  DeviceGuard dg(device);
  unsigned* bar = nullptr;
  cudaStream_t st = nullptr;
  if (cudaMalloc(&bar, kIcpBarWords * sizeof(unsigned)) != cudaSuccess ||
      cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) {
    cudaGetLastError();
    if (bar) cudaFree(bar);
    return DYN_ERR_OOM;
  }
  const dyn_status r = icp_barrier_selftest(blocks, missing, bar, st);
  cudaStreamSynchronize(st);
  cudaStreamDestroy(st);
  cudaFree(bar);
  return r;
}

dyn_status dyn_sessions_submit(dyn_session* const* sessions, int32_t n,
                               const uint16_t* const* depth_host,
                               const uint8_t* const* rgb_host) {
  if (!sessions || n < 0 || !depth_host) return DYN_ERR_INVALID_ARG;
  for (int i = 0; i < n; ++i) {
    dyn_status r = dyn_frame_submit(sessions[i], depth_host[i], rgb_host ? rgb_host[i] : nullptr);
    if (r != DYN_OK) return r;
  }
  return DYN_OK;
}

}  // extern "C"

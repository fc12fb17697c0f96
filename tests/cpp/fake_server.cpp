// A stand-in for the serving entry points of libdynamap_b200 (dynamap.h),
// for CPU tests of the streaming front end's policies
// (include/nodeHandler/nodeHandler.h) without a GPU.  It keeps the C ABI's
// contract as the front end relies on it:
//  * a session costs num_blocks * 100 bytes of the server's budget;
//    admission beyond the budget returns DYN_ERR_BUDGET_EXCEEDED;
//  * dyn_server_step processes every pushed frame at once (synchronously):
//    a frame whose first depth pixel is k adds blocks (k, session id, 0..2)
//    with every voxel's sdf = k and moves the pose 0.01 m along x from the
//    last pose (the first frame of a session keeps its first pose);
//  * blocks download and upload as coordinates plus 512 voxels.
//  * dyn_evict_blocks removes the blocks of frames more than max_age before
//    the last processed one.
// Every call is counted in fake_calls() for the test driver.
#include <cstdint>
#include <cstring>
#include <map>
#include <tuple>
#include <vector>

#include "dynamap.h"

struct dyn_session {
  int id = 0;
  std::map<std::tuple<int, int, int>, std::vector<dyn_voxel>> blocks;
  float pose[16];
  int frames = 0;
  int pending = -1;  // the pushed frame's first depth pixel, -1 when none
  int last_k = 0;    // the last processed frame's
  int64_t bytes = 0;
};

struct dyn_server {
  size_t budget = 0, used = 0;
  std::vector<dyn_session*> slots;
  int next_id = 0;
  int64_t steps = 0;
};

static int64_t g_calls[8];  // admits, releases, steps, downloads, uploads

extern "C" {

const int64_t* fake_calls() { return g_calls; }

const char* dyn_status_string(dyn_status s) { return s == DYN_OK ? "ok" : "error"; }

dyn_status dyn_server_create(const dyn_server_params* p, dyn_server** out) {
  dyn_server* sv = new dyn_server();
  sv->budget = p->budget_bytes;
  sv->slots.assign(p->max_sessions > 0 ? p->max_sessions : 256, nullptr);
  *out = sv;
  return DYN_OK;
}

dyn_status dyn_server_destroy(dyn_server* sv) {
  for (dyn_session* s : sv->slots) delete s;
  delete sv;
  return DYN_OK;
}

dyn_status dyn_server_admit(dyn_server* sv, const dyn_tsdf_params* tsdf, const dyn_gn_params*,
                            const dyn_bilateral_params*, const dyn_sensor*, int32_t,
                            const float pose0[16], int32_t* slot_out) {
  const int64_t bytes = (int64_t)tsdf->num_blocks * 100;
  if (sv->used + bytes > sv->budget) return DYN_ERR_BUDGET_EXCEEDED;
  for (size_t i = 0; i < sv->slots.size(); ++i)
    if (!sv->slots[i]) {
      dyn_session* s = new dyn_session();
      s->id = sv->next_id++;
      s->bytes = bytes;
      std::memcpy(s->pose, pose0, sizeof(s->pose));
      sv->slots[i] = s;
      sv->used += bytes;
      *slot_out = (int32_t)i;
      g_calls[0]++;
      return DYN_OK;
    }
  return DYN_ERR_BUDGET_EXCEEDED;
}

dyn_status dyn_server_release(dyn_server* sv, int32_t slot) {
  dyn_session* s = sv->slots.at(slot);
  if (!s) return DYN_ERR_INVALID_ARG;
  sv->used -= s->bytes;
  delete s;
  sv->slots[slot] = nullptr;
  g_calls[1]++;
  return DYN_OK;
}

dyn_status dyn_server_session(dyn_server* sv, int32_t slot, dyn_session** out) {
  if (slot < 0 || slot >= (int)sv->slots.size() || !sv->slots[slot]) return DYN_ERR_INVALID_ARG;
  *out = sv->slots[slot];
  return DYN_OK;
}

dyn_status dyn_server_push(dyn_server* sv, int32_t slot, const uint16_t* depth_host,
                           const uint8_t*) {
  dyn_session* s = sv->slots.at(slot);
  if (!s) return DYN_ERR_INVALID_ARG;
  if (s->pending >= 0) return DYN_ERR_NOT_READY;
  s->pending = depth_host[0];
  return DYN_OK;
}

dyn_status dyn_server_step(dyn_server* sv, int32_t* n_out) {
  int n = 0;
  for (dyn_session* s : sv->slots) {
    if (!s || s->pending < 0) continue;
    const int k = s->pending;
    if (s->frames > 0) s->pose[3] += 0.01f;
    for (int z = 0; z < 3; ++z) {
      std::vector<dyn_voxel> v(512);
      for (dyn_voxel& x : v) {
        std::memset(&x, 0, sizeof(x));
        x.weight = 1;
        x.sdf = (float)k;
      }
      s->blocks[std::make_tuple(k, s->id, z)] = v;
    }
    s->frames++;
    s->last_k = k;
    s->pending = -2;  // processed, result not read
    ++n;
  }
  sv->steps++;
  g_calls[2]++;
  if (n_out) *n_out = n;
  return DYN_OK;
}

dyn_status dyn_server_poll(dyn_server* sv, int32_t slot, int32_t* ready_out) {
  dyn_session* s = sv->slots.at(slot);
  *ready_out = s && s->pending == -2 ? 1 : 0;
  return DYN_OK;
}

dyn_status dyn_server_result(dyn_server* sv, int32_t slot, float pose_out[16],
                             dyn_frame_stats* stats) {
  dyn_session* s = sv->slots.at(slot);
  if (!s || s->pending != -2) return DYN_ERR_NOT_READY;
  s->pending = -1;
  std::memcpy(pose_out, s->pose, sizeof(s->pose));
  if (stats) {
    std::memset(stats, 0, sizeof(*stats));
    stats->frame_index = s->frames - 1;
    stats->blocks_total = (int32_t)s->blocks.size();
  }
  return DYN_OK;
}

dyn_status dyn_num_blocks(dyn_session* s, int64_t* n_out) {
  *n_out = (int64_t)s->blocks.size();
  return DYN_OK;
}

dyn_status dyn_download_blocks(dyn_session* s, int32_t* coords_out, dyn_voxel* voxels_out,
                               int64_t capacity, int64_t* n_out) {
  int64_t i = 0;
  for (const auto& kv : s->blocks) {
    if (i < capacity) {
      coords_out[3 * i] = std::get<0>(kv.first);
      coords_out[3 * i + 1] = std::get<1>(kv.first);
      coords_out[3 * i + 2] = std::get<2>(kv.first);
      if (voxels_out) std::memcpy(voxels_out + 512 * i, kv.second.data(), 512 * sizeof(dyn_voxel));
    }
    ++i;
  }
  *n_out = i;
  g_calls[3]++;
  return DYN_OK;
}

dyn_status dyn_upload_blocks(dyn_session* s, const int32_t* coords, const dyn_voxel* voxels,
                             int64_t n, int64_t counts_out[4]) {
  int64_t placed = 0, present = 0;
  for (int64_t i = 0; i < n; ++i) {
    const auto key = std::make_tuple(coords[3 * i], coords[3 * i + 1], coords[3 * i + 2]);
    if (s->blocks.count(key)) {
      ++present;
      continue;
    }
    s->blocks[key] = std::vector<dyn_voxel>(voxels + 512 * i, voxels + 512 * (i + 1));
    ++placed;
  }
  counts_out[0] = placed;
  counts_out[1] = present;
  counts_out[2] = counts_out[3] = 0;
  g_calls[4]++;
  return DYN_OK;
}

// blocks of frames more than max_age frames before the last one leave
dyn_status dyn_evict_blocks(dyn_session* s, int32_t max_age, int32_t* coords_out,
                            dyn_voxel* voxels_out, int64_t capacity, int64_t* n_out) {
  int64_t i = 0;
  for (auto it = s->blocks.begin(); it != s->blocks.end();) {
    if (std::get<0>(it->first) >= s->last_k - max_age) {
      ++it;
      continue;
    }
    if (i < capacity) {
      coords_out[3 * i] = std::get<0>(it->first);
      coords_out[3 * i + 1] = std::get<1>(it->first);
      coords_out[3 * i + 2] = std::get<2>(it->first);
      std::memcpy(voxels_out + 512 * i, it->second.data(), 512 * sizeof(dyn_voxel));
    }
    ++i;
    it = s->blocks.erase(it);
  }
  *n_out = i;
  g_calls[5]++;
  return DYN_OK;
}

}  // extern "C"

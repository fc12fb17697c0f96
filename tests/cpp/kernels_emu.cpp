// The mesh-extraction and eviction kernels themselves (mesh_kernels.cuh,
// evict_kernels.cuh), run on the CPU by the thread-block emulation of
// cuda_emu.h, over a volume built in host memory with the library's own
// upload kernel, in the order the library's entry points launch them
// (dyn_extract_mesh in mesh.cu, remove_blocks in evict.cu).  The tests
// compare the results with the host builds of the same walks
// (mesh_host.cpp, evict_host.cpp).
#include "cuda_emu.h"

#include <algorithm>
#include <cstdint>
#include <map>
#include <vector>

#include "../../dynamap_b200/csrc/evict_kernels.cuh"
#include "../../dynamap_b200/csrc/mesh_kernels.cuh"

namespace {

constexpr int kGrid = 3;  // blocks per launch: the kernels stride over their work

struct HostVolume {
  dyn::VolumeDev v{};
  std::vector<dyn::Entry> entries;
  std::vector<unsigned long long> keys;
  std::vector<dyn_voxel> voxels;
  std::vector<unsigned> vox16;
  std::vector<uchar4> colors;
  std::vector<int> nonsat;
  std::vector<unsigned char> freecell;
  dyn::Counters cnt{};
  dyn::PoseState ps{};

  HostVolume(float vs, float trunc, int nb, int bsz, int num_blocks, bool fp16) {
    entries.assign((size_t)nb * bsz, dyn::Entry{dyn::kEmptyKey, -1, -1});
    keys.assign(num_blocks, 0);
    if (fp16) {
      vox16.assign((size_t)num_blocks * dyn::kBlockVox, 0u);
      colors.assign((size_t)num_blocks * dyn::kBlockVox, make_uchar4(0, 0, 0, 0));
    } else {
      voxels.assign((size_t)num_blocks * dyn::kBlockVox, dyn_voxel{0, 0, 0, 0, 0.0f});
    }
    v.entries = entries.data();
    v.block_keys = keys.data();
    v.voxels = fp16 ? nullptr : voxels.data();
    v.vox16 = fp16 ? vox16.data() : nullptr;
    v.colors = fp16 ? colors.data() : nullptr;
    v.fp16 = fp16 ? 1 : 0;
    nonsat.assign(num_blocks, 0);
    freecell.assign(num_blocks, 0);
    v.nonsat = nonsat.data();
    v.freecell = freecell.data();
    v.cnt = &cnt;
    v.t.vs = vs;
    v.t.bsm = 8.0f * vs;
    v.t.trunc = trunc;
    v.t.num_buckets = nb;
    v.t.nb_mask = (nb & (nb - 1)) == 0 ? nb - 1 : -1;
    v.t.bucket_size = bsz;
    v.t.num_blocks = num_blocks;
    v.t.max_w = 255;
    v.sat_lo = (float)((double)trunc * (1.0 - 1e-6));
    v.free_ok = v.sat_lo >= vs ? 1 : 0;
  }
  int n() const { return std::min(cnt.nalloc, v.t.num_blocks); }
};

// dyn_upload_blocks: blocks grouped by stamp (the frame counter the upload
// kernel stamps them with).
void upload(HostVolume& H, const int32_t* coords, const dyn_voxel* vox, const int32_t* stamps,
            int n, int64_t counts[4]) {
  std::map<int, std::vector<int>> by_stamp;
  for (int j = 0; j < n; ++j) by_stamp[stamps ? stamps[j] : 0].push_back(j);
  int c[4] = {0, 0, 0, 0};
  for (auto& [stamp, idx] : by_stamp) {
    std::vector<int32_t> cc;
    std::vector<dyn_voxel> vv;
    for (int j : idx) {
      cc.insert(cc.end(), coords + 3 * j, coords + 3 * j + 3);
      vv.insert(vv.end(), vox + (size_t)j * 512, vox + (size_t)j * 512 + 512);
    }
    H.ps.frame = stamp;
    const int m = (int)idx.size();
    emu::launch(std::min(m, kGrid), 64, [&] {
      dyn::upload_kernel(H.v, &H.ps, cc.data(), vv.data(), m, c);
    });
  }
  for (int k = 0; k < 4; ++k) counts[k] = c[k];
}

// dyn_download_blocks's view: heap order, 8-byte voxels.
int64_t download(HostVolume& H, int32_t* coords, dyn_voxel* vox) {
  const int n = H.n();
  for (int i = 0; i < n; ++i) {
    coords[3 * i] = dyn::key_x(H.keys[i]);
    coords[3 * i + 1] = dyn::key_y(H.keys[i]);
    coords[3 * i + 2] = dyn::key_z(H.keys[i]);
    for (int j = 0; j < 512; ++j) vox[(size_t)i * 512 + j] = dyn::voxel8(H.v, (size_t)i * 512 + j);
  }
  return n;
}

}  // namespace

extern "C" {

void* emu_volume(float vs, float trunc, int nb, int bsz, int num_blocks, int fp16) {
  return new HostVolume(vs, trunc, nb, bsz, num_blocks, fp16 != 0);
}
void emu_volume_free(void* h) { delete (HostVolume*)h; }
int emu_nalloc(void* h) { return ((HostVolume*)h)->cnt.nalloc; }
void emu_set_frame(void* h, int frame) { ((HostVolume*)h)->ps.frame = frame; }

void emu_upload(void* h, const int32_t* coords, const void* vox8, const int32_t* stamps,
                int64_t n, int64_t counts[4]) {
  upload(*(HostVolume*)h, coords, (const dyn_voxel*)vox8, stamps, (int)n, counts);
}
int64_t emu_download(void* h, int32_t* coords, void* vox8) {
  return download(*(HostVolume*)h, coords, (dyn_voxel*)vox8);
}

// dyn_extract_mesh: count pass, scan, write pass.
int64_t emu_mesh(void* h, const float lo[3], const float hi[3], float* out, int64_t cap) {
  HostVolume& H = *(HostVolume*)h;
  dyn::mesh::Grid g;
  if (!dyn::mesh::make_grid(lo, hi, H.v.t.vs, &g)) return -1;
  const int n = H.n();
  if (n == 0 || g.n[0] == 0 || g.n[1] == 0 || g.n[2] == 0) return 0;
  std::memcpy(dyn::d_mc_tri, dyn::kMcTriangles, sizeof(dyn::kMcTriangles));
  std::vector<long long> counts(n), offsets(n + 1);
  emu::launch(std::min(n, kGrid), dyn::kMeshThreads, [&] {
    dyn::mesh_blocks_kernel<false>(H.v, g, n, counts.data(), nullptr, nullptr, 0);
  });
  emu::launch(1, 1024, [&] {
    dyn::mesh_scan_kernel(counts.data(), n, offsets.data(), offsets.data() + n);
  });
  const long long total = offsets[n];
  const long long m = std::min<long long>(total, cap);
  if (out && m > 0)
    emu::launch(std::min(n, kGrid), dyn::kMeshThreads, [&] {
      dyn::mesh_blocks_kernel<true>(H.v, g, n, counts.data(), offsets.data(), out, m);
    });
  return total;
}

// remove_blocks: mode 0 by age (frame counter 'last'), mode 1 the blocks at
// the m coordinates; the removed blocks (heap order) into coords_out /
// vox_out up to cap.  Returns the number removed.
int64_t emu_remove(void* h, int mode, int last, int max_age, const int32_t* del, int64_t m,
                   int32_t* coords_out, void* vox_out, int64_t cap) {
  HostVolume& H = *(HostVolume*)h;
  const int n = H.n();
  if (n == 0) return 0;
  std::vector<int> keep(n), pos(n + 1), dead_at(n), dest(n);
  int removed = 0;
  const int T = dyn::kEvT;
  if (mode == 0) {
    std::fill(keep.begin(), keep.end(), 0);
    H.ps.frame = last;
    const long long ne = (long long)H.entries.size();
    emu::launch(kGrid, T, [&] {
      dyn::mark_age_kernel(H.entries.data(), ne, n, &H.ps, max_age, keep.data());
    });
  } else {
    emu::launch(kGrid, T, [&] { dyn::fill_kernel(keep.data(), n, 1); });
    if (m > 0)
      emu::launch(kGrid, T, [&] {
        dyn::mark_coords_kernel(H.v, del, m, n, keep.data(), &removed);
      });
  }
  emu::launch(1, 1024, [&] { dyn::scan_flags_kernel(keep.data(), n, pos.data()); });
  const int L = pos[n];
  const int dead = n - L;
  if (dead == 0) return 0;
  if (mode == 1 && removed != dead) return -1;  // the kernel's own count disagrees
  emu::launch(kGrid, T, [&] { dyn::dead_list_kernel(keep.data(), pos.data(), n, dead_at.data()); });
  const int mm = (int)std::min<int64_t>(dead, cap);
  if (mm > 0 && (coords_out || vox_out)) {
    std::vector<int> gc(3 * (size_t)mm);
    std::vector<dyn_voxel> gv((size_t)mm * 512);
    emu::launch(std::min(mm, kGrid), T, [&] {
      dyn::gather_kernel(H.v, dead_at.data(), mm, gc.data(), gv.data());
    });
    if (coords_out) std::memcpy(coords_out, gc.data(), sizeof(int) * gc.size());
    if (vox_out) std::memcpy(vox_out, gv.data(), sizeof(dyn_voxel) * gv.size());
  }
  emu::launch(kGrid, T, [&] {
    dyn::dest_kernel(keep.data(), pos.data(), n, L, dead_at.data(), dest.data());
  });
  emu::launch(std::min(n - L, kGrid), T, [&] { dyn::move_kernel(H.v, n, L, dest.data()); });
  emu::launch(kGrid, T, [&] {
    dyn::rewrite_kernel(H.entries.data(), H.v.t.num_buckets, H.v.t.bucket_size, n, keep.data(),
                        dest.data());
  });
  const size_t from = (size_t)L * 512, tail = (size_t)(n - L) * 512;
  if (H.v.voxels) std::memset(H.v.voxels + from, 0, sizeof(dyn_voxel) * tail);
  if (H.v.vox16) std::memset(H.v.vox16 + from, 0, sizeof(unsigned) * tail);
  if (H.v.colors) std::memset(H.v.colors + from, 0, sizeof(uchar4) * tail);
  std::fill(H.nonsat.begin() + L, H.nonsat.begin() + n, 0);
  std::fill(H.freecell.begin() + L, H.freecell.begin() + n, 0);
  H.cnt.nalloc = L;
  return dead;
}

// The free-space summaries of heap indices [0, n): counts, then flags.
void emu_summaries(void* h, int32_t* nonsat, uint8_t* freecell) {
  HostVolume& H = *(HostVolume*)h;
  const int n = H.n();
  std::copy(H.nonsat.begin(), H.nonsat.begin() + n, nonsat);
  std::copy(H.freecell.begin(), H.freecell.begin() + n, freecell);
}
// Set block p's flag (a stand-in for the per-frame free-cell pass).
void emu_set_free(void* h, int p, int value) { ((HostVolume*)h)->freecell[p] = (unsigned char)value; }

// A lookup through the library's find_block: heap index or -1.
int emu_find(void* h, int x, int y, int z) {
  HostVolume& H = *(HostVolume*)h;
  return dyn::find_block(H.v.entries, H.v.t, x, y, z);
}

}  // extern "C"

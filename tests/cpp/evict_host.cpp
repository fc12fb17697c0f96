// Host build of block eviction (dynamap_b200/csrc/evict.cu) over the same
// evict_ops.h steps, for the CPU tests: a volume laid out as the device's
// (buckets of {key, ptr, stamp} entries, front-packed; heap of 512-voxel
// blocks with a key per heap index; a bump-allocated heap top), the removal
// run serially step for step, and the checks of its invariants.
#include <cstdint>
#include <cstring>
#include <vector>

#include "../../dynamap_b200/csrc/evict_ops.h"

namespace {

struct Entry {
  unsigned long long key;
  int ptr;
  int stamp;
};
struct Voxel {  // dyn_voxel
  uint8_t r, g, b, w;
  float sdf;
};
static_assert(sizeof(Voxel) == 8, "8-byte voxels");

constexpr int kVox = 512;

unsigned long long pack(int x, int y, int z) {  // 21 bits per axis
  const unsigned long long m = (1ull << 21) - 1;
  return (((unsigned long long)x & m) << 42) | (((unsigned long long)y & m) << 21) |
         ((unsigned long long)z & m);
}
int unpack(unsigned long long k, int shift) {
  return (int)(((long long)((k >> shift) & 0x1FFFFF) << 43) >> 43);
}

struct Vol {
  int nb, bsz, num_blocks;
  int nalloc = 0;
  std::vector<Entry> entries;
  std::vector<unsigned long long> keys;
  std::vector<Voxel> vox;
  int slot(int x, int y, int z) const {  // HashTable::Hash, hashTable.cu:152-163
    const int h = (int)(((unsigned)x * 73856093u) ^ ((unsigned)y * 19349669u) ^
                        ((unsigned)z * 83492791u));
    int r = h % nb;
    if (r < 0) r += nb;
    return r * bsz;
  }
  int find(int x, int y, int z) const {  // the device's find_block
    const int b = slot(x, y, z);
    const unsigned long long k = pack(x, y, z);
    for (int i = 0; i < bsz; ++i) {
      const Entry& e = entries[b + i];
      if (e.key == k) return e.ptr;
      if (e.key == dyn::evict::kNoKey) return -1;
    }
    return -1;
  }
};

}  // namespace

extern "C" {

void* evh_create(int nb, int bsz, int num_blocks) {
  Vol* v = new Vol{nb, bsz, num_blocks};
  v->entries.assign((size_t)nb * bsz, Entry{dyn::evict::kNoKey, -1, -1});
  v->keys.assign(num_blocks, 0);
  v->vox.assign((size_t)num_blocks * kVox, Voxel{0, 0, 0, 0, 0.0f});
  return v;
}
void evh_destroy(void* h) { delete (Vol*)h; }
int evh_nalloc(void* h) { return ((Vol*)h)->nalloc; }

// The allocation's insert (bucket_insert + the bump pointer) and the
// upload's voxel write; counts [placed, present, bucket full, heap exhausted].
void evh_insert(void* h, const int32_t* coords, const uint8_t* vox8, const int32_t* stamps,
                int64_t n, int64_t counts[4]) {
  Vol& v = *(Vol*)h;
  for (int k = 0; k < 4; ++k) counts[k] = 0;
  for (int64_t j = 0; j < n; ++j) {
    const int x = coords[3 * j], y = coords[3 * j + 1], z = coords[3 * j + 2];
    const unsigned long long key = pack(x, y, z);
    const int b = v.slot(x, y, z);
    int r = -2;
    for (int i = 0; i < v.bsz; ++i) {
      Entry& e = v.entries[b + i];
      if (e.key == dyn::evict::kNoKey) {
        e.key = key;
        e.stamp = stamps[j];
        r = b + i;
        break;
      }
      if (e.key == key) {
        e.stamp = stamps[j];
        r = -1;
        break;
      }
    }
    if (r < 0) {
      ++counts[r == -1 ? 1 : 2];
      continue;
    }
    const int ptr = v.nalloc++;
    if (ptr >= v.num_blocks) {
      ++counts[3];
      continue;
    }
    v.entries[r].ptr = ptr;
    v.keys[ptr] = key;
    std::memcpy(&v.vox[(size_t)ptr * kVox], vox8 + (size_t)j * kVox * 8, kVox * 8);
    ++counts[0];
  }
}

// The removal of evict.cu's remove_blocks, serially: mode 0 keeps the blocks
// with last - stamp <= max_age, mode 1 removes those at the m coordinates.
// Removed blocks (heap order) into coords_out / vox_out up to cap; returns
// the number removed.
int64_t evh_remove(void* h, int mode, int last, int max_age, const int32_t* del, int64_t m,
                   int32_t* coords_out, uint8_t* vox_out, int64_t cap) {
  Vol& v = *(Vol*)h;
  const int n = v.nalloc < v.num_blocks ? v.nalloc : v.num_blocks;
  if (n == 0) return 0;
  std::vector<int> keep(n, mode == 0 ? 0 : 1), pos(n + 1), dead_at(n), dest(n);
  if (mode == 0) {
    for (const Entry& e : v.entries) {
      const int p = dyn::evict::entry_block(e, n);
      if (p >= 0 && dyn::evict::young(e, last, max_age)) keep[p] = 1;
    }
  } else {
    for (int64_t j = 0; j < m; ++j) {
      const int p = v.find(del[3 * j], del[3 * j + 1], del[3 * j + 2]);
      if (p >= 0 && p < n) keep[p] = 0;
    }
  }
  int run = 0;
  for (int i = 0; i < n; ++i) {
    pos[i] = run;
    run += keep[i];
  }
  pos[n] = run;
  const int L = run;
  if (L == n) return 0;
  for (int i = 0; i < n; ++i)
    if (!keep[i]) dead_at[dyn::evict::hole_rank(i, pos.data())] = i;
  const int dead = n - L;
  for (int k = 0; k < dead && k < cap; ++k) {
    const int i = dead_at[k];
    if (coords_out) {
      coords_out[3 * k] = unpack(v.keys[i], 42);
      coords_out[3 * k + 1] = unpack(v.keys[i], 21);
      coords_out[3 * k + 2] = unpack(v.keys[i], 0);
    }
    if (vox_out) std::memcpy(vox_out + (size_t)k * kVox * 8, &v.vox[(size_t)i * kVox], kVox * 8);
  }
  for (int i = 0; i < n; ++i)
    dest[i] = dyn::evict::destination(i, L, keep.data(), pos.data(), dead_at.data());
  for (int j = L; j < n; ++j) {
    const int d = dest[j];
    if (d < 0) continue;
    std::memcpy(&v.vox[(size_t)d * kVox], &v.vox[(size_t)j * kVox], kVox * 8);
    v.keys[d] = v.keys[j];
  }
  for (int b = 0; b < v.nb; ++b)
    dyn::evict::rewrite_bucket(&v.entries[(size_t)b * v.bsz], v.bsz, n, keep.data(), dest.data());
  std::memset(&v.vox[(size_t)L * kVox], 0, (size_t)(n - L) * kVox * 8);
  v.nalloc = L;
  return dead;
}

// Blocks [0, nalloc) in heap order.
int64_t evh_download(void* h, int32_t* coords, uint8_t* vox8) {
  Vol& v = *(Vol*)h;
  for (int i = 0; i < v.nalloc && i < v.num_blocks; ++i) {
    coords[3 * i] = unpack(v.keys[i], 42);
    coords[3 * i + 1] = unpack(v.keys[i], 21);
    coords[3 * i + 2] = unpack(v.keys[i], 0);
    std::memcpy(vox8 + (size_t)i * kVox * 8, &v.vox[(size_t)i * kVox], kVox * 8);
  }
  return v.nalloc;
}

int evh_find(void* h, int x, int y, int z) { return ((Vol*)h)->find(x, y, z); }

// 0 when the structure is consistent: every bucket front-packed; each entry
// with a block names a heap index below the top whose key is the entry's;
// every heap index below the top named by exactly one entry; the heap above
// the top zero.  Otherwise a code naming the first broken rule.
int evh_check(void* h) {
  Vol& v = *(Vol*)h;
  const int n = v.nalloc < v.num_blocks ? v.nalloc : v.num_blocks;
  std::vector<int> refs(n, 0);
  for (int b = 0; b < v.nb; ++b) {
    bool empty_seen = false;
    for (int i = 0; i < v.bsz; ++i) {
      const Entry& e = v.entries[(size_t)b * v.bsz + i];
      if (e.key == dyn::evict::kNoKey) {
        empty_seen = true;
        continue;
      }
      if (empty_seen) return 1;
      if (e.ptr < 0) continue;
      if (e.ptr >= n) return 2;
      if (v.keys[e.ptr] != e.key) return 3;
      if (v.slot(unpack(e.key, 42), unpack(e.key, 21), unpack(e.key, 0)) != b * v.bsz) return 4;
      ++refs[e.ptr];
    }
  }
  for (int i = 0; i < n; ++i)
    if (refs[i] != 1) return 5;
  for (size_t i = (size_t)n * kVox; i < v.vox.size(); ++i) {
    const Voxel& x = v.vox[i];
    if (x.r || x.g || x.b || x.w || x.sdf != 0.0f) return 6;
  }
  return 0;
}

}  // extern "C"

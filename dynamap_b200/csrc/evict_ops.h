// evict_ops.h -- the per-element steps of block eviction, shared by the CUDA
// kernels (evict.cu) and a host build of the same steps that the tests run.
// Plain C++ plus DYN_HD qualifiers; the entry type is a template parameter
// with the fields key (u64, ~0 when empty), ptr (heap index, -1 none) and
// stamp (last frame whose allocation touched the block).
//
// Eviction removes a set of allocated blocks and keeps the heap dense: with
// n blocks allocated of which L survive, every survivor ends in [0, L).
// Survivors already below L stay where they are; the holes below L (dead
// blocks) are filled, in index order, by the survivors at L and above, in
// index order -- sources at L and above, destinations below L, so all moves
// can run at once.  Each bucket then keeps its surviving entries in their
// order, front-packed (a lookup stops at the first empty slot), with moved
// heap indices rewritten; heap indices [L, n) are cleared and the heap top
// becomes L, so the allocation's bump pointer resumes there.  The
// reference frees one block at a time onto its heap's free stack
// (HashTable::DeleteBlock, hashTable.cu:112-134, which also zeroes the
// block): the blocks, voxels and lookups that remain are the same.
#pragma once

#include <stdint.h>

#if defined(__CUDACC__)
#define DYN_EV_HD __host__ __device__ __forceinline__
#else
#define DYN_EV_HD inline
#endif

namespace dyn {
namespace evict {

constexpr unsigned long long kNoKey = ~0ull;

// Whether an entry's block survives an age cut: touched by the allocation
// of frame 'last' or of one of the max_age frames before it.
template <class E>
DYN_EV_HD bool young(const E& e, int last, int max_age) {
  return (long long)last - (long long)e.stamp <= (long long)max_age;
}

// The entry's heap index when it holds an allocated block among the first
// n, else -1 (empty slots, and keys whose block the heap could not hold).
template <class E>
DYN_EV_HD int entry_block(const E& e, int n) {
  return (e.key != kNoKey && e.ptr >= 0 && e.ptr < n) ? e.ptr : -1;
}

// Where block i goes, given keep flags, their exclusive prefix sums 'pos'
// (pos[i] = survivors below i) and the holes below L in order ('hole_at'):
// i itself when it survives below L, hole k for the k-th survivor at or
// above L, -1 when it is evicted.
DYN_EV_HD int destination(int i, int L, const int* keep, const int* pos, const int* hole_at) {
  if (!keep[i]) return -1;
  if (i < L) return i;
  return hole_at[pos[i] - pos[L]];
}

// The rank of hole i (a dead block below L) among the holes, in order.
DYN_EV_HD int hole_rank(int i, const int* pos) { return i - pos[i]; }

// One bucket of bsz entries rewritten in place: survivors front-packed in
// their order with their new heap index, the rest emptied.  Returns the
// survivors kept.
template <class E>
DYN_EV_HD int rewrite_bucket(E* bucket, int bsz, int n, const int* keep, const int* dest) {
  int w = 0;
  for (int i = 0; i < bsz; ++i) {
    E e = bucket[i];
    const int p = entry_block(e, n);
    if (p < 0 || !keep[p]) continue;
    e.ptr = dest[p];
    bucket[w++] = e;
  }
  for (int i = w; i < bsz; ++i) {
    bucket[i].key = kNoKey;
    bucket[i].ptr = -1;
    bucket[i].stamp = -1;
  }
  return w;
}

}  // namespace evict
}  // namespace dyn

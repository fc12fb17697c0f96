// Host emulation of CUDA thread blocks, for running this project's kernels
// on the CPU in tests: each CUDA thread of a block is a user-space context
// (ucontext) with its own stack, all run by one host thread, one block at a
// time -- so __shared__ variables become statics -- switching at
// __syncthreads (a barrier of the block) and at the per-warp exchange of
// __shfl_up_sync (a barrier of the warp); atomics are plain operations
// (one host thread), and the float intrinsics the kernels use are the IEEE
// operations they name (compile with -ffp-contract=off).  One-dimensional
// blocks and grids only; a block whose threads wait on a barrier that
// cannot complete aborts the test.
#pragma once

#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <ucontext.h>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <vector>

#define __launch_bounds__(...)
#undef __grid_constant__
#define __grid_constant__
#undef __shared__
#define __shared__ static

inline uint3 threadIdx;
inline uint3 blockIdx;
inline dim3 blockDim;
inline dim3 gridDim;

namespace emu {

enum Wait { kNone = 0, kBlock = 1, kWarp = 2, kDone = 3 };

struct Fiber {
  ucontext_t ctx;
  std::vector<char> stack;
  int wait = kNone;
};

struct Block {
  ucontext_t sched;
  std::vector<Fiber> f;
  std::vector<int> xbuf;  // one 32-bit slot per thread (shuffles)
  std::function<void()> body;
  int cur = 0;
};
inline Block* g_block = nullptr;

inline void fiber_main() {
  g_block->body();
  g_block->f[g_block->cur].wait = kDone;
  // returning resumes uc_link (the scheduler)
}

inline void wait_here(int kind) {
  Block& b = *g_block;
  b.f[b.cur].wait = kind;
  swapcontext(&b.f[b.cur].ctx, &b.sched);
}

// Runs body() as a grid of 'grid' blocks of 'threads' threads.
template <class F>
void launch(int grid, int threads, F body) {
  gridDim = dim3(grid, 1, 1);
  blockDim = dim3(threads, 1, 1);
  Block b;
  b.f.resize(threads);
  b.xbuf.assign(threads, 0);
  b.body = body;
  for (Fiber& x : b.f) x.stack.resize(256 * 1024);
  g_block = &b;
  for (int blk = 0; blk < grid; ++blk) {
    for (int t = 0; t < threads; ++t) {
      Fiber& x = b.f[t];
      getcontext(&x.ctx);
      x.ctx.uc_stack.ss_sp = x.stack.data();
      x.ctx.uc_stack.ss_size = x.stack.size();
      x.ctx.uc_link = &b.sched;
      makecontext(&x.ctx, fiber_main, 0);
      x.wait = kNone;
    }
    for (;;) {
      bool ran = false;
      for (int t = 0; t < threads; ++t) {
        if (b.f[t].wait != kNone) continue;
        b.cur = t;
        threadIdx = make_uint3(t, 0, 0);
        blockIdx = make_uint3(blk, 0, 0);
        swapcontext(&b.sched, &b.f[t].ctx);
        ran = true;
      }
      int done = 0, at_block = 0;
      for (const Fiber& x : b.f) {
        done += x.wait == kDone;
        at_block += x.wait == kBlock;
      }
      if (done == threads) break;
      bool released = false;
      if (at_block > 0 && at_block + done == threads) {
        for (Fiber& x : b.f)
          if (x.wait == kBlock) x.wait = kNone;
        released = true;
      }
      for (int w = 0; w * 32 < threads; ++w) {
        const int lo = 32 * w, hi = std::min(threads, lo + 32);
        int at = 0;
        for (int t = lo; t < hi; ++t) at += b.f[t].wait == kWarp;
        if (at == hi - lo) {
          for (int t = lo; t < hi; ++t) b.f[t].wait = kNone;
          released = true;
        }
      }
      if (!ran && !released) {
        std::fprintf(stderr, "cuda_emu: block %d cannot make progress\n", blk);
        std::abort();
      }
    }
  }
  g_block = nullptr;
}

}  // namespace emu

inline void __syncthreads() { emu::wait_here(emu::kBlock); }

inline int __shfl_up_sync(unsigned, int v, unsigned o) {
  emu::Block& b = *emu::g_block;
  const int t = (int)threadIdx.x, lane = t & 31;
  b.xbuf[t] = v;
  emu::wait_here(emu::kWarp);
  const int r = lane >= (int)o ? b.xbuf[t - (int)o] : v;
  emu::wait_here(emu::kWarp);
  return r;
}

template <class T>
inline T __ldg(const T* p) {
  return *p;
}
inline float __fadd_rn(float a, float b) { return a + b; }
inline float __fmul_rn(float a, float b) { return a * b; }
inline float __fmaf_rn(float a, float b, float c) { return std::fmaf(a, b, c); }
inline unsigned __float_as_uint(float f) {
  unsigned u;
  std::memcpy(&u, &f, 4);
  return u;
}
inline float __uint_as_float(unsigned u) {
  float f;
  std::memcpy(&f, &u, 4);
  return f;
}

inline int atomicAdd(int* p, int v) { return __atomic_fetch_add(p, v, __ATOMIC_SEQ_CST); }
inline int atomicExch(int* p, int v) { return __atomic_exchange_n(p, v, __ATOMIC_SEQ_CST); }
inline int atomicCAS(int* p, int cmp, int v) {
  __atomic_compare_exchange_n(p, &cmp, v, false, __ATOMIC_SEQ_CST, __ATOMIC_SEQ_CST);
  return cmp;
}
inline unsigned long long atomicCAS(unsigned long long* p, unsigned long long cmp,
                                    unsigned long long v) {
  __atomic_compare_exchange_n(p, &cmp, v, false, __ATOMIC_SEQ_CST, __ATOMIC_SEQ_CST);
  return cmp;
}

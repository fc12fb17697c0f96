// Host emulation of CUDA thread blocks, for running this project's kernels
// on the CPU in tests: each thread block is run by blockDim.x host threads
// (one block at a time, so __shared__ variables become statics), with
// __syncthreads as a barrier of the block, __shfl_up_sync through a
// per-warp exchange and barrier, atomics as GCC atomic builtins, and the
// float intrinsics the kernels use as the IEEE operations they name
// (compile with -ffp-contract=off).  One-dimensional blocks and grids only.
#pragma once

#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <barrier>
#include <cmath>
#include <cstring>
#include <memory>
#include <thread>
#include <vector>

#define __launch_bounds__(...)
#undef __grid_constant__
#define __grid_constant__
#undef __shared__
#define __shared__ static

inline thread_local uint3 threadIdx;
inline thread_local uint3 blockIdx;
inline dim3 blockDim;
inline dim3 gridDim;

namespace emu {

struct Block {
  std::unique_ptr<std::barrier<>> all;
  std::vector<std::unique_ptr<std::barrier<>>> warp;
  std::vector<int> xbuf;  // one 32-bit slot per thread
};
inline Block* g_block = nullptr;

// Runs body() as a grid of 'grid' blocks of 'threads' threads.
template <class F>
void launch(int grid, int threads, F body) {
  gridDim = dim3(grid, 1, 1);
  blockDim = dim3(threads, 1, 1);
  Block b;
  b.all = std::make_unique<std::barrier<>>(threads);
  for (int w = 0; w < (threads + 31) / 32; ++w)
    b.warp.push_back(std::make_unique<std::barrier<>>(std::min(32, threads - 32 * w)));
  b.xbuf.assign(threads, 0);
  g_block = &b;
  for (int blk = 0; blk < grid; ++blk) {
    std::vector<std::thread> ts;
    ts.reserve(threads);
    for (int t = 0; t < threads; ++t)
      ts.emplace_back([=] {
        threadIdx = make_uint3(t, 0, 0);
        blockIdx = make_uint3(blk, 0, 0);
        body();
      });
    for (auto& th : ts) th.join();
  }
  g_block = nullptr;
}

}  // namespace emu

inline void __syncthreads() { emu::g_block->all->arrive_and_wait(); }

inline int __shfl_up_sync(unsigned, int v, unsigned o) {
  emu::Block& b = *emu::g_block;
  const int t = (int)threadIdx.x, lane = t & 31;
  std::barrier<>& w = *b.warp[t >> 5];
  b.xbuf[t] = v;
  w.arrive_and_wait();
  const int r = lane >= (int)o ? b.xbuf[t - (int)o] : v;
  w.arrive_and_wait();
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
inline unsigned long long atomicCAS(unsigned long long* p, unsigned long long cmp,
                                    unsigned long long v) {
  __atomic_compare_exchange_n(p, &cmp, v, false, __ATOMIC_SEQ_CST, __ATOMIC_SEQ_CST);
  return cmp;
}

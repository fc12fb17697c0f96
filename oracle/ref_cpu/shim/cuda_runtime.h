// Host-side stand-in for <cuda_runtime.h>, used ONLY to compile the
// reference's own kernel sources for the CPU (oracle/_ref, test
// infrastructure).  It supplies the CUDA vector types, the qualifiers as
// no-ops, the built-in thread indices as thread-local variables, host
// versions of the few device intrinsics and atomics the reference uses, and
// managed memory as host memory.  A kernel launch K<<<g, b>>>(args) is
// rewritten by build_ref.sh into DYNREF_LAUNCH(K)(args): the kernel body
// runs on nthreads host threads, each with its own blockIdx and
// gridDim = nthreads, blockDim = 1 -- every kernel on the path walks its
// work with a grid-stride loop, so the launch covers all of it.
#pragma once

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <thread>
#include <vector>

#define __host__
#define __device__
#define __global__
#define __forceinline__ inline
#define __shared__
#define __constant__

struct uint3 { unsigned int x, y, z; };
struct dim3 {
  unsigned int x, y, z;
  dim3(unsigned int a = 1, unsigned int b = 1, unsigned int c = 1) : x(a), y(b), z(c) {}
};
struct float2 { float x, y; };
struct float3 { float x, y, z; };
struct float4 { float x, y, z, w; };
struct double2 { double x, y; };
struct double3 { double x, y, z; };
struct int2 { int x, y; };
struct int3 { int x, y, z; };
struct int4 { int x, y, z, w; };
struct uint2 { unsigned int x, y; };
struct uint4 { unsigned int x, y, z, w; };
struct uchar2 { unsigned char x, y; };
struct uchar3 { unsigned char x, y, z; };
struct uchar4 { unsigned char x, y, z, w; };
struct char3 { signed char x, y, z; };
struct short3 { short x, y, z; };

inline float2 make_float2(float x, float y) { return {x, y}; }
inline float3 make_float3(float x, float y, float z) { return {x, y, z}; }
inline float4 make_float4(float x, float y, float z, float w) { return {x, y, z, w}; }
inline double3 make_double3(double x, double y, double z) { return {x, y, z}; }
inline int2 make_int2(int x, int y) { return {x, y}; }
inline int3 make_int3(int x, int y, int z) { return {x, y, z}; }
inline int4 make_int4(int x, int y, int z, int w) { return {x, y, z, w}; }
inline uint2 make_uint2(unsigned x, unsigned y) { return {x, y}; }
inline uint3 make_uint3(unsigned x, unsigned y, unsigned z) { return {x, y, z}; }
inline uint4 make_uint4(unsigned x, unsigned y, unsigned z, unsigned w) { return {x, y, z, w}; }
inline uchar3 make_uchar3(unsigned char x, unsigned char y, unsigned char z) { return {x, y, z}; }
inline uchar4 make_uchar4(unsigned char x, unsigned char y, unsigned char z, unsigned char w) {
  return {x, y, z, w};
}

// Built-in indices (one set per host thread running a kernel body).
inline thread_local uint3 threadIdx = {0, 0, 0};
inline thread_local uint3 blockIdx = {0, 0, 0};
inline thread_local dim3 blockDim = dim3(1, 1, 1);
inline thread_local dim3 gridDim = dim3(1, 1, 1);

// Device intrinsics with their IEEE / rounding-mode semantics.
inline unsigned int __float2uint_rd(float x) { return (unsigned int)std::floor(x); }
inline int __float2int_rd(float x) { return (int)std::floor(x); }
inline int __float2int_rn(float x) { return (int)std::nearbyint(x); }
inline float __expf(float x) { return std::exp(x); }
inline float __fdividef(float a, float b) { return a / b; }
inline void __syncthreads() {}

// Atomics (GCC builtins: correct when kernel bodies run on several threads).
inline int atomicCAS(int* a, int cmp, int val) {
  __atomic_compare_exchange_n(a, &cmp, val, false, __ATOMIC_SEQ_CST, __ATOMIC_SEQ_CST);
  return cmp;
}
inline unsigned int atomicCAS(unsigned int* a, unsigned int cmp, unsigned int val) {
  __atomic_compare_exchange_n(a, &cmp, val, false, __ATOMIC_SEQ_CST, __ATOMIC_SEQ_CST);
  return cmp;
}
inline int atomicAdd(int* a, int v) { return __atomic_fetch_add(a, v, __ATOMIC_SEQ_CST); }
inline unsigned int atomicAdd(unsigned int* a, unsigned int v) {
  return __atomic_fetch_add(a, v, __ATOMIC_SEQ_CST);
}
inline int atomicSub(int* a, int v) { return __atomic_fetch_sub(a, v, __ATOMIC_SEQ_CST); }
inline unsigned int atomicSub(unsigned int* a, unsigned int v) {
  return __atomic_fetch_sub(a, v, __ATOMIC_SEQ_CST);
}
inline float atomicAdd(float* a, float v) {
  unsigned int* u = reinterpret_cast<unsigned int*>(a);
  unsigned int old = __atomic_load_n(u, __ATOMIC_SEQ_CST), nv;
  do {
    float f;
    std::memcpy(&f, &old, 4);
    f += v;
    std::memcpy(&nv, &f, 4);
  } while (!__atomic_compare_exchange_n(u, &old, nv, false, __ATOMIC_SEQ_CST, __ATOMIC_SEQ_CST));
  float r;
  std::memcpy(&r, &old, 4);
  return r;
}

// Runtime API subset: managed memory is zeroed host memory.
typedef enum cudaError { cudaSuccess = 0, cudaErrorMemoryAllocation = 2 } cudaError_t;
enum cudaMemcpyKind {
  cudaMemcpyHostToHost = 0,
  cudaMemcpyHostToDevice = 1,
  cudaMemcpyDeviceToHost = 2,
  cudaMemcpyDeviceToDevice = 3,
  cudaMemcpyDefault = 4
};
typedef void* cudaStream_t;
inline cudaError_t cudaMallocManagedRaw(void** p, size_t n) {
  *p = std::calloc(1, n ? n : 1);
  return *p ? cudaSuccess : cudaErrorMemoryAllocation;
}
template <class T>
inline cudaError_t cudaMallocManaged(T** p, size_t n, unsigned int = 1) {
  return cudaMallocManagedRaw(reinterpret_cast<void**>(p), n);
}
template <class T>
inline cudaError_t cudaMalloc(T** p, size_t n) {
  return cudaMallocManagedRaw(reinterpret_cast<void**>(p), n);
}
inline cudaError_t cudaFree(void* p) {
  std::free(p);
  return cudaSuccess;
}
inline cudaError_t cudaMemset(void* p, int v, size_t n) {
  std::memset(p, v, n);
  return cudaSuccess;
}
inline cudaError_t cudaMemcpy(void* d, const void* s, size_t n, cudaMemcpyKind) {
  std::memmove(d, s, n);
  return cudaSuccess;
}
inline cudaError_t cudaDeviceSynchronize() { return cudaSuccess; }
inline cudaError_t cudaSetDevice(int) { return cudaSuccess; }
inline cudaError_t cudaGetLastError() { return cudaSuccess; }
inline const char* cudaGetErrorString(cudaError_t) { return "cuda shim"; }

namespace dynref {
inline int& nthreads() {
  static int n = 1;
  return n;
}
// The photometric weight of buildNLSKernel.  The reference hard-codes
// `float color_weight = 0.0f;` (gnSolver.cu:180); build_ref.sh rewrites
// that one declaration to read this value, so the golden generator can run
// the kernel's colour term at a nonzero weight.  Default 0: unchanged.
inline float& color_weight() {
  static float w = 0.0f;
  return w;
}
template <class F>
struct Launcher {
  F f;
  template <class... A>
  void operator()(A&&... a) const {
    const int n = nthreads();
    if (n <= 1) {
      blockIdx = {0, 0, 0};
      gridDim = dim3(1, 1, 1);
      f(a...);
      return;
    }
    std::vector<std::thread> th;
    for (int t = 0; t < n; ++t)
      th.emplace_back([&, t]() {
        blockIdx = {(unsigned)t, 0, 0};
        threadIdx = {0, 0, 0};
        blockDim = dim3(1, 1, 1);
        gridDim = dim3((unsigned)n, 1, 1);
        f(a...);
      });
    for (auto& x : th) x.join();
  }
};
template <class F>
Launcher<F> make_launcher(F f) {
  return Launcher<F>{f};
}
}  // namespace dynref
#define DYNREF_LAUNCH(K) ::dynref::make_launcher(&K)

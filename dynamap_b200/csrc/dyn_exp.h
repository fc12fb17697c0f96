// dyn_exp.h -- single-precision exp for the bilateral range weight, written
// so that the CUDA kernel and the CPU oracle evaluate it with the identical
// sequence of IEEE operations (bit-identical results on both).
//
// Method (Cody and Waite range reduction): x = k ln2 + r with k = rint(x /
// ln2), r computed with ln2 split into a 12-bit-exact high part and a low
// part so that k*hi is exact; exp(r), |r| <= ln2/2, by its Taylor series to
// degree 7 (truncation error below 6e-9 relative, under half a float ulp)
// in Horner form with fused multiply-adds; the result times 2^k, one IEEE
// multiplication by a power of two built from its bits (exact unless the
// product is subnormal, where it rounds once: the correctly rounded
// ldexpf(p, k)).  Inputs below -87 return 0 (float underflow).
#pragma once

#ifdef __CUDACC__
#define DYN_HD __host__ __device__ inline
#else
#define DYN_HD inline
#endif
#include <cmath>
#include <cstdint>
#include <cstring>

namespace dyn {

// 2^k for -126 <= k <= 127 (a normal float), exactly.
DYN_HD float pow2i(int k) {
#ifdef __CUDA_ARCH__
  return __int_as_float((k + 127) << 23);
#else
  const uint32_t u = (uint32_t)(k + 127) << 23;
  float f;
  std::memcpy(&f, &u, sizeof f);
  return f;
#endif
}

DYN_HD float dyn_expf(float x) {
  if (!(x >= -87.0f)) return 0.0f;
  if (x > 88.0f) x = 88.0f;
  const float log2e = 1.44269504088896341f;
  const float ln2_hi = 0.693145751953125f;        // 0x3F317200: low 12 bits 0
  const float ln2_lo = 1.42860682030941723e-6f;   // ln 2 - ln2_hi
  float k = rintf(x * log2e);
  float r = fmaf(-k, ln2_hi, x);
  r = fmaf(-k, ln2_lo, r);
  float p = 1.98412698412698413e-4f;              // 1/7!
  p = fmaf(p, r, 1.38888888888888889e-3f);        // 1/6!
  p = fmaf(p, r, 8.33333333333333333e-3f);        // 1/5!
  p = fmaf(p, r, 4.16666666666666667e-2f);        // 1/4!
  p = fmaf(p, r, 1.66666666666666667e-1f);        // 1/3!
  p = fmaf(p, r, 0.5f);                           // 1/2!
  p = fmaf(p, r, 1.0f);
  p = fmaf(p, r, 1.0f);
  return p * pow2i((int)k);  // |x| <= 88: -126 <= k <= 127
}

// Bilateral range weight exp(-(x^2)/(2 sigma^2)) / (2 pi sigma^2) given
// inv2s2 = 1/(2 sigma^2) and norm = 1/(2 pi sigma^2) (both precomputed in
// double and rounded to float).
DYN_HD float range_weight(float x, float inv2s2, float norm) {
  return dyn_expf(-(x * x) * inv2s2) * norm;
}

}  // namespace dyn

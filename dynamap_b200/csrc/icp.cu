// icp.cu -- normal equations of projective point-to-plane (+photometric) ICP
// and the Gauss-Newton step, on the device.
//
// Reference: buildNLSKernel (include/solver/gnSolver/gnSolver.cu:26-196) and
// gnSolver::solve (:317-438).  The reference adds 42 FP32 atomics per
// correspondence into one 6x6 system and round-trips to the host (Eigen LDLT)
// every iteration.  Here each thread accumulates its pixels' 21 upper-
// triangle JtJ terms, 6 Jtr terms, r^2 and a count in registers (FP64 sums
// of the FP32 terms; compensated FP32 sums in the mixed form), the block
// reduces them with warp shuffles into a partial per pixel tile, and the
// tiles' partials are summed in FP64 in tile order -- a fixed reduction
// order, so results are run-to-run deterministic and do not depend on the
// grid -- before the GN update (scale by 1/max(A), damping, 6x6 LDL^T,
// convergence test) and the SE(3) exponential for the next iteration, in
// FP64, with no host round trip.  Per frame this runs either as one chained
// launch per iteration (the last block to finish a level's tiles updates
// the solver) or as one persistent cooperative launch for all levels and
// iterations (below); both give the same bits.
#include "icp.cuh"

#include <algorithm>
#include <mutex>

#include "sessdev.cuh"

namespace dyn {

namespace {

__device__ inline bool normal_ok(float4 n) {
  if (isnan(n.x) || isnan(n.y) || isnan(n.z)) return false;
  return !(n.x == 0.0f && n.y == 0.0f && n.z == 0.0f);
}

// Per-thread sums of the per-pixel terms.  The FP32 form adds each pixel's
// FP32 terms in FP64 (as the oracle does), so that its normal equations
// differ from the oracle's only by the order of FP64 additions.  The mixed
// form (KAHAN) sums a thread's few pixels in FP32 by fused multiply-adds;
// from the warp sums on, its sums are compensated pairs (block_reduce).
struct Acc {
  double d[kIcpVals];  // FP64 sums (kahan == 0)
  float v[kIcpVals];   // FP32 sums (kahan != 0)
};

__device__ inline void acc_add(Acc& a, int k, float x) { a.d[k] += (double)x; }

// Per-pixel terms of buildNLSKernel (gnSolver.cu:55-194) for source pixel
// idx; the reference's unchecked projection is bounded (z > 0, inside the
// image) and photometric gradient taps outside the image read the centre.
// Three steps, so that a thread can issue the loads of several pixels
// before it waits on any: the source pixel's depth and normal, its
// projection into the target, the target's depth, normal and intensities.
struct PixSrc {
  float d;
  float4 n;
};
struct PixProj {
  F3 p;        // source point in the target frame
  float4 sn;   // source normal
  int index;   // target pixel
  int px, py;
};
struct PixTgt {
  float td;
  float4 tn;
  float ic, il, iu, si;  // photometric taps (colour weight != 0)
};

__device__ inline PixSrc load_src(const IcpLevel& L, int idx) {
  PixSrc a;
  a.d = L.sd[idx];
  a.n = L.sn[idx];
  return a;
}

// Pixel (u, v) of index idx in an image of 'cols' columns, exactly: a
// reciprocal estimate of the row (relative error a few 2^-24, so under one
// row off for images of up to 2^26 pixels) corrected by one step.
__device__ inline void pixel_uv(int idx, int cols, int& u, int& v) {
  v = __float2int_rz(__int2float_rn(idx) * __fdividef(1.0f, (float)cols));
  u = idx - v * cols;
  if (u < 0) {
    --v;
    u += cols;
  } else if (u >= cols) {
    ++v;
    u -= cols;
  }
}

// getPoint3d and Project (utils.h:104-119) by fused multiply-adds and
// approximate division: the mixed form's projective association.
__device__ inline F3 point3d_fast(int u, int v, float d, const DSensor& s) {
  return f3(__fdividef(((float)u - s.cx) * d, s.fx), __fdividef(((float)v - s.cy) * d, s.fy), d);
}
__device__ inline bool project_fast(F3 p, const DSensor& s, int* px, int* py) {
  const float rz = __fdividef(1.0f, p.z);
  const float x = __fmaf_rn(s.fx * p.x, rz, s.cx), y = __fmaf_rn(s.fy * p.y, rz, s.cy);
  if (!(fabsf(x) < 2e9f) || !(fabsf(y) < 2e9f)) return false;
  *px = (int)roundf(x);
  *py = (int)roundf(y);
  return true;
}
__device__ inline F3 xform_fma_icp(const M4f& T, F3 v) {
  return f3(__fmaf_rn(T.m[0], v.x, __fmaf_rn(T.m[1], v.y, __fmaf_rn(T.m[2], v.z, T.m[3]))),
            __fmaf_rn(T.m[4], v.x, __fmaf_rn(T.m[5], v.y, __fmaf_rn(T.m[6], v.z, T.m[7]))),
            __fmaf_rn(T.m[8], v.x, __fmaf_rn(T.m[9], v.y, __fmaf_rn(T.m[10], v.z, T.m[11]))));
}

// FAST: the mixed form (fused multiply-adds, approximate division); else
// the reference's expressions with IEEE rounding.
template <bool FAST>
__device__ inline bool project_src(const IcpLevel& L, const IcpParams& P, const M4f& T, int idx,
                                   const PixSrc& a, PixProj& q) {
  const DSensor& s = L.s;
  if (a.d < P.dmin || a.d > P.dmax) return false;
  if (!normal_ok(a.n)) return false;
  int u, v;
  pixel_uv(idx, s.cols, u, v);
  F3 p = FAST ? xform_fma_icp(T, point3d_fast(u, v, a.d, s)) : xform(T, point3d_uv(u, v, a.d, s));
  if (!(p.z > 0.0f)) return false;
  int px, py;
  if (!(FAST ? project_fast(p, s, &px, &py) : project(p, s, &px, &py))) return false;
  if (px < 0 || py < 0 || px >= s.cols || py >= s.rows) return false;
  q.p = p;
  q.sn = a.n;
  q.index = py * s.cols + px;
  q.px = px;
  q.py = py;
  return true;
}

__device__ inline PixTgt load_tgt(const IcpLevel& L, const IcpParams& P, const PixProj& q,
                                  int idx) {
  PixTgt t;
  t.td = L.td[q.index];
  t.tn = L.tn[q.index];
  if (P.cw != 0.0f) {
    const int il = q.px >= 1 ? q.index - 1 : q.index;
    const int iu = q.py >= 1 ? q.index - L.s.cols : q.index;
    t.ic = L.ti[q.index];
    t.il = L.ti[il];
    t.iu = L.ti[iu];
    t.si = L.si[idx];
  }
  return t;
}

// The mixed form's terms of one pixel (the same terms as below, by fused
// multiply-adds: b_k = cn_k (pq . n), the reference's three-product sum in
// exact arithmetic) added into FP32 per-thread sums.
__device__ inline void accumulate_mixed(const IcpParams& P, const F3 p, const F3 n, const F3 pq,
                                        const PixTgt& t, Acc& a) {
  const F3 c = cross3(p, n);
  const float cn[6] = {c.x, c.y, c.z, n.x, n.y, n.z};
  const float r = __fmaf_rn(pq.x, n.x, __fmaf_rn(pq.y, n.y, __fmul_rn(pq.z, n.z)));
  if (P.cw != 0.0f) {
    const float gx = (t.ic - t.il) * 0.5f, gy = (t.ic - t.iu) * 0.5f;
    const float Jc[6] = {-gy * p.z, gx * p.z, __fmaf_rn(gy, p.x, -gx * p.y), gx, gy, 0.0f};
    const float e = t.ic - t.si;
    const float w1 = 1.0f - P.cw;
    float wcn[6], cj[6];
#pragma unroll
    for (int i = 0; i < 6; ++i) {
      wcn[i] = w1 * cn[i];
      cj[i] = P.cw * Jc[i];
    }
    int u = 0;
#pragma unroll
    for (int i = 0; i < 6; ++i)
#pragma unroll
      for (int j = i; j < 6; ++j, ++u)
        a.v[u] = __fmaf_rn(wcn[i], cn[j], __fmaf_rn(cj[i], Jc[j], a.v[u]));
#pragma unroll
    for (int k = 0; k < 6; ++k)
      a.v[21 + k] = __fmaf_rn(-wcn[k], r, __fmaf_rn(-cj[k], e, a.v[21 + k]));
  } else {
    int u = 0;
#pragma unroll
    for (int i = 0; i < 6; ++i)
#pragma unroll
      for (int j = i; j < 6; ++j, ++u) a.v[u] = __fmaf_rn(cn[i], cn[j], a.v[u]);
#pragma unroll
    for (int k = 0; k < 6; ++k) a.v[21 + k] = __fmaf_rn(-cn[k], r, a.v[21 + k]);
  }
  a.v[27] = __fmaf_rn(r, r, a.v[27]);
  a.v[28] = __fadd_rn(a.v[28], 1.0f);
}

template <bool KAHAN>
__device__ inline void accumulate(const IcpLevel& L, const IcpParams& P, const PixProj& q,
                                  const PixTgt& t, Acc& a) {
  const DSensor& s = L.s;
  if (t.td < P.dmin || t.td > P.dmax) return;
  if (!normal_ok(t.tn)) return;
  const F3 p = q.p;
  F3 n = f3(t.tn.x, t.tn.y, t.tn.z);
  float cosT = dot3(n, f3(q.sn.x, q.sn.y, q.sn.z));
  F3 qq = KAHAN ? point3d_fast(q.px, q.py, t.td, s) : point3d_uv(q.px, q.py, t.td, s);
  if (!(fabsf(cosT) > P.cos_thr)) return;
  F3 pq = p - qq;
  if (KAHAN) {
    accumulate_mixed(P, p, n, pq, t, a);
    return;
  }
  F3 c = cross3(p, n);
  float cn[6] = {c.x, c.y, c.z, n.x, n.y, n.z};
  float b[6];
#pragma unroll
  for (int k = 0; k < 6; ++k)
    b[k] = pq.x * (cn[k] * n.x) + pq.y * (cn[k] * n.y) + pq.z * (cn[k] * n.z);
  float r = dot3(pq, n);
  if (P.cw != 0.0f) {
    // gnSolver.cu:137-190: J_c = grad(I_t)(1x3) * [-p^ | I](3x6)
    float gx = (t.ic - t.il) / 2.0f;
    float gy = (t.ic - t.iu) / 2.0f;
    float Jc[6] = {gx * 0.0f + gy * (-p.z), gx * p.z + gy * 0.0f, gx * (-p.y) + gy * p.x,
                   gx, gy, 0.0f};
    float e = t.ic - t.si;
    float w1 = 1.0f - P.cw;
    int u = 0;
#pragma unroll
    for (int i = 0; i < 6; ++i)
#pragma unroll
      for (int j = i; j < 6; ++j) acc_add(a, u++, w1 * (cn[i] * cn[j]) + (P.cw * Jc[i]) * Jc[j]);
#pragma unroll
    for (int k = 0; k < 6; ++k) acc_add(a, 21 + k, -(w1 * b[k] + (P.cw * Jc[k]) * e));
  } else {
    int u = 0;
#pragma unroll
    for (int i = 0; i < 6; ++i)
#pragma unroll
      for (int j = i; j < 6; ++j) acc_add(a, u++, cn[i] * cn[j]);
#pragma unroll
    for (int k = 0; k < 6; ++k) acc_add(a, 21 + k, -b[k]);
  }
  acc_add(a, 27, r * r);
  acc_add(a, 28, 1.0f);
}

template <bool KAHAN>
__device__ inline void pixel_terms(const IcpLevel& L, const IcpParams& P, const M4f& T,
                                   int idx, Acc& a) {
  PixProj q;
  if (!project_src<KAHAN>(L, P, T, idx, load_src(L, idx), q)) return;
  accumulate<KAHAN>(L, P, q, load_tgt(L, P, q, idx), a);
}

// Two pixels with their loads issued together (source, then target), then
// added in order: the same sums as pixel_terms on i0, then on i1.
template <bool KAHAN>
__device__ inline void pixel_pair(const IcpLevel& L, const IcpParams& P, const M4f& T, int i0,
                                  int i1, int n, Acc& a) {
  const bool v0 = i0 < n, v1 = i1 < n;
  PixSrc a0, a1;
  if (v0) a0 = load_src(L, i0);
  if (v1) a1 = load_src(L, i1);
  PixProj q0, q1;
  const bool ok0 = v0 && project_src<KAHAN>(L, P, T, i0, a0, q0);
  const bool ok1 = v1 && project_src<KAHAN>(L, P, T, i1, a1, q1);
  PixTgt t0, t1;
  if (ok0) t0 = load_tgt(L, P, q0, i0);
  if (ok1) t1 = load_tgt(L, P, q1, i1);
  if (ok0) accumulate<KAHAN>(L, P, q0, t0, a);
  if (ok1) accumulate<KAHAN>(L, P, q1, t1, a);
}

// ---- block and tile sums
// The FP32 form adds in FP64 throughout.  The mixed form keeps the normal
// equations in FP32 up to the solve: a compensated pair (s, c) -- value
// s + c, c the rounding error carried along -- is added with Knuth's
// two-sum at every step (thread, warp shuffles, warps of a block, tiles),
// and only the level's total becomes FP64 for the 6x6 solve.  A pair is
// stored in a double-sized slot as two floats.
__device__ inline void two_sum(float a, float b, float& s, float& e) {
  s = __fadd_rn(a, b);
  const float ap = __fsub_rn(s, b), bp = __fsub_rn(s, ap);
  e = __fadd_rn(__fsub_rn(a, ap), __fsub_rn(b, bp));
}
__device__ inline void pair_add(float& s, float& c, float s2, float c2) {
  float e;
  two_sum(s, s2, s, e);
  c = __fadd_rn(__fadd_rn(c, c2), e);
}
__device__ inline double pack_pair(float s, float c) {
  return __longlong_as_double((long long)(((unsigned long long)__float_as_uint(c) << 32) |
                                          (unsigned long long)__float_as_uint(s)));
}
__device__ inline void unpack_pair(double d, float& s, float& c) {
  const unsigned long long u = (unsigned long long)__double_as_longlong(d);
  s = __uint_as_float((unsigned)(u & 0xffffffffull));
  c = __uint_as_float((unsigned)(u >> 32));
}

// Block sum of the 29 accumulators in a fixed order; result in red[0..28]
// (shared) after the call: FP64 values, or packed compensated pairs (KAHAN).
// The warp sum is a halving exchange over 32 slots (values 29..31 zero):
// at offset o every lane keeps the half of its remaining slots that its
// bit o selects, sends the other half to lane ^ o and adds what that lane
// sent; after offsets 16, 8, 4, 2, 1 lane l holds the warp's total of value
// l.  31 exchanges per lane instead of 29 x 5 for a butterfly per value.
template <bool KAHAN>
__device__ inline void block_reduce(const Acc& a, double* red /*[8][29]*/) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (KAHAN) {
    float s[32], c[32];
#pragma unroll
    for (int k = 0; k < kIcpVals; ++k) {
      s[k] = a.v[k];
      c[k] = 0.0f;
    }
#pragma unroll
    for (int k = kIcpVals; k < 32; ++k) s[k] = c[k] = 0.0f;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const bool up = (lane & o) != 0;
#pragma unroll
      for (int k = 0; k < o; ++k) {
        const float ks = up ? s[k + o] : s[k], kc = up ? c[k + o] : c[k];
        const float gs = up ? s[k] : s[k + o], gc = up ? c[k] : c[k + o];
        const float rs = __shfl_xor_sync(0xffffffffu, gs, o);
        const float rc = __shfl_xor_sync(0xffffffffu, gc, o);
        s[k] = ks;
        c[k] = kc;
        pair_add(s[k], c[k], rs, rc);
      }
    }
    if (lane < kIcpVals) red[warp * kIcpVals + lane] = pack_pair(s[0], c[0]);
  } else {
    double s[32];
#pragma unroll
    for (int k = 0; k < kIcpVals; ++k) s[k] = a.d[k];
#pragma unroll
    for (int k = kIcpVals; k < 32; ++k) s[k] = 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const bool up = (lane & o) != 0;
#pragma unroll
      for (int k = 0; k < o; ++k) {
        const double keep = up ? s[k + o] : s[k], give = up ? s[k] : s[k + o];
        s[k] = keep + __shfl_xor_sync(0xffffffffu, give, o);
      }
    }
    if (lane < kIcpVals) red[warp * kIcpVals + lane] = s[0];
  }
  __syncthreads();
  if (threadIdx.x < kIcpVals) {
    if (KAHAN) {
      float sv = 0.0f, sc = 0.0f;
      for (int w = 0; w < kIcpThreads / 32; ++w) {
        float s2, c2;
        unpack_pair(red[w * kIcpVals + threadIdx.x], s2, c2);
        pair_add(sv, sc, s2, c2);
      }
      red[threadIdx.x] = pack_pair(sv, sc);  // row 0 reused: each thread its own column
    } else {
      double sum = 0.0;
      for (int w = 0; w < kIcpThreads / 32; ++w) sum += red[w * kIcpVals + threadIdx.x];
      red[threadIdx.x] = sum;
    }
  }
  __syncthreads();
}

// Sum of the per-tile (or per-block) partials in a fixed order: thread
// (g, k) of 8 x 29 sums value k of rows g, g + 8, g + 16, ... (all 29
// values' loads in flight at once, coalesced along k), then thread k adds
// the 8 group sums in group order.  'scratch' is 8 x 29 doubles of shared
// memory; out[29] (shared) receives FP64 values (a compensated pair's
// s + c in the KAHAN form).
template <bool KAHAN>
__device__ inline void final_reduce(const double* __restrict__ partials, int nblocks,
                                    double* out, double* scratch) {
  constexpr int kGroups = kIcpThreads / 32;  // 8: scratch is the block-reduce array
  static_assert(kGroups * kIcpVals <= kIcpThreads, "one thread per (group, value)");
  const int t = threadIdx.x;
  if (t < kGroups * kIcpVals) {
    const int g = t / kIcpVals, k = t - g * kIcpVals;
    if (KAHAN) {
      float sv = 0.0f, sc = 0.0f;
#pragma unroll 4
      for (int b = g; b < nblocks; b += kGroups) {
        float s2, c2;
        unpack_pair(__ldcg(partials + (size_t)b * kIcpVals + k), s2, c2);
        pair_add(sv, sc, s2, c2);
      }
      scratch[g * kIcpVals + k] = pack_pair(sv, sc);
    } else {
      double sum = 0.0;
#pragma unroll 4
      for (int b = g; b < nblocks; b += kGroups) sum += __ldcg(partials + (size_t)b * kIcpVals + k);
      scratch[g * kIcpVals + k] = sum;
    }
  }
  __syncthreads();
  if (t < kIcpVals) {
    if (KAHAN) {
      float sv = 0.0f, sc = 0.0f;
#pragma unroll
      for (int g = 0; g < kGroups; ++g) {
        float s2, c2;
        unpack_pair(scratch[g * kIcpVals + t], s2, c2);
        pair_add(sv, sc, s2, c2);
      }
      out[t] = (double)sv + (double)sc;  // FP64 from here on: the 6x6 solve
    } else {
      double sum = 0.0;
#pragma unroll
      for (int g = 0; g < kGroups; ++g) sum += scratch[g * kIcpVals + t];
      out[t] = sum;
    }
  }
  __syncthreads();
}

// ---- FP64 6x6 algebra (one thread) --------------------------------------
// The 6x6 system lives in registers: every loop below has compile-time
// bounds and is unrolled, so no array is indexed at run time (a run-time
// index would put the arrays in local memory and make each dependent step
// of the one-thread solve wait on an L1 round trip).  The lower triangle is
// kept packed, row i at tri(i, 0) (the system is symmetric; the
// factorisation reads only the lower triangle).
__host__ __device__ constexpr int tri(int i, int j) { return i * (i + 1) / 2 + j; }

// LDL^T of a symmetric positive definite 6x6 in place (stands in for
// Eigen's A.ldlt().solve(b), gnSolver.cu:439-442): column j gives the pivot
// D[j] = A[j][j] - sum_k L[j][k]^2 D[k] and L[i][j] = (A[i][j] - sum_k
// L[i][k] L[j][k] D[k]) / D[j], each sum in increasing k; then forward
// substitution, division by D, back substitution.  L overwrites the strict
// lower triangle of a, D its diagonal.  Each pivot's reciprocal is taken
// once and multiplies (one FP64 division per column instead of one per
// entry: the one-thread solve sits between every two ICP iterations).
// Returns false on a zero pivot.
__device__ __forceinline__ bool ldlt6(double (&a)[21], const double (&b)[6], double (&x)[6]) {
  double rd[6];  // 1 / D[j]
  // triangular bounds are written as guards on fixed-length loops, so that
  // every loop has a constant trip count and unrolls completely
#pragma unroll
  for (int j = 0; j < 6; ++j) {
    double s = a[tri(j, j)];
#pragma unroll
    for (int k = 0; k < 6; ++k)
      if (k < j) s -= a[tri(j, k)] * a[tri(j, k)] * a[tri(k, k)];
    a[tri(j, j)] = s;
    if (!(fabs(s) > 0.0)) return false;
    rd[j] = 1.0 / s;
#pragma unroll
    for (int i = 0; i < 6; ++i) {
      if (i <= j) continue;
      double t = a[tri(i, j)];
#pragma unroll
      for (int k = 0; k < 6; ++k)
        if (k < j) t -= a[tri(i, k)] * a[tri(j, k)] * a[tri(k, k)];
      a[tri(i, j)] = t * rd[j];
    }
  }
  double y[6];
#pragma unroll
  for (int i = 0; i < 6; ++i) {
    double t = b[i];
#pragma unroll
    for (int k = 0; k < 6; ++k)
      if (k < i) t -= a[tri(i, k)] * y[k];
    y[i] = t;
  }
#pragma unroll
  for (int i = 0; i < 6; ++i) y[i] *= rd[i];
#pragma unroll
  for (int i = 5; i >= 0; --i) {
    double t = y[i];
#pragma unroll
    for (int k = 0; k < 6; ++k)
      if (k > i) t -= a[tri(k, i)] * x[k];
    x[i] = t;
  }
  return true;
}

// exp of the twist matrix v2t(xi) (gnSolver.cu:443-455): rotation by
// Rodrigues' formula and translation through the SE(3) left Jacobian,
// R = I + a W + b W^2, t = (I + b W + c W^2) v, with a = sin t / t,
// b = (1 - cos t)/t^2, c = (t - sin t)/t^3 (Taylor below t = 1e-4).
__device__ __forceinline__ void se3_exp(const double* xi, double* T) {
  double w0 = xi[0], w1 = xi[1], w2 = xi[2];
  double th2 = w0 * w0 + w1 * w1 + w2 * w2, th = sqrt(th2);
  double a, b, c;
  if (th < 1e-4) {
    a = 1.0 - th2 / 6.0;
    b = 0.5 - th2 / 24.0;
    c = 1.0 / 6.0 - th2 / 120.0;
  } else {
    double sn, cs;
    sincos(th, &sn, &cs);
    a = sn / th;
    b = (1.0 - cs) / th2;
    c = (th - sn) / (th2 * th);
  }
  double W[9] = {0, -w2, w1, w2, 0, -w0, -w1, w0, 0};
  double W2[9];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      double s = 0;
      for (int k = 0; k < 3; ++k) s += W[i * 3 + k] * W[k * 3 + j];
      W2[i * 3 + j] = s;
    }
  for (int i = 0; i < 3; ++i) {
    for (int j = 0; j < 3; ++j) {
      double I = (i == j) ? 1.0 : 0.0;
      T[i * 4 + j] = I + a * W[i * 3 + j] + b * W2[i * 3 + j];
    }
    double V0 = (i == 0 ? 1.0 : 0.0) + b * W[i * 3 + 0] + c * W2[i * 3 + 0];
    double V1 = (i == 1 ? 1.0 : 0.0) + b * W[i * 3 + 1] + c * W2[i * 3 + 1];
    double V2 = (i == 2 ? 1.0 : 0.0) + b * W[i * 3 + 2] + c * W2[i * 3 + 2];
    T[i * 4 + 3] = V0 * xi[3] + V1 * xi[4] + V2 * xi[5];
  }
  T[12] = T[13] = T[14] = 0.0;
  T[15] = 1.0;
}

__device__ void matmul4d(const double* A, const double* B, double* C) {
  double t[16];
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) {
      double s = 0;
      for (int k = 0; k < 4; ++k) s += A[i * 4 + k] * B[k * 4 + j];
      t[i * 4 + j] = s;
    }
  for (int k = 0; k < 16; ++k) C[k] = t[k];
}

// float4x4::getInverse, utils_matrix.h:970-1086: cofactors summed in the
// reference's order, determinant from row 0, times 1/det.
__device__ void inverse4f(const float* e, float* out) {
  float inv[16];
  inv[0] = e[5] * e[10] * e[15] - e[5] * e[11] * e[14] - e[9] * e[6] * e[15] +
           e[9] * e[7] * e[14] + e[13] * e[6] * e[11] - e[13] * e[7] * e[10];
  inv[4] = -e[4] * e[10] * e[15] + e[4] * e[11] * e[14] + e[8] * e[6] * e[15] -
           e[8] * e[7] * e[14] - e[12] * e[6] * e[11] + e[12] * e[7] * e[10];
  inv[8] = e[4] * e[9] * e[15] - e[4] * e[11] * e[13] - e[8] * e[5] * e[15] +
           e[8] * e[7] * e[13] + e[12] * e[5] * e[11] - e[12] * e[7] * e[9];
  inv[12] = -e[4] * e[9] * e[14] + e[4] * e[10] * e[13] + e[8] * e[5] * e[14] -
            e[8] * e[6] * e[13] - e[12] * e[5] * e[10] + e[12] * e[6] * e[9];
  inv[1] = -e[1] * e[10] * e[15] + e[1] * e[11] * e[14] + e[9] * e[2] * e[15] -
           e[9] * e[3] * e[14] - e[13] * e[2] * e[11] + e[13] * e[3] * e[10];
  inv[5] = e[0] * e[10] * e[15] - e[0] * e[11] * e[14] - e[8] * e[2] * e[15] +
           e[8] * e[3] * e[14] + e[12] * e[2] * e[11] - e[12] * e[3] * e[10];
  inv[9] = -e[0] * e[9] * e[15] + e[0] * e[11] * e[13] + e[8] * e[1] * e[15] -
           e[8] * e[3] * e[13] - e[12] * e[1] * e[11] + e[12] * e[3] * e[9];
  inv[13] = e[0] * e[9] * e[14] - e[0] * e[10] * e[13] - e[8] * e[1] * e[14] +
            e[8] * e[2] * e[13] + e[12] * e[1] * e[10] - e[12] * e[2] * e[9];
  inv[2] = e[1] * e[6] * e[15] - e[1] * e[7] * e[14] - e[5] * e[2] * e[15] +
           e[5] * e[3] * e[14] + e[13] * e[2] * e[7] - e[13] * e[3] * e[6];
  inv[6] = -e[0] * e[6] * e[15] + e[0] * e[7] * e[14] + e[4] * e[2] * e[15] -
           e[4] * e[3] * e[14] - e[12] * e[2] * e[7] + e[12] * e[3] * e[6];
  inv[10] = e[0] * e[5] * e[15] - e[0] * e[7] * e[13] - e[4] * e[1] * e[15] +
            e[4] * e[3] * e[13] + e[12] * e[1] * e[7] - e[12] * e[3] * e[5];
  inv[14] = -e[0] * e[5] * e[14] + e[0] * e[6] * e[13] + e[4] * e[1] * e[14] -
            e[4] * e[2] * e[13] - e[12] * e[1] * e[6] + e[12] * e[2] * e[5];
  inv[3] = -e[1] * e[6] * e[11] + e[1] * e[7] * e[10] + e[5] * e[2] * e[11] -
           e[5] * e[3] * e[10] - e[9] * e[2] * e[7] + e[9] * e[3] * e[6];
  inv[7] = e[0] * e[6] * e[11] - e[0] * e[7] * e[10] - e[4] * e[2] * e[11] +
           e[4] * e[3] * e[10] + e[8] * e[2] * e[7] - e[8] * e[3] * e[6];
  inv[11] = -e[0] * e[5] * e[11] + e[0] * e[7] * e[9] + e[4] * e[1] * e[11] -
            e[4] * e[3] * e[9] - e[8] * e[1] * e[7] + e[8] * e[3] * e[5];
  inv[15] = e[0] * e[5] * e[10] - e[0] * e[6] * e[9] - e[4] * e[1] * e[10] +
            e[4] * e[2] * e[9] + e[8] * e[1] * e[6] - e[8] * e[2] * e[5];
  float det = e[0] * inv[0] + e[1] * inv[4] + e[2] * inv[8] + e[3] * inv[12];
  float detr = 1.0f / det;
  for (int i = 0; i < 16; ++i) out[i] = inv[i] * detr;
}

// gnSolver::solve's per-iteration host block (gnSolver.cu:389-415) for the
// summed system 'acc' (upper triangle row by row, then the 6 right-hand
// sides): scale by 1 / max(A), add reg * max(scaled A) / it to the
// diagonal, solve, accumulate.  The maxima run over all 36 entries in
// row-major order, as over the full symmetric matrix.  Updates inc/prev
// (the solver state's, in global or shared memory); returns true when
// converged.
__device__ __forceinline__ double max21(const double (&a)[21]) {
  double m[11];
#pragma unroll
  for (int k = 0; k < 10; ++k) m[k] = fmax(a[2 * k], a[2 * k + 1]);
  m[10] = a[20];
#pragma unroll
  for (int w = 1; w < 11; w *= 2)
#pragma unroll
    for (int k = 0; k + w < 11; k += 2 * w) m[k] = fmax(m[k], m[k + w]);
  return m[0];
}
__device__ bool gn_update(const double* acc, const IcpParams& P, int it, double* st_inc,
                          double* st_prev) {
  double a[21], b[6];
  {  // acc holds the upper triangle row by row
#pragma unroll
    for (int i = 0; i < 6; ++i)
#pragma unroll
      for (int j = 0; j < 6; ++j)
        if (j >= i) a[tri(j, i)] = acc[i * 6 - i * (i - 1) / 2 + (j - i)];
  }
#pragma unroll
  for (int k = 0; k < 6; ++k) b[k] = acc[21 + k];
  // the maxima over all 36 entries are the maxima over the 21 stored ones
  // (fmax ignores NaNs in any order), taken as a tree
  const double mx = max21(a);
  const double scaling = 1.0 / mx;
#pragma unroll
  for (int k = 0; k < 6; ++k) b[k] *= scaling;
#pragma unroll
  for (int k = 0; k < 21; ++k) a[k] *= scaling;
  const double mx2 = max21(a);
  const double alpha = (double)P.reg * mx2;
#pragma unroll
  for (int k = 0; k < 6; ++k) a[tri(k, k)] += alpha / (double)it;
  double d[6] = {0, 0, 0, 0, 0, 0};
  if (!ldlt6(a, b, d)) {
#pragma unroll
    for (int k = 0; k < 6; ++k) d[k] = __longlong_as_double(0x7ff8000000000000LL);
  }
  double inc[6], ch = 0.0;
#pragma unroll
  for (int k = 0; k < 6; ++k) {
    inc[k] = st_inc[k] + d[k];
    st_inc[k] = inc[k];
    double c = inc[k] - st_prev[k];
    ch += c * c;
  }
  bool conv = fabs(sqrt(ch)) <= (double)P.min_inc;
  if (!conv) {
#pragma unroll
    for (int k = 0; k < 6; ++k) st_prev[k] = inc[k];
  }
  return conv;
}

// Blocks of a level's chained reduction: one per tile, at most
// kIcpMaxBlocks (a block then takes several tiles).
inline __host__ __device__ int icp_grid(int n) {
  int g = icp_tiles(n);
  if (g > kIcpMaxBlocks) g = kIcpMaxBlocks;
  if (g < 1) g = 1;
  return g;
}

// The partial sums of tile 'tile' of level L into row[0..28]: each thread
// accumulates its pixels (tile * tile_px + threadIdx.x + m * 256) in
// FP32, the block adds them in FP64 in a fixed order.  Every thread of the
// block calls it; 'red' is the block's shared scratch.
template <bool KAHAN>
__device__ inline void tile_partial(const IcpLevel& L, const IcpParams& P, const M4f& T,
                                    int tile, double* red, double* __restrict__ row) {
  Acc a;
#pragma unroll
  for (int k = 0; k < kIcpVals; ++k) {
    a.v[k] = 0.0f;
    a.d[k] = 0.0;
  }
  const int n = L.s.rows * L.s.cols;
  const int tpx = icp_tile_px(n);
  const int base = tile * tpx + (int)threadIdx.x;
  if (tpx == kIcpThreads) {
    if (base < n) pixel_terms<KAHAN>(L, P, T, base, a);
  } else if (!KAHAN) {  // FP64 sums hold most registers: one pixel at a time
    for (int m = 0; m < tpx / kIcpThreads; ++m)
      if (base + m * kIcpThreads < n) pixel_terms<KAHAN>(L, P, T, base + m * kIcpThreads, a);
  } else {
    for (int m = 0; m < tpx / kIcpThreads; m += 2)
      pixel_pair<KAHAN>(L, P, T, base + m * kIcpThreads, base + (m + 1) * kIcpThreads, n, a);
  }
  block_reduce<KAHAN>(a, red);
  if (threadIdx.x < kIcpVals) row[threadIdx.x] = red[threadIdx.x];
  __syncthreads();  // red is reused by the next tile
}

// The level's total (tiles in index order), the iteration's statistics, the
// GN update and the next transform, for a solver state held at st_* (global
// memory in the chained kernels, shared memory in the persistent one).
// tot[] must be shared; the update runs on thread 0.
template <bool KAHAN>
__device__ inline void level_update(const double* __restrict__ partials, int ntiles,
                                    const IcpParams& P, int pl, int it, double* tot, double* red,
                                    double* st_inc, double* st_prev, float* st_T,
                                    int* st_converged, int* st_iters, int* st_inliers,
                                    float* st_rms) {
  final_reduce<KAHAN>(partials, ntiles, tot, red);
  if (threadIdx.x == 0) {
    st_iters[pl] = it;
    st_inliers[pl] = (int)tot[28];
    st_rms[pl] = tot[28] > 0 ? (float)sqrt(tot[27] / tot[28]) : 0.0f;
    const bool conv = gn_update(tot, P, it, st_inc, st_prev);
    *st_converged = conv ? 1 : 0;
    double Td[16];
    se3_exp(st_inc, Td);
    for (int k = 0; k < 16; ++k) st_T[k] = (float)Td[k];
  }
}

// One GN iteration of level slot pl, iteration it (1-based), block 'bid' of
// 'nb' blocks: the partial sums of the block's tiles, then -- in the last
// block to finish -- the FP64 total and the GN update (gnSolver.cu:379-415).
template <bool KAHAN>
__device__ inline void icp_iteration_body(const IcpLevel& L, const IcpParams& P, int pl, int it,
                                          IcpState* st, double* __restrict__ partials, int bid,
                                          int nb) {
  __shared__ double red[(kIcpThreads / 32) * kIcpVals];
  __shared__ M4f Ts;
  __shared__ int skip;
  if (threadIdx.x == 0) {
    int sk = (st->have_target == 0) || (it > 1 && st->converged);
    skip = sk;
  }
  if (threadIdx.x < 16) Ts.m[threadIdx.x] = st->T[threadIdx.x];
  __syncthreads();
  if (skip) return;
  // the transform stays in shared memory (registers go to the sums)
  const int ntiles = icp_tiles(L.s.rows * L.s.cols);
  for (int tile = bid; tile < ntiles; tile += nb)
    tile_partial<KAHAN>(L, P, Ts, tile, red, partials + (size_t)tile * kIcpVals);
  __threadfence();
  __shared__ unsigned int ticket;
  if (threadIdx.x == 0) ticket = atomicAdd(&st->ticket, 1u);
  __syncthreads();
  if (ticket != (unsigned)nb - 1) return;
  __threadfence();
  __shared__ double tot[kIcpVals];
  level_update<KAHAN>(partials, ntiles, P, pl, it, tot, red, st->inc, st->prev, st->T,
                      &st->converged, st->iters, st->inliers, st->rms);
  if (threadIdx.x == 0) st->ticket = 0;
}

// Programmatic dependent launch: an iteration kernel launched with the
// programmatic-serialization attribute may start while its predecessor
// still runs.  It reads only data that no kernel of the ICP chain writes
// (the session table, the level maps) before griddepcontrol.wait, which
// returns once the predecessor grid has completed and its writes are
// visible; it then lets its own successor launch.  Without the attribute
// both instructions are no-ops.
__device__ inline void wait_predecessor() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ inline void release_successor() {
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

__device__ inline IcpLevel level_of(const SessDev& S, int l) {
  IcpLevel L;
  L.sd = S.sdep[l];
  L.sn = S.snrm[l];
  L.si = S.sint[l];
  L.td = S.tdep[l];
  L.tn = S.tnrm[l];
  L.ti = S.tint[l];
  L.s = S.ls[l];
  return L;
}

// Every session of the frame in one launch (blockIdx.z); a session uses
// only the blocks of its own grid.  One instantiation per summation kind;
// sessions of the other kind return.
template <bool KAHAN>
__global__ void __launch_bounds__(kIcpThreads, 2)
    fused_icp_iteration_kernel(const SessDev* __restrict__ tab, int pl, int it) {
  const SessDev& S = tab[blockIdx.z];
  if ((S.icpp.kahan != 0) != KAHAN) return;
  if (it >= S.slot_iters[pl]) return;  // the reference runs iterations 1 .. N-1
  const int l = S.slot_level[pl];
  const int nb = icp_grid(S.ls[l].rows * S.ls[l].cols);
  if ((int)blockIdx.x >= nb) return;
  __shared__ IcpLevel L;  // shared: registers go to the sums
  if (threadIdx.x == 0) L = level_of(S, l);
  wait_predecessor();  // the solver state and partials of the previous iteration
  release_successor();
  icp_iteration_body<KAHAN>(L, S.icpp, pl, it, S.icp, S.partials, blockIdx.x, nb);
}

// ---- the persistent form: one launch walks every level and iteration
//
// A cooperative launch (all blocks resident at once) over the table: each
// session owns a run of blocks (icp_share: about its share of the tiles),
// every block keeps its session's solver state in shared memory, and one
// grid-wide barrier per iteration separates the tiles' partial sums from
// their use: after it, every block of the session adds the partials (the
// same sums, in the same order, so every block holds the same state) and
// runs the GN update itself -- no second barrier.  Iterations alternate
// between two rows of partials, so a block may start the next iteration's
// tiles while another still reads this one's.  The results are those of the
// chained kernels bit for bit (the same tiles, summed in the same order).

// Current value of the GPU's nanosecond timer.
__device__ inline unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Grid-wide barrier number k (1, 2, ...) of a launch of 'nb' blocks (the
// grid) whose barrier words (kIcpBarWords, zero at launch) are 'bar'.
// Arrivals and releases are spread over kIcpBarSpread counters and flags,
// each on its own 128-byte line: block b adds one to counter
// b % kIcpBarSpread; block 0 alone polls the counters (one thread each)
// until each holds k times its blocks, then writes k to every release
// flag; block b polls flag b % kIcpBarSpread.  So no line takes
// more than a few dozen blocks' polls beside the arrivals it counts.  Every
// wait is bounded: after kBarrierWaitNs (or once the abort word is raised)
// the block gives up, raises the abort word and returns false.
constexpr unsigned long long kBarrierWaitNs = 500000000ull;  // half a second
__device__ inline unsigned* bar_counter(unsigned* bar, int i) { return bar + 32 * i; }
__device__ inline unsigned* bar_flag(unsigned* bar, int i) {
  return bar + 32 * (kIcpBarSpread + i);
}
__device__ inline int* bar_abort(unsigned* bar) {
  return reinterpret_cast<int*>(bar + 32 * (2 * kIcpBarSpread));
}
__device__ inline bool grid_barrier(unsigned* bar, unsigned k, unsigned nb) {
  __shared__ int ok;
  const unsigned me = blockIdx.x;
  int* abort = bar_abort(bar);
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();  // this block's partial sums before its arrival
    atomicAdd(bar_counter(bar, (int)(me % kIcpBarSpread)), 1u);
  }
  if (me == 0) {  // block 0: threads 0 .. kIcpBarSpread-1 poll one counter each
    int good = 1;
    if (threadIdx.x < kIcpBarSpread) {
      const unsigned want =
          k * ((nb + kIcpBarSpread - 1 - threadIdx.x) / kIcpBarSpread);
      volatile unsigned* c = bar_counter(bar, (int)threadIdx.x);
      const unsigned long long t0 = global_ns();
      while (*c < want) {
        if (*(volatile int*)abort || global_ns() - t0 > kBarrierWaitNs) {
          good = 0;
          break;
        }
        __nanosleep(32);
      }
      __threadfence();  // the arrivals' partial sums before the release
    }
    good = __syncthreads_and(good);
    if (threadIdx.x == 0) {
      if (good)
        for (int i = 0; i < kIcpBarSpread; ++i) *(volatile unsigned*)bar_flag(bar, i) = k;
      else
        atomicExch(abort, 1);
      ok = good;
    }
  } else if (threadIdx.x == 0) {
    volatile unsigned* flag = bar_flag(bar, (int)(me % kIcpBarSpread));
    const unsigned long long t0 = global_ns();
    int good = 1;
    while (*flag < k) {
      if (*(volatile int*)abort || global_ns() - t0 > kBarrierWaitNs) {
        good = 0;
        break;
      }
      __nanosleep(64);
    }
    if (!good) atomicExch(abort, 1);
    __threadfence();  // the other blocks' partial sums after the release
    ok = good;
  }
  __syncthreads();
  return ok != 0;
}

// Blocks of a session in a persistent launch of 'budget' blocks over a table
// whose sessions have sum_tiles level-0 tiles in all.
__host__ __device__ inline int icp_share(int tiles, long long sum_tiles, int budget) {
  long long b = (long long)budget * tiles / (sum_tiles > 0 ? sum_tiles : 1);
  if (b > tiles) b = tiles;
  if (b < 1) b = 1;
  return (int)b;
}

// One instantiation per summation kind: a table whose sessions sum both
// ways gets one launch per kind, each over that kind's sessions only.
template <bool KAHAN>
__global__ void __launch_bounds__(kIcpThreads, 2)
    fused_icp_persistent_kernel(const SessDev* __restrict__ tab, int n, int budget,
                                int it0, int it1, int it2, unsigned* __restrict__ bar) {
  // this block's session and its index among the session's blocks
  __shared__ int z_s, local_s, nblk_s;
  if (threadIdx.x == 0) {
    long long sum = 0;
    for (int j = 0; j < n; ++j)
      if ((tab[j].icpp.kahan != 0) == KAHAN) sum += icp_tiles(tab[j].npx);
    int first = 0, z = n - 1, nb = 1;
    for (int j = 0; j < n; ++j) {
      if ((tab[j].icpp.kahan != 0) != KAHAN) continue;
      nb = icp_share(icp_tiles(tab[j].npx), sum, budget);
      if ((int)blockIdx.x < first + nb) {
        z = j;
        break;
      }
      first += nb;
    }
    z_s = z;
    local_s = (int)blockIdx.x - first;
    nblk_s = nb;
  }
  __syncthreads();
  const SessDev& S = tab[z_s];
  const int local = local_s, nblk = nblk_s;
  const bool own = local >= 0 && local < nblk;  // spare blocks only pass the barriers
  // the session's solver state, one copy per block
  __shared__ double red[(kIcpThreads / 32) * kIcpVals];
  __shared__ double tot[kIcpVals];
  __shared__ double inc[6], prev[6];
  __shared__ M4f Tm;                      // the transform of the iteration
  __shared__ IcpLevel Ls;                 // the iteration's level
  float* const Tf = Tm.m;
  __shared__ int conv, have, iters[3], inliers[3];
  __shared__ float rms[3];
  if (threadIdx.x < 6) {
    inc[threadIdx.x] = S.icp->inc[threadIdx.x];
    prev[threadIdx.x] = S.icp->prev[threadIdx.x];
  }
  if (threadIdx.x < 16) Tf[threadIdx.x] = S.icp->T[threadIdx.x];
  if (threadIdx.x < 3) {
    iters[threadIdx.x] = S.icp->iters[threadIdx.x];
    inliers[threadIdx.x] = S.icp->inliers[threadIdx.x];
    rms[threadIdx.x] = S.icp->rms[threadIdx.x];
  }
  if (threadIdx.x == 0) {
    conv = S.icp->converged;
    have = S.icp->have_target;
  }
  __syncthreads();
  const int maxit[3] = {it0, it1, it2};
  const size_t row = (size_t)icp_tiles(S.npx) * kIcpVals;
  unsigned nbar = 0;
  int parity = 0;
  for (int pl = 0; pl < 3; ++pl)
    for (int it = 1; it < maxit[pl]; ++it) {
      const bool sess_active = it < S.slot_iters[pl] && have && !(it > 1 && conv);
      // a lone session's blocks all hold its state: once it has converged
      // (or has no target) they skip the level's remaining barriers together
      if (n == 1 && !sess_active) continue;
      const bool active = own && sess_active;
      const int l = S.slot_level[pl];
      const int ntiles = icp_tiles(S.ls[l].rows * S.ls[l].cols);
      double* part = S.partials + (size_t)parity * row;
      if (active) {
        // level and transform stay in shared memory (registers go to the sums)
        if (threadIdx.x == 0) Ls = level_of(S, l);
        __syncthreads();
        for (int tile = local; tile < ntiles; tile += nblk)
          tile_partial<KAHAN>(Ls, S.icpp, Tm, tile, red, part + (size_t)tile * kIcpVals);
      }
      ++nbar;
      if (!grid_barrier(bar, nbar, gridDim.x)) {
        if (threadIdx.x == 0) atomicExch(&S.vol.cnt->icp_timeout, 1);
        return;
      }
      if (active) {
        level_update<KAHAN>(part, ntiles, S.icpp, pl, it, tot, red, inc, prev, Tf, &conv, iters,
                            inliers, rms);
        __syncthreads();
      }
      parity ^= 1;
    }
  // the session's first block hands the state on (pose finalisation)
  if (own && local == 0) {
    if (threadIdx.x < 6) {
      S.icp->inc[threadIdx.x] = inc[threadIdx.x];
      S.icp->prev[threadIdx.x] = prev[threadIdx.x];
    }
    if (threadIdx.x < 16) S.icp->T[threadIdx.x] = Tf[threadIdx.x];
    if (threadIdx.x < 3) {
      S.icp->iters[threadIdx.x] = iters[threadIdx.x];
      S.icp->inliers[threadIdx.x] = inliers[threadIdx.x];
      S.icp->rms[threadIdx.x] = rms[threadIdx.x];
    }
    if (threadIdx.x == 0) {
      S.icp->converged = conv;
      S.icp->ticket = 0;
    }
  }
}

// A barrier self-test: the launch's blocks meet at barrier 1 expecting
// 'expect' blocks (more than were launched: a wait that cannot complete,
// which must end in the bounded timeout).
__global__ void barrier_selftest_kernel(unsigned* bar, unsigned expect) {
  grid_barrier(bar, 1u, expect);
}

// Normal equations only (stage entry point): no solver state.
template <bool KAHAN>
__global__ void __launch_bounds__(kIcpThreads)
    icp_reduce_kernel(IcpLevel L, IcpParams P, const float* __restrict__ Tdev,
                      double* __restrict__ partials, unsigned int* ticket_ctr,
                      double* __restrict__ out) {
  __shared__ double red[(kIcpThreads / 32) * kIcpVals];
  __shared__ M4f Ts;
  if (threadIdx.x < 16) Ts.m[threadIdx.x] = Tdev[threadIdx.x];
  __syncthreads();
  const M4f T = Ts;
  Acc a;
#pragma unroll
  for (int k = 0; k < kIcpVals; ++k) {
    a.v[k] = 0.0f;
    a.d[k] = 0.0;
  }
  const int n = L.s.rows * L.s.cols;
  for (int idx = blockIdx.x * kIcpThreads + threadIdx.x; idx < n;
       idx += gridDim.x * kIcpThreads)
    pixel_terms<KAHAN>(L, P, T, idx, a);
  block_reduce<KAHAN>(a, red);
  if (threadIdx.x < kIcpVals) partials[(size_t)blockIdx.x * kIcpVals + threadIdx.x] = red[threadIdx.x];
  __threadfence();
  __shared__ unsigned int ticket;
  if (threadIdx.x == 0) ticket = atomicAdd(ticket_ctr, 1u);
  __syncthreads();
  if (ticket != gridDim.x - 1) return;
  __threadfence();
  __shared__ double tot[kIcpVals];
  final_reduce<KAHAN>(partials, gridDim.x, tot, red);
  if (threadIdx.x < kIcpVals) out[threadIdx.x] = tot[threadIdx.x];
  if (threadIdx.x == 0) *ticket_ctr = 0;
}

__device__ void finish_pose(PoseState* ps) {
  for (int k = 0; k < 16; ++k) ps->posef[k] = (float)ps->pose[k];
  inverse4f(ps->posef, ps->invf);
}

// gnSolver.cu:426-430 + builder pose bookkeeping (one thread).
__device__ void pose_finalize_body(const IcpParams& P, IcpState* st, PoseState* ps) {
  ps->reset = 0;
  if (st->have_target) {
    double s = 0.0;
    for (int k = 0; k < 6; ++k) s += st->inc[k];
    bool reset = isnan(s) || isinf(s) || s >= (double)P.max_inc;
    if (reset)
      for (int k = 0; k < 6; ++k) st->inc[k] = 0.0;
    double E[16];
    se3_exp(st->inc, E);
    if (P.compose_left) matmul4d(E, ps->pose, ps->pose);
    else matmul4d(ps->pose, E, ps->pose);
    ps->reset = reset ? 1 : 0;
  } else {
    for (int k = 0; k < 3; ++k) {
      st->iters[k] = 0;
      st->inliers[k] = 0;
      st->rms[k] = 0.0f;
    }
  }
  for (int k = 0; k < 6; ++k) {
    ps->last_inc[k] = st->inc[k];
    st->inc[k] = 0.0;
    st->prev[k] = 0.0;
  }
  for (int k = 0; k < 16; ++k) st->T[k] = (k % 5 == 0) ? 1.0f : 0.0f;
  st->converged = 0;
  st->ticket = 0;
  finish_pose(ps);
}

__global__ void pose_finalize_kernel(IcpParams P, IcpState* st, PoseState* ps) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  pose_finalize_body(P, st, ps);
}

// one thread per session; bump != 0 also advances the frame counter
__global__ void fused_pose_finalize_kernel(const SessDev* __restrict__ tab, int n, int bump) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  const SessDev& S = tab[s];
  pose_finalize_body(S.icpp, S.icp, S.pose);
  if (bump) S.pose->frame += 1;
}

// SE(3) logarithm of a rigid transform T (row-major 4x4), the inverse of
// se3_exp: w from the rotation angle and axis, t = V^-1 translation with
// V^-1 = I - W/2 + (1 - a / (2 b)) / th^2 W^2 (a = sin th / th,
// b = (1 - cos th) / th^2; series below th = 1e-4).
__device__ void se3_log(const double* T, double* xi) {
  const double tr = T[0] + T[5] + T[10];
  double c = 0.5 * (tr - 1.0);
  c = c > 1.0 ? 1.0 : (c < -1.0 ? -1.0 : c);
  const double th = acos(c);
  const double vx = T[9] - T[6], vy = T[2] - T[8], vz = T[4] - T[1];
  double f;  // th / (2 sin th)
  if (th < 1e-4) f = 0.5 + th * th / 12.0;
  else f = th / (2.0 * sin(th));
  const double w0 = f * vx, w1 = f * vy, w2 = f * vz;
  double g;  // (1 - a / (2 b)) / th^2
  if (th < 1e-4) g = 1.0 / 12.0 + th * th / 720.0;
  else g = (1.0 - (sin(th) / th) / (2.0 * (1.0 - cos(th)) / (th * th))) / (th * th);
  const double W[9] = {0, -w2, w1, w2, 0, -w0, -w1, w0, 0};
  double W2[9];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      double s = 0;
      for (int k = 0; k < 3; ++k) s += W[i * 3 + k] * W[k * 3 + j];
      W2[i * 3 + j] = s;
    }
  const double t[3] = {T[3], T[7], T[11]};
  xi[0] = w0;
  xi[1] = w1;
  xi[2] = w2;
  for (int i = 0; i < 3; ++i) {
    double s = 0;
    for (int j = 0; j < 3; ++j) {
      const double Vi = (i == j ? 1.0 : 0.0) - 0.5 * W[i * 3 + j] + g * W2[i * 3 + j];
      s += Vi * t[j];
    }
    xi[3 + i] = s;
  }
}

// rel = pose^-1 * hint (hint * pose^-1 when increments compose on the
// left); the solver starts at log(rel).  Before the first target exists
// the hint becomes the pose.
__global__ void pose_hint_kernel(PoseState* ps, IcpState* st, const double* hint,
                                 int compose_left) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  if (!st->have_target) {
    for (int k = 0; k < 16; ++k) ps->pose[k] = hint[k];
    finish_pose(ps);
    return;
  }
  const double* P = ps->pose;
  double inv[16];
  for (int i = 0; i < 3; ++i) {
    for (int j = 0; j < 3; ++j) inv[i * 4 + j] = P[j * 4 + i];
    inv[i * 4 + 3] = -(P[0 * 4 + i] * P[3] + P[1 * 4 + i] * P[7] + P[2 * 4 + i] * P[11]);
  }
  inv[12] = inv[13] = inv[14] = 0.0;
  inv[15] = 1.0;
  double rel[16];
  if (compose_left) matmul4d(hint, inv, rel);
  else matmul4d(inv, hint, rel);
  double xi[6];
  se3_log(rel, xi);
  for (int k = 0; k < 6; ++k) {
    st->inc[k] = xi[k];
    st->prev[k] = xi[k];
  }
  double Td[16];
  se3_exp(xi, Td);
  for (int k = 0; k < 16; ++k) st->T[k] = (float)Td[k];
}

__global__ void pose_set_kernel(PoseState* ps, const double* pose) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  for (int k = 0; k < 16; ++k) ps->pose[k] = pose[k];
  finish_pose(ps);
}

}  // namespace

size_t icp_scratch_bytes() { return sizeof(double) * (size_t)kIcpMaxBlocks * kIcpVals; }

size_t icp_frame_scratch_bytes(size_t npx) {
  const size_t rows = 2 * (size_t)icp_tiles((int)npx) * kIcpVals * sizeof(double);
  return rows > icp_scratch_bytes() ? rows : icp_scratch_bytes();
}

int icp_persistent_capacity(int device) {
  static std::mutex mu;
  static int cap[64] = {};
  if (device < 0 || device >= 64) return 0;
  std::lock_guard<std::mutex> lk(mu);
  if (cap[device] == 0) {
    int coop = 0, sms = 0, per_sm = 0, per_k = 0;
    if (cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, device) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fused_icp_persistent_kernel<false>,
                                                      kIcpThreads, 0) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_k, fused_icp_persistent_kernel<true>,
                                                      kIcpThreads, 0) != cudaSuccess) {
      cudaGetLastError();
      coop = 0;
    }
    per_sm = std::min(per_sm, per_k);
    cap[device] = coop ? std::max(1, per_sm * sms) : -1;
  }
  return cap[device] > 0 ? cap[device] : 0;
}

int icp_persistent_grid(const int* npx, const int* kahan, int n, int budget, int* grid_k) {
  grid_k[0] = grid_k[1] = 0;
  if (budget <= 0 || n <= 0) return 0;
  for (int kind = 0; kind < 2; ++kind) {
    long long sum = 0;
    for (int j = 0; j < n; ++j)
      if ((kahan[j] != 0) == (kind == 1)) sum += icp_tiles(npx[j]);
    long long g = 0;
    for (int j = 0; j < n; ++j)
      if ((kahan[j] != 0) == (kind == 1)) g += icp_share(icp_tiles(npx[j]), sum, budget);
    if (g > budget) {
      grid_k[0] = grid_k[1] = 0;
      return 0;
    }
    grid_k[kind] = (int)g;
  }
  return grid_k[0] + grid_k[1];
}

template <bool KAHAN>
static void launch_persistent(const SessDev* tab, const BatchShape& b, cudaStream_t st) {
  // the barrier's counters, flags and abort word start at zero every launch
  cudaMemsetAsync(b.icp_bar, 0, kIcpBarWords * sizeof(unsigned), st);
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(b.icp_grid_k[KAHAN ? 1 : 0]);
  cfg.blockDim = dim3(kIcpThreads);
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  cudaLaunchKernelEx(&cfg, fused_icp_persistent_kernel<KAHAN>, tab, b.n, b.icp_budget,
                     b.max_slot_iters[0], b.max_slot_iters[1], b.max_slot_iters[2], b.icp_bar);
}

void fused_icp_persistent(const SessDev* tab, const BatchShape& b, cudaStream_t st) {
  if (b.icp_grid_k[0] > 0) launch_persistent<false>(tab, b, st);
  if (b.icp_grid_k[1] > 0) launch_persistent<true>(tab, b, st);
}

dyn_status icp_barrier_selftest(int blocks, int missing, unsigned* bar_dev, cudaStream_t st) {
  if (blocks < 1 || missing < 0) return DYN_ERR_INVALID_ARG;
  int dev = 0, sms = 0, per_sm = 0;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, barrier_selftest_kernel, 32, 0) !=
          cudaSuccess) {
    cudaGetLastError();
    return DYN_ERR_CUDA;
  }
  if (blocks > per_sm * sms) return DYN_ERR_INVALID_ARG;  // not all resident at once
  if (cudaMemsetAsync(bar_dev, 0, kIcpBarWords * sizeof(unsigned), st) != cudaSuccess)
    return DYN_ERR_CUDA;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(blocks);
  cfg.blockDim = dim3(32);
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  const cudaError_t e =
      cudaLaunchKernelEx(&cfg, barrier_selftest_kernel, bar_dev, (unsigned)(blocks + missing));
  if (e != cudaSuccess) {
    cudaGetLastError();
    return e == cudaErrorCooperativeLaunchTooLarge ? DYN_ERR_INVALID_ARG : DYN_ERR_CUDA;
  }
  int abort_h = 0;
  if (cudaMemcpyAsync(&abort_h, bar_dev + 32 * (2 * kIcpBarSpread), sizeof(int),
                      cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess)
    return DYN_ERR_CUDA;
  return abort_h ? DYN_ERR_TIMEOUT : DYN_OK;
}

void launch_pose_finalize(const IcpParams& P, IcpState* st, PoseState* ps, cudaStream_t stream) {
  pose_finalize_kernel<<<1, 32, 0, stream>>>(P, st, ps);
}

void launch_pose_hint(PoseState* ps, IcpState* st, const double* hint_dev, int compose_left,
                      cudaStream_t stream) {
  pose_hint_kernel<<<1, 32, 0, stream>>>(ps, st, hint_dev, compose_left);
}

void launch_pose_set(PoseState* ps, const double* pose_dev, cudaStream_t stream) {
  pose_set_kernel<<<1, 32, 0, stream>>>(ps, pose_dev);
}

void launch_icp_reduce_only(const IcpLevel& L, const IcpParams& P, const float* T_dev,
                            double* partials, unsigned int* ticket, double* out_dev,
                            cudaStream_t stream) {
  int g = icp_grid(L.s.rows * L.s.cols);
  if (P.kahan)
    icp_reduce_kernel<true><<<g, kIcpThreads, 0, stream>>>(L, P, T_dev, partials, ticket, out_dev);
  else
    icp_reduce_kernel<false><<<g, kIcpThreads, 0, stream>>>(L, P, T_dev, partials, ticket, out_dev);
}

void launch_icp_reduce_grid(const IcpLevel& L, const IcpParams& P, const float* T_dev,
                            double* partials, unsigned int* ticket, double* out_dev, int grid,
                            cudaStream_t stream) {
  if (P.kahan)
    icp_reduce_kernel<true><<<grid, kIcpThreads, 0, stream>>>(L, P, T_dev, partials, ticket,
                                                               out_dev);
  else
    icp_reduce_kernel<false><<<grid, kIcpThreads, 0, stream>>>(L, P, T_dev, partials, ticket,
                                                                out_dev);
}

// 'chained': launched with programmatic stream serialization, so that the
// kernel's launch and prologue overlap its predecessor (an earlier ICP
// iteration kernel, never the first of the frame, whose predecessor writes
// the level maps).
void fused_icp_iteration(const SessDev* tab, const BatchShape& b, int slot, int it, bool chained,
                         cudaStream_t st) {
  if (it >= b.max_slot_iters[slot]) return;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(icp_grid(b.max_slot_px[slot]), 1, b.n);
  cfg.blockDim = dim3(kIcpThreads);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  if (b.kahan_mask & 1) {
    cfg.numAttrs = chained ? 1 : 0;
    cudaLaunchKernelEx(&cfg, fused_icp_iteration_kernel<false>, tab, slot, it);
    chained = true;
  }
  if (b.kahan_mask & 2) {
    cfg.numAttrs = chained ? 1 : 0;
    cudaLaunchKernelEx(&cfg, fused_icp_iteration_kernel<true>, tab, slot, it);
  }
}

void fused_pose_finalize(const SessDev* tab, const BatchShape& b, int bump, cudaStream_t st) {
  fused_pose_finalize_kernel<<<(b.n + 31) / 32, 32, 0, st>>>(tab, b.n, bump);
}

}  // namespace dyn

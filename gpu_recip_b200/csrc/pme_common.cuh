// pme_common.cuh -- device math shared by the PME reciprocal-space kernels (sm_100a).
//
// Every FP32 operation that feeds the fixed-point charge grid is written with an explicit
// rounding intrinsic (__fmul_rn, __fadd_rn, __fsub_rn, __fmaf_rn) so that the compiler cannot
// contract or reorder it: each contribution q*thx*thy*thz is then the same bit pattern on every
// run and on every launch shape, and the int64 grid it accumulates into is exact.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace pme {

constexpr double kCcelec = 332.0716;          // 1/(4 pi eps0) in kcal/mol A/e^2 (CHARMM value)
constexpr double kPi = 3.14159265358979323846;
constexpr float kFixedScale = 1099511627776.0f;        // 2^40: grid fixed point
constexpr double kInvFixedScale = 1.0 / 1099511627776.0;
constexpr float kInvFixedScaleF = 1.0f / 1099511627776.0f;   // 2^-40, exact
constexpr int kMaxOrder = 8;

// Per-system geometry in the form the kernels use.
struct Geom {
  int nx, ny, nz;       // grid
  int hx;               // nx/2 + 1 (half-complex extent along x)
  float rx, ry, rz;     // reciprocal box diagonal, FP32
  float sx_hi, sy_hi, sz_hi;   // n_d * r_d as a float-float pair (hi + lo), used to map a
  float sx_lo, sy_lo, sz_lo;   // coordinate to grid units without losing its low bits
};

// Fractional coordinate of one axis in grid units: fr = n * frac(x*r + 1/2) in [0, n), split into
// the stencil origin i0 and the offset u in [0, 1].  This is the function of
// CudaPMERecip.cu:510-529 (fr = n (w - (floor(w + 0.5) - 0.5)), w = x r + 2), evaluated without
// its FP32 cancellation: t = x (s_hi + s_lo) + n/2 is formed as p + e with p = fl(x s_hi) and
// e = x s_lo + (x s_hi - p) exactly recovered with an FMA, so u carries ~1e-7 grid units of
// error instead of ~1e-5.  Non-finite or huge inputs map to i0 = 0, u = 0.
__device__ __forceinline__ void frac_coord(float x, float s_hi, float s_lo, int n, int& i0, float& u) {
  float p = __fmul_rn(x, s_hi);
  float e = __fmaf_rn(x, s_lo, __fmaf_rn(x, s_hi, -p));
  if (!(fabsf(p) < 16777216.0f)) { p = 0.0f; e = 0.0f; }
  const float fl = floorf(p);
  float f = __fsub_rn(p, fl);
  int i = (int)fl + (n >> 1);
  if (n & 1) f = __fadd_rn(f, 0.5f);
  float v = __fadd_rn(f, e);
  if (v >= 1.0f) { v = __fsub_rn(v, 1.0f); i += 1; }
  if (v < 0.0f) { v = __fadd_rn(v, 1.0f); i -= 1; }
  i %= n;
  if (i < 0) i += n;
  i0 = i;
  u = v;
}

// Cardinal B-spline weights of order P at offset u (weights of grid points i0..i0+P-1), built
// by the standard recursion from order 2 (CudaPMERecip.cu:181-208).  If dth != nullptr the
// derivatives d theta/du are taken from the order P-1 weights (CudaPMERecip.cu:150-159).
template <int P>
__device__ __forceinline__ void bspline(float u, float* th, float* dth) {
#pragma unroll
  for (int i = 0; i < P; i++) th[i] = 0.0f;
  th[0] = __fsub_rn(1.0f, u);
  th[1] = u;
#pragma unroll
  for (int k = 3; k <= P; k++) {
    if (k == P && dth != nullptr) {
      dth[0] = -th[0];
#pragma unroll
      for (int j = 1; j < P; j++) dth[j] = __fsub_rn(th[j - 1], th[j]);
    }
    const float d = 1.0f / (float)(k - 1);
    th[k - 1] = __fmul_rn(__fmul_rn(d, u), th[k - 2]);
#pragma unroll
    for (int j = 1; j <= k - 2; j++) {
      float a = __fadd_rn(u, (float)j);
      float b = __fsub_rn((float)(k - j), u);
      float hi = __fmul_rn(b, th[k - j - 1]);
      th[k - j - 1] = __fmul_rn(d, __fmaf_rn(a, th[k - j - 2], hi));
    }
    th[0] = __fmul_rn(__fmul_rn(d, __fsub_rn(1.0f, u)), th[0]);
  }
}

// One grid contribution in fixed point: round_to_nearest_even(((q thx) thy) thz * 2^40).
__device__ __forceinline__ long long fixed_contrib(float qthx, float thy, float thz) {
  float v = __fmul_rn(__fmul_rn(qthx, thy), thz);
  return __float2ll_rn(__fmul_rn(v, kFixedScale));
}

// Fixed point -> FP32 in FP32 arithmetic: v rounded once to the nearest float, then scaled by
// 2^-40, which is exact (|v| >= 1 stays far from the subnormal range).  Equal to rounding the exact
// quotient v * 2^-40 once.
__device__ __forceinline__ float fixed_to_float(long long v) {
  return __fmul_rn(__ll2float_rn(v), kInvFixedScaleF);
}

__device__ __forceinline__ int wrap_add(int i, int a, int n) {
  int r = i + a;
  return r >= n ? r - n : r;
}

}  // namespace pme

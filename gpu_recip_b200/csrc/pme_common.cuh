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
  int tric;                    // 1: triclinic box (a reciprocal matrix with off-diagonals)
  float shi[9], slo[9];        // triclinic: S[j][d] = n_d R[j][d] (index 3 j + d) as hi + lo
};

// Grid-unit coordinate t = p + e (p the leading float, e its small correction, both already
// carrying the n/2 shift of w = x r + 2 modulo n) -> stencil origin i0 and offset u in [0, 1].
// Non-finite or huge inputs map to i0 = 0, u = 0.
__device__ __forceinline__ void frac_finish(float p, float e, int n, int& i0, float& u) {
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

// Fractional coordinate of one axis in grid units: fr = n * frac(x*r + 1/2) in [0, n), split into
// the stencil origin i0 and the offset u in [0, 1].  This is the function of
// CudaPMERecip.cu:510-529 (fr = n (w - (floor(w + 0.5) - 0.5)), w = x r + 2), evaluated without
// its FP32 cancellation: t = x (s_hi + s_lo) + n/2 is formed as p + e with p = fl(x s_hi) and
// e = x s_lo + (x s_hi - p) exactly recovered with an FMA, so u carries ~1e-7 grid units of
// error instead of ~1e-5.
__device__ __forceinline__ void frac_coord(float x, float s_hi, float s_lo, int n, int& i0, float& u) {
  const float p = __fmul_rn(x, s_hi);
  const float e = __fmaf_rn(x, s_lo, __fmaf_rn(x, s_hi, -p));
  frac_finish(p, e, n, i0, u);
}

// Triclinic axis d: t = x S[0][d] + y S[1][d] + z S[2][d] in float-float.  Each product is split
// into its rounded value and exact error as in frac_coord, the three leading parts are summed with
// two error-free two-sums (Knuth), and all error terms go into e.  With S[1][d] = S[2][d] = 0 this
// is frac_coord bit for bit.
__device__ __forceinline__ void frac_coord_tric(float x, float y, float z, const float* shi,
                                                const float* slo, int d, int n, int& i0, float& u) {
  const float p0 = __fmul_rn(x, shi[d]), p1 = __fmul_rn(y, shi[3 + d]), p2 = __fmul_rn(z, shi[6 + d]);
  const float e0 = __fmaf_rn(x, slo[d], __fmaf_rn(x, shi[d], -p0));
  const float e1 = __fmaf_rn(y, slo[3 + d], __fmaf_rn(y, shi[3 + d], -p1));
  const float e2 = __fmaf_rn(z, slo[6 + d], __fmaf_rn(z, shi[6 + d], -p2));
  const float s01 = __fadd_rn(p0, p1);
  const float b01 = __fsub_rn(s01, p0);
  const float t01 = __fadd_rn(__fsub_rn(p0, __fsub_rn(s01, b01)), __fsub_rn(p1, b01));
  const float p = __fadd_rn(s01, p2);
  const float b2 = __fsub_rn(p, s01);
  const float t2 = __fadd_rn(__fsub_rn(s01, __fsub_rn(p, b2)), __fsub_rn(p2, b2));
  const float e = __fadd_rn(__fadd_rn(__fadd_rn(e0, e1), e2), __fadd_rn(t01, t2));
  frac_finish(p, e, n, i0, u);
}

// Stencil origins and offsets of one atom on all three axes (orthorhombic or triclinic box).
__device__ __forceinline__ void frac_coords(const Geom& g, float x, float y, float z, int& ix, int& iy,
                                            int& iz, float& ux, float& uy, float& uz) {
  if (!g.tric) {
    frac_coord(x, g.sx_hi, g.sx_lo, g.nx, ix, ux);
    frac_coord(y, g.sy_hi, g.sy_lo, g.ny, iy, uy);
    frac_coord(z, g.sz_hi, g.sz_lo, g.nz, iz, uz);
  } else {
    frac_coord_tric(x, y, z, g.shi, g.slo, 0, g.nx, ix, ux);
    frac_coord_tric(x, y, z, g.shi, g.slo, 1, g.ny, iy, uy);
    frac_coord_tric(x, y, z, g.shi, g.slo, 2, g.nz, iz, uz);
  }
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

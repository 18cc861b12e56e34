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
constexpr int kMaxOrder = 8;

// Per-system geometry in the form the kernels use.
struct Geom {
  int nx, ny, nz;       // grid
  int hx;               // nx/2 + 1 (half-complex extent along x)
  float rx, ry, rz;     // reciprocal box diagonal, FP32
};

// Fractional coordinate of one axis: fr = n * frac(x*r + 0.5) in [0, n); stencil origin i0 and
// offset u in [0,1).  Follows CudaPMERecip.cu:510-529 (w = x r + 2, fr = n (w - (floor(w+0.5) -
// 0.5))).  A non-finite or out-of-range fr maps to 0, so that no coordinate can index outside
// the grid.
__device__ __forceinline__ void frac_coord(float x, float r, int n, int& i0, float& u) {
  float w = __fmaf_rn(x, r, 2.0f);
  float t = __fsub_rn(floorf(__fadd_rn(w, 0.5f)), 0.5f);
  float fr = __fmul_rn((float)n, __fsub_rn(w, t));
  if (!(fr >= 0.0f && fr < (float)n)) fr = 0.0f;
  int i = (int)fr;
  i0 = i;
  u = __fsub_rn(fr, (float)i);
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

__device__ __forceinline__ float fixed_to_float(long long v) {
  return (float)((double)v * kInvFixedScale);
}

__device__ __forceinline__ int wrap_add(int i, int a, int n) {
  int r = i + a;
  return r >= n ? r - n : r;
}

}  // namespace pme

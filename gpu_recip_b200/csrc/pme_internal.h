// pme_internal.h -- host-side launch interface of the PME reciprocal-space kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "pme_common.cuh"
#include "pme_fft.cuh"

namespace pme {

// Energy/virial record layout in device memory (doubles).  Accumulated, never overwritten,
// like the reference's CudaEnergyVirial slots (CudaEnergyVirial.cu:158-167).
enum EvSlot { kEvRecip = 0, kEvSelf = 1, kEvVirial = 2, kEvCount = 11 };

// Per-axis line-FFT tiling of one pass.
struct PassTiling {
  int tx;        // lines per CTA tile
  int ny;        // threadIdx.y extent (butterfly lanes)
};

// Deterministic cross-CTA reduction scratch: per-CTA partials and a ticket counter that the
// last CTA resets.
struct ReduceScratch {
  double* partials;      // [max_blocks][8]
  unsigned int* ticket;  // one counter per reduction site
  int max_blocks;
};

// Solve parameters (CudaPMERecip.cu:1988-2012: fac = pi^2/kappa^2, piv_inv = 1/(pi V)).
struct SolveParams {
  float fac;
  float piv_inv;
  const float* bmx;   // B-spline moduli, FP32 (1/|b|^2)
  const float* bmy;
  const float* bmz;
  int calc_ev;
  double* ev;         // energy/virial record
};

enum ForceKind { kForceF32Soa = 0, kForceF32x3 = 1, kForceI64SoaAccum = 2 };

cudaError_t launch_spread(const float4* xyzq, int n, const Geom& g, int order,
                          unsigned long long* accum, cudaStream_t s);

cudaError_t launch_x_r2c(const long long* accum, float2* cgrid, const Geom& g,
                         const FftPlan1D& px, const float2* tw, const PassTiling& t,
                         cudaStream_t s);

// Complex passes along y (axis 1) or z (axis 2) of the half-complex grid [z][y][kx].
// mode: 0 forward, 1 inverse, 2 forward + solve + inverse (axis 2 only), 3 solve only (axis 2).
cudaError_t launch_c2c(float2* cgrid, const Geom& g, int axis, int mode, const FftPlan1D& plan,
                       const float2* tw, const PassTiling& t, const SolveParams* sp,
                       const ReduceScratch& rs, int rs_site, cudaStream_t s);

cudaError_t launch_x_c2r(const float2* cgrid, float* rgrid, const Geom& g, const FftPlan1D& px,
                         const float2* tw, const PassTiling& t, cudaStream_t s);

cudaError_t launch_gather(const float4* xyzq, int n, const Geom& g, int order, const float* rgrid,
                          int kind, int stride, void* force, cudaStream_t s);

cudaError_t launch_self_energy(const float4* xyzq, int n, double kappa, double* ev,
                               const ReduceScratch& rs, int rs_site, cudaStream_t s);

cudaError_t launch_fixed_to_float(const long long* accum, float* out, size_t count,
                                  cudaStream_t s);

size_t c2c_smem_bytes(int L, const PassTiling& t);
int c2c_num_blocks(const Geom& g, int axis, const PassTiling& t);

}  // namespace pme

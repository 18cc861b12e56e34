// ref_shim.h -- force-included (nvcc -include) when the reference's own CUDA sources are compiled
// for sm_100a with CUDA 12.9; measurement only.  The reference sources are not edited:
// these definitions bridge the APIs they use that current CUDA no longer provides (the last one,
// cuFFT's native in-place layout, at the end of this file).
//  - gpu_utils.h:35 defines atomicAdd(double*, double), which CUDA now declares itself: every
//    atomicAdd in the reference is renamed to atomicAdd_ref, which forwards to CUDA's for the
//    types the reference does not define itself.
//  - cufftSetCompatibilityMode and its modes were removed from cuFFT (CudaPMERecip.cu:1526-1607):
//    the call becomes a no-op that succeeds.
//  - __shfl and friends without _sync were removed for sm_70+ (CudaPMERecip.cu:805-855,
//    :1186-1196): they map to the _sync forms over the active lanes.
#pragma once
#include <cuda_runtime.h>
#include <cufft.h>

template <class T, class U>
static __device__ __forceinline__ T atomicAdd_ref(T* address, U value) {
  return atomicAdd(address, (T)value);
}
#define atomicAdd atomicAdd_ref

#define cufftSetCompatibilityMode(plan, mode) CUFFT_SUCCESS
#define CUFFT_COMPATIBILITY_NATIVE 0
#define CUFFT_COMPATIBILITY_FFTW_PADDING 0

#define __shfl(v, ...) __shfl_sync(__activemask(), v, __VA_ARGS__)
#define __shfl_xor(v, ...) __shfl_xor_sync(__activemask(), v, __VA_ARGS__)
#define __shfl_up(v, ...) __shfl_up_sync(__activemask(), v, __VA_ARGS__)
#define __shfl_down(v, ...) __shfl_down_sync(__activemask(), v, __VA_ARGS__)

// In-place R2C / C2R on unpadded grids.  The reference runs its real<->complex transforms in
// place on grids whose real rows are NOT padded (x + xsize (y + ysize z), CudaPMERecip.cu:1360,
// :2269, :2295, :2421, :2464), which the removed CUFFT_COMPATIBILITY_NATIVE mode allowed.  Current
// cuFFT reads an in-place real array as FFTW-padded rows, so those calls transform the wrong
// elements (and read the uncleared tail of the buffer).  The wrappers below keep the reference's
// calls and results: an in-place R2C/C2R first copies its input (the plan's real or complex
// element count) to a scratch buffer on the plan's stream and then runs out of place from the
// scratch into the original buffer, which gives the unpadded layout the reference expects.
// Out-of-place calls and every C2C pass through unchanged.
#include <map>

struct RefShimPlan {
  size_t real_elems = 0, cplx_elems = 0;
  cudaStream_t stream = 0;
};

inline std::map<cufftHandle, RefShimPlan>& ref_shim_plans() {
  static std::map<cufftHandle, RefShimPlan> m;
  return m;
}

// Real and half-complex element counts of a plan of `rank` dimensions n[0..rank) (last fastest).
inline void ref_shim_record(cufftHandle plan, int rank, const int* n, long long batch) {
  size_t r = 1, c = 1;
  for (int i = 0; i < rank; i++) {
    r *= (size_t)n[i];
    c *= (size_t)(i == rank - 1 ? n[i] / 2 + 1 : n[i]);
  }
  RefShimPlan& p = ref_shim_plans()[plan];
  p.real_elems = r * (size_t)batch;
  p.cplx_elems = c * (size_t)batch;
}

inline cufftResult ref_shim_plan3d(cufftHandle* plan, int nx, int ny, int nz, cufftType type) {
  const cufftResult r = cufftPlan3d(plan, nx, ny, nz, type);
  const int n[3] = {nx, ny, nz};
  if (r == CUFFT_SUCCESS) ref_shim_record(*plan, 3, n, 1);
  return r;
}

inline cufftResult ref_shim_plan_many(cufftHandle* plan, int rank, int* n, int* inembed, int istride, int idist,
                                      int* onembed, int ostride, int odist, cufftType type, int batch) {
  const cufftResult r = cufftPlanMany(plan, rank, n, inembed, istride, idist, onembed, ostride, odist, type, batch);
  if (r == CUFFT_SUCCESS) ref_shim_record(*plan, rank, n, batch);
  return r;
}

inline cufftResult ref_shim_set_stream(cufftHandle plan, cudaStream_t stream) {
  const cufftResult r = cufftSetStream(plan, stream);
  if (r == CUFFT_SUCCESS) ref_shim_plans()[plan].stream = stream;
  return r;
}

// Scratch of at least `bytes` (grows; allocated on the first transform, outside the timed steps).
inline void* ref_shim_scratch(size_t bytes) {
  static void* buf = nullptr;
  static size_t cap = 0;
  if (bytes > cap) {
    if (buf) cudaFree(buf);
    buf = nullptr;
    cap = 0;
    if (cudaMalloc(&buf, bytes) != cudaSuccess) return nullptr;
    cap = bytes;
  }
  return buf;
}

inline cufftResult ref_shim_exec_r2c(cufftHandle plan, cufftReal* idata, cufftComplex* odata) {
  if ((void*)idata != (void*)odata) return cufftExecR2C(plan, idata, odata);
  const RefShimPlan p = ref_shim_plans()[plan];
  const size_t bytes = p.real_elems * sizeof(cufftReal);
  void* s = ref_shim_scratch(bytes);
  if (!s || cudaMemcpyAsync(s, idata, bytes, cudaMemcpyDeviceToDevice, p.stream) != cudaSuccess)
    return CUFFT_INTERNAL_ERROR;
  return cufftExecR2C(plan, (cufftReal*)s, odata);
}

inline cufftResult ref_shim_exec_c2r(cufftHandle plan, cufftComplex* idata, cufftReal* odata) {
  if ((void*)idata != (void*)odata) return cufftExecC2R(plan, idata, odata);
  const RefShimPlan p = ref_shim_plans()[plan];
  const size_t bytes = p.cplx_elems * sizeof(cufftComplex);
  void* s = ref_shim_scratch(bytes);
  if (!s || cudaMemcpyAsync(s, idata, bytes, cudaMemcpyDeviceToDevice, p.stream) != cudaSuccess)
    return CUFFT_INTERNAL_ERROR;
  return cufftExecC2R(plan, (cufftComplex*)s, odata);
}

#define cufftPlan3d(plan, nx, ny, nz, type) ref_shim_plan3d(plan, nx, ny, nz, type)
#define cufftPlanMany(plan, rank, n, ie, is, id, oe, os, od, type, batch) \
  ref_shim_plan_many(plan, rank, n, ie, is, id, oe, os, od, type, batch)
#define cufftSetStream(plan, stream) ref_shim_set_stream(plan, stream)
#define cufftExecR2C(plan, idata, odata) ref_shim_exec_r2c(plan, idata, odata)
#define cufftExecC2R(plan, idata, odata) ref_shim_exec_c2r(plan, idata, odata)

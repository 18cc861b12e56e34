// ref_shim.h -- force-included (nvcc -include) when the reference's own CUDA sources are compiled
// for sm_100a with CUDA 12.9; measurement only.  The reference sources are not edited:
// these definitions bridge the four APIs they use that current CUDA no longer provides.
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

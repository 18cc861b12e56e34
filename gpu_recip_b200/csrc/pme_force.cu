// pme_force.cu -- conversion of accumulated fixed-point forces to floating point.
//
// An MD step accumulates the reciprocal force (PME_FORCE_I64_SOA_ACCUM), the direct-space and
// the 1-4 forces into one int64 SoA array at scale 2^40, and converts it once at the end of the
// step (CudaPMEForcefield.cu:514, force.convert<double>).  These kernels are that conversion:
// Force<long long>::convert<T2> (Force.cu:103-128, reduce.cu:15-53), its in-place form
// convert<double>() (Force.cu:143-157, reduce.cu:125-145) and convert_add (Force.cu:167-184,
// reduce.cu:152-170).  Each value is the int64 rounded once to the output type and scaled by
// 2^-40, which is exact, so the result is (T)v * 2^-40 bit for bit.
#include <cuda_runtime.h>

#include <cstdint>
#include <string>

#include "../../include/pme_recip.h"
#include "pme_internal.h"

using namespace pme;

namespace {

constexpr double kInvScaleD = 1.0 / 1099511627776.0;   // 2^-40, exact
constexpr float kInvScaleF = 1.0f / 1099511627776.0f;

// One thread per (atom, row): row = blockIdx.y.  in and out may be the same array (in place):
// every element is read and written by the same thread.
template <typename T>
__global__ void k_force_convert(const long long* in, int in_stride, int n, T* out, int out_stride) {
  const int row = blockIdx.y;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const long long v = in[(size_t)row * in_stride + i];
    T r;
    if (sizeof(T) == 8) r = (T)__dmul_rn(__ll2double_rn(v), kInvScaleD);
    else r = (T)__fmul_rn(__ll2float_rn(v), kInvScaleF);
    out[(size_t)row * out_stride + i] = r;
  }
}

template <typename A>
__global__ void k_force_convert_add(long long* inout, int stride, int n, const A* add, int add_stride) {
  const int row = blockIdx.y;
  double* out = reinterpret_cast<double*>(inout);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const size_t k = (size_t)row * stride + i;
    const double v = __dmul_rn(__ll2double_rn(inout[k]), kInvScaleD);
    out[k] = __dadd_rn(v, (double)add[(size_t)row * add_stride + i]);
  }
}

int conv_fail(int status, const std::string& msg) {
  set_last_error(msg.c_str());
  return status;
}

dim3 conv_grid(int n) {
  int bx = (n + 255) / 256;
  if (bx > 1184) bx = 1184;   // 8 CTAs per SM on 148 SMs; the loop covers the rest
  if (bx < 1) bx = 1;
  return dim3(bx, 3);
}

// Byte range [lo, hi) of three rows of n elements of `size` bytes with `stride`.
void rows_range(const void* p, int stride, int n, size_t size, uintptr_t* lo, uintptr_t* hi) {
  *lo = (uintptr_t)p;
  *hi = (uintptr_t)p + ((size_t)2 * stride + n) * size;
}

}  // namespace

extern "C" {

int pme_force_convert(const long long* in, int in_stride, int ncoord, void* out, int out_stride, int out_type,
                      void* stream) {
  if (ncoord < 0) return conv_fail(PME_EINVAL, "ncoord must be >= 0");
  if (out_type != PME_REAL_F32 && out_type != PME_REAL_F64) return conv_fail(PME_EINVAL, "unknown output type");
  if (ncoord == 0) return PME_OK;
  if (!in || !out) return conv_fail(PME_EINVAL, "NULL force array");
  if (in_stride < ncoord || out_stride < ncoord) return conv_fail(PME_EINVAL, "strides must be >= ncoord");
  const size_t osize = out_type == PME_REAL_F64 ? 8 : 4;
  uintptr_t ilo, ihi, olo, ohi;
  rows_range(in, in_stride, ncoord, 8, &ilo, &ihi);
  rows_range(out, out_stride, ncoord, osize, &olo, &ohi);
  const bool same = (const void*)in == out;
  if (same && (out_type != PME_REAL_F64 || out_stride != in_stride))
    return conv_fail(PME_EINVAL, "in-place conversion needs double output with the same stride");
  if (!same && olo < ihi && ilo < ohi) return conv_fail(PME_EINVAL, "input and output overlap");
  cudaStream_t s = (cudaStream_t)stream;
  if (out_type == PME_REAL_F64)
    k_force_convert<double><<<conv_grid(ncoord), 256, 0, s>>>(in, in_stride, ncoord, (double*)out, out_stride);
  else
    k_force_convert<float><<<conv_grid(ncoord), 256, 0, s>>>(in, in_stride, ncoord, (float*)out, out_stride);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return conv_fail(PME_ECUDA, std::string("force_convert: ") + cudaGetErrorString(e));
  return PME_OK;
}

int pme_force_convert_add(long long* inout, int stride, int ncoord, const void* add, int add_stride, int add_type,
                          void* stream) {
  if (ncoord < 0) return conv_fail(PME_EINVAL, "ncoord must be >= 0");
  if (add_type != PME_REAL_F32 && add_type != PME_REAL_F64) return conv_fail(PME_EINVAL, "unknown type of add");
  if (ncoord == 0) return PME_OK;
  if (!inout || !add) return conv_fail(PME_EINVAL, "NULL force array");
  if (stride < ncoord || add_stride < ncoord) return conv_fail(PME_EINVAL, "strides must be >= ncoord");
  uintptr_t ilo, ihi, alo, ahi;
  rows_range(inout, stride, ncoord, 8, &ilo, &ihi);
  rows_range(add, add_stride, ncoord, add_type == PME_REAL_F64 ? 8 : 4, &alo, &ahi);
  if (alo < ihi && ilo < ahi) return conv_fail(PME_EINVAL, "add overlaps the converted array");
  cudaStream_t s = (cudaStream_t)stream;
  if (add_type == PME_REAL_F64)
    k_force_convert_add<double><<<conv_grid(ncoord), 256, 0, s>>>(inout, stride, ncoord, (const double*)add, add_stride);
  else
    k_force_convert_add<float><<<conv_grid(ncoord), 256, 0, s>>>(inout, stride, ncoord, (const float*)add, add_stride);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return conv_fail(PME_ECUDA, std::string("force_convert_add: ") + cudaGetErrorString(e));
  return PME_OK;
}

}  // extern "C"

// recip_driver.cpp -- a C++ caller of the C ABI in include/pme_recip.h, written the way the
// reference's recip test driver uses CudaPMERecip (gpu_recip.cu:133-138): create the operator,
// clear the energy/virial record, spread, R2C, scalar sum, C2R, gather, read energy and virial;
// then the same evaluation through pme_eval_ortho (the CudaDomdecRecip::calc sequence).
//
// Input (binary, little endian): int32 natom, order, nx, ny, nz; float64 box[3], kappa;
// float32 xyzq[natom][4].  Output (binary): per sequence (staged, fused) float64 energy,
// virial[9] and float32 forces[natom][3].  Exit status 0 on success.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstdlib>
#include <vector>

#include "pme_recip.h"

#define CHECK(call)                                                                      \
  do {                                                                                   \
    int rc_ = (call);                                                                    \
    if (rc_ != PME_OK) {                                                                 \
      std::fprintf(stderr, "%s failed: %d %s\n", #call, rc_, pme_last_error_string()); \
      return 1;                                                                          \
    }                                                                                    \
  } while (0)

#define CUDA(call)                                                                        \
  do {                                                                                    \
    cudaError_t e_ = (call);                                                              \
    if (e_ != cudaSuccess) {                                                              \
      std::fprintf(stderr, "%s failed: %s\n", #call, cudaGetErrorString(e_));            \
      return 1;                                                                           \
    }                                                                                     \
  } while (0)

int main(int argc, char** argv) {
  if (argc != 3) {
    std::fprintf(stderr, "usage: %s input.bin output.bin\n", argv[0]);
    return 2;
  }
  FILE* in = std::fopen(argv[1], "rb");
  if (!in) return 2;
  int hdr[5];
  double box[3], kappa;
  if (std::fread(hdr, sizeof(int), 5, in) != 5 || std::fread(box, sizeof(double), 3, in) != 3 ||
      std::fread(&kappa, sizeof(double), 1, in) != 1)
    return 2;
  const int natom = hdr[0], order = hdr[1], nx = hdr[2], ny = hdr[3], nz = hdr[4];
  std::vector<float> xyzq((size_t)natom * 4);
  if (std::fread(xyzq.data(), sizeof(float), xyzq.size(), in) != xyzq.size()) return 2;
  std::fclose(in);

  float* d_xyzq = nullptr;
  float* d_force = nullptr;
  CUDA(cudaMalloc(&d_xyzq, xyzq.size() * sizeof(float)));
  CUDA(cudaMalloc(&d_force, (size_t)natom * 3 * sizeof(float)));
  CUDA(cudaMemcpy(d_xyzq, xyzq.data(), xyzq.size() * sizeof(float), cudaMemcpyHostToDevice));

  pme_recip* h = nullptr;
  CHECK(pme_create(nx, ny, nz, order, PME_FFT_BOX, 1, 0, nullptr, &h));
  const double recip[9] = {1.0 / box[0], 0, 0, 0, 1.0 / box[1], 0, 0, 0, 1.0 / box[2]};

  FILE* out = std::fopen(argv[2], "wb");
  if (!out) return 2;
  std::vector<float> f((size_t)natom * 3);
  for (int seq = 0; seq < 2; seq++) {
    CHECK(pme_clear_energy_virial(h));
    if (seq == 0) {   // the reference driver's staged calls
      CHECK(pme_spread_charge(h, d_xyzq, natom, recip));
      CHECK(pme_r2c_fft(h));
      CHECK(pme_scalar_sum(h, recip, kappa, 1, 1));
      CHECK(pme_c2r_fft(h));
      CHECK(pme_gather_force(h, d_xyzq, natom, recip, 1, PME_FORCE_F32X3, d_force));
    } else {          // one fused evaluation
      CHECK(pme_eval_ortho(h, recip[0], recip[4], recip[8], d_xyzq, natom, kappa, 1, 1, PME_FORCE_F32X3,
                           d_force, 1));
    }
    double e_recip = 0, e_self = 0, vir[9];
    CHECK(pme_get_energy_virial(h, &e_recip, &e_self, vir));
    CUDA(cudaMemcpy(f.data(), d_force, f.size() * sizeof(float), cudaMemcpyDeviceToHost));
    std::fwrite(&e_recip, sizeof(double), 1, out);
    std::fwrite(vir, sizeof(double), 9, out);
    std::fwrite(f.data(), sizeof(float), f.size(), out);
  }
  std::fclose(out);
  CHECK(pme_destroy(h));
  CUDA(cudaFree(d_xyzq));
  CUDA(cudaFree(d_force));
  return 0;
}

// direct_driver.cpp -- a C++ caller of the C ABI in include/pme_direct.h, written the way the
// reference's direct test driver uses CudaPMEDirectForce (gpu_direct.cu:151-233): set up the
// operator (box, kappa, roff, ron, e14fac, VDW_VSH, EWALD), the vdW parameters and types, the CHARMM
// exclusions, the 1-4 lists; clear the energy/virial record; calc_force into an int64 force array;
// read energies and virial; then calc_14_force on top.
//
// Input (binary, little endian): int32 natom, nvdwparam, nvdwparam14, nin14, nex14, ninb14;
// float64 box[3], kappa, roff, ron, e14fac; float32 xyzq[natom][4], vdwparam[nvdwparam],
// vdwparam14[nvdwparam14]; int32 vdwtype[natom], iblo14[natom], inb14[ninb14], loc2glo[natom],
// in14[nin14][3], ex14[nex14][3].  Output (binary): float64 e_vdw, e_elec, e_excl, virial[9] and
// float64 forces[natom][3] after calc_force, then the same after calc_14_force.  Exit status 0 on
// success.
#include <cuda_runtime.h>

#include <cstdio>
#include <vector>

#include "pme_direct.h"

#define CHECK(call)                                                                      \
  do {                                                                                   \
    int rc_ = (call);                                                                    \
    if (rc_ != PME_OK) {                                                                 \
      std::fprintf(stderr, "%s failed: %d %s\n", #call, rc_, pme_last_error_string()); \
      return 1;                                                                          \
    }                                                                                    \
  } while (0)

#define CUDA(call)                                                             \
  do {                                                                         \
    cudaError_t e_ = (call);                                                   \
    if (e_ != cudaSuccess) {                                                   \
      std::fprintf(stderr, "%s failed: %s\n", #call, cudaGetErrorString(e_)); \
      return 1;                                                                \
    }                                                                          \
  } while (0)

template <class T>
static bool read(FILE* f, std::vector<T>& v, size_t n) {
  v.resize(n);
  return std::fread(v.data(), sizeof(T), n, f) == n;
}

static int dump(FILE* out, pme_direct* dir, const long long* d_force, int natom, int stride) {
  double e[3], vir[9];
  CHECK(pme_direct_get_energy_virial(dir, &e[0], &e[1], &e[2], vir));   // synchronises
  std::vector<long long> h((size_t)3 * stride);
  CUDA(cudaMemcpy(h.data(), d_force, h.size() * sizeof(long long), cudaMemcpyDeviceToHost));
  std::vector<double> f((size_t)natom * 3);
  for (int i = 0; i < natom; i++)
    for (int d = 0; d < 3; d++) f[3 * (size_t)i + d] = (double)h[(size_t)d * stride + i] / 1099511627776.0;
  std::fwrite(e, sizeof(double), 3, out);
  std::fwrite(vir, sizeof(double), 9, out);
  std::fwrite(f.data(), sizeof(double), f.size(), out);
  return 0;
}

int main(int argc, char** argv) {
  if (argc != 3) {
    std::fprintf(stderr, "usage: %s input.bin output.bin\n", argv[0]);
    return 2;
  }
  FILE* in = std::fopen(argv[1], "rb");
  if (!in) return 2;
  int hdr[6];
  double set[7];
  if (std::fread(hdr, sizeof(int), 6, in) != 6 || std::fread(set, sizeof(double), 7, in) != 7) return 2;
  const int natom = hdr[0], nvdw = hdr[1], nvdw14 = hdr[2], nin14 = hdr[3], nex14 = hdr[4], ninb = hdr[5];
  std::vector<float> xyzq, vdwparam, vdwparam14;
  std::vector<int> vdwtype, iblo14, inb14, loc2glo, in14, ex14;
  if (!read(in, xyzq, (size_t)natom * 4) || !read(in, vdwparam, nvdw) || !read(in, vdwparam14, nvdw14) ||
      !read(in, vdwtype, natom) || !read(in, iblo14, natom) || !read(in, inb14, ninb) || !read(in, loc2glo, natom) ||
      !read(in, in14, (size_t)nin14 * 3) || !read(in, ex14, (size_t)nex14 * 3))
    return 2;
  std::fclose(in);

  cudaStream_t stream;
  CUDA(cudaStreamCreate(&stream));
  const int stride = ((natom + 31) / 32) * 32;
  float4* d_xyzq = nullptr;
  long long* d_force = nullptr;
  CUDA(cudaMalloc(&d_xyzq, sizeof(float4) * natom));
  CUDA(cudaMalloc(&d_force, sizeof(long long) * 3 * stride));
  CUDA(cudaMemcpy(d_xyzq, xyzq.data(), sizeof(float4) * natom, cudaMemcpyHostToDevice));
  CUDA(cudaMemset(d_force, 0, sizeof(long long) * 3 * stride));   // force_fp.clear()

  // CudaPMEDirectForce<long long, float> dir(energyVirial, "vdw", "elec", "excl");
  pme_direct* dir = nullptr;
  CHECK(pme_direct_create(stream, &dir));
  // dir.setup(boxx, boxy, boxz, kappa, roff, ron, e14fac, VDW_VSH, EWALD);
  CHECK(pme_direct_setup(dir, set[0], set[1], set[2], set[3], set[4], set[5], set[6], PME_VDW_VSH, PME_ELEC_EWALD));
  CHECK(pme_direct_set_vdwparam(dir, nvdw, vdwparam.data()));
  CHECK(pme_direct_set_vdwparam14(dir, nvdw14, vdwparam14.data()));
  CHECK(pme_direct_set_vdwtype(dir, natom, vdwtype.data()));
  // CudaTopExcl topExcl(ncoord, iblo14, inb14) and the neighbour list's loc2glo
  CHECK(pme_direct_set_exclusions(dir, natom, iblo14.data(), inb14.data(), loc2glo.data()));
  CHECK(pme_direct_set_14_list(dir, nin14, nex14, in14.data(), ex14.data()));

  FILE* out = std::fopen(argv[2], "wb");
  if (!out) return 2;
  // energyVirial.clear(); dir.calc_force(xyzq, nlist, true, true, stride, force)
  CHECK(pme_direct_clear_energy_virial(dir));
  CHECK(pme_direct_calc_force(dir, d_xyzq, natom, 1, 1, stride, d_force));
  if (dump(out, dir, d_force, natom, stride)) return 1;
  // dir.calc_14_force(xyzq, true, true, stride, force)
  CHECK(pme_direct_calc_14_force(dir, d_xyzq, 1, 1, stride, d_force));
  if (dump(out, dir, d_force, natom, stride)) return 1;
  std::fclose(out);

  CHECK(pme_direct_destroy(dir));
  CUDA(cudaFree(d_xyzq));
  CUDA(cudaFree(d_force));
  CUDA(cudaStreamDestroy(stream));
  return 0;
}

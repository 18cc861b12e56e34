// ref_gpu_bench.cu -- times the reference's own reciprocal-space operator on this GPU, as a
// same-GPU comparator for the bench; measurement only (it is never part of the library).
//
// The operator is the reference's CudaPMERecip<float, float, float2> (the instance its own test
// drives, gpu_recip.cu:59), compiled from the reference's unmodified sources with ref_shim.h.
// One evaluation is the sequence the reference's test and CudaDomdecRecip::calc run
// (gpu_recip.cu:133-138, CudaDomdecRecip.h:50-81): clear the energy/virial record, spread_charge,
// r2c_fft, scalar_sum with energy and virial, c2r_fft, gather_force<float>, calc_self_energy.
//
// stdin: a Header, then n float4 (x, y, z, q).  The L2 cache is flushed (a 256 MiB memset)
// before every evaluation, outside the CUDA events that time it.  stdout: one JSON line with the
// per-evaluation times, the energy/virial record of the last evaluation and the forces of the
// first `nforce` atoms (the reference's sign: +dE/dx).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "CudaEnergyVirial.h"
#include "CudaPMERecip.h"

struct Header {
  int n, nx, ny, nz, order, fft_type, warmup, steps, nforce;
  double kappa, boxx, boxy, boxz;
};

static void check(cudaError_t e, const char* what) {
  if (e != cudaSuccess) {
    std::fprintf(stderr, "ref_gpu_bench: %s: %s\n", what, cudaGetErrorString(e));
    std::exit(2);
  }
}

// A JSON number, or null for NaN / infinity.
static void put_num(double v, const char* sep) {
  if (std::isfinite(v)) std::printf("%s%.12g", sep, v);
  else std::printf("%snull", sep);
}

int main() {
  Header h;
  if (std::fread(&h, sizeof(h), 1, stdin) != 1 || h.n <= 0 || h.steps <= 0 || h.warmup < 0 ||
      (h.fft_type != COLUMN && h.fft_type != BOX) || h.nforce < 0 || h.nforce > h.n) {
    std::fprintf(stderr, "ref_gpu_bench: bad header\n");
    return 2;
  }
  std::vector<float> xyzq(4 * (size_t)h.n);
  if (std::fread(xyzq.data(), sizeof(float), xyzq.size(), stdin) != xyzq.size()) {
    std::fprintf(stderr, "ref_gpu_bench: short coordinate block\n");
    return 2;
  }
  const int stride = (h.n + 63) / 64 * 64;
  float4* d_xyzq = nullptr;
  float* d_force = nullptr;
  void* d_flush = nullptr;
  const size_t flush_bytes = 256u << 20;
  check(cudaMalloc(&d_xyzq, sizeof(float4) * h.n), "malloc xyzq");
  check(cudaMalloc(&d_force, sizeof(float) * 3 * stride), "malloc force");
  check(cudaMalloc(&d_flush, flush_bytes), "malloc flush");
  check(cudaMemcpy(d_xyzq, xyzq.data(), sizeof(float4) * h.n, cudaMemcpyHostToDevice), "copy xyzq");
  cudaStream_t stream;
  check(cudaStreamCreate(&stream), "stream");

  CudaEnergyVirial energyVirial;
  CudaPMERecip<float, float, float2> recip(h.nx, h.ny, h.nz, h.order, (FFTtype)h.fft_type, 1, 0, energyVirial,
                                           "recip", "self", stream);
  const double rm[9] = {1.0 / h.boxx, 0.0, 0.0, 0.0, 1.0 / h.boxy, 0.0, 0.0, 0.0, 1.0 / h.boxz};
  auto one_eval = [&]() {
    energyVirial.clear(stream);
    recip.spread_charge(d_xyzq, h.n, rm);
    recip.r2c_fft();
    recip.scalar_sum(rm, h.kappa, true, true);
    recip.c2r_fft();
    recip.gather_force(d_xyzq, h.n, rm, stride, d_force);
    recip.calc_self_energy(d_xyzq, h.n, h.kappa);
  };
  std::vector<cudaEvent_t> ev(2 * h.steps);
  for (auto& e : ev) check(cudaEventCreate(&e), "event");
  for (int i = 0; i < h.warmup; i++) {
    check(cudaMemsetAsync(d_flush, i & 0xff, flush_bytes, stream), "flush");
    one_eval();
  }
  for (int i = 0; i < h.steps; i++) {
    check(cudaMemsetAsync(d_flush, i & 0xff, flush_bytes, stream), "flush");
    check(cudaEventRecord(ev[2 * i], stream), "record");
    one_eval();
    check(cudaEventRecord(ev[2 * i + 1], stream), "record");
  }
  check(cudaStreamSynchronize(stream), "sync");
  std::vector<double> us(h.steps);
  for (int i = 0; i < h.steps; i++) {
    float ms = 0.0f;
    check(cudaEventElapsedTime(&ms, ev[2 * i], ev[2 * i + 1]), "elapsed");
    us[i] = 1000.0 * ms;
  }
  double mean = 0.0;
  for (double u : us) mean += u;
  mean /= h.steps;
  std::vector<double> sorted = us;
  std::sort(sorted.begin(), sorted.end());
  const double p50 = sorted[h.steps / 2];

  energyVirial.copyToHost(stream);
  check(cudaStreamSynchronize(stream), "sync record");
  double vir[9];
  energyVirial.getVirial(vir);
  std::vector<float> f(3 * (size_t)stride);
  check(cudaMemcpy(f.data(), d_force, sizeof(float) * f.size(), cudaMemcpyDeviceToHost), "copy force");

  std::printf("{\"fft_type\": \"%s\", \"steps\": %d, \"us_mean\": %.4f, \"us_p50\": %.4f, ",
              h.fft_type == BOX ? "box" : "column", h.steps, mean, p50);
  put_num(energyVirial.getEnergy("recip"), "\"energy_recip\": ");
  put_num(energyVirial.getEnergy("self"), ", \"energy_self\": ");
  std::printf(", \"virial\": [");
  for (int k = 0; k < 9; k++) put_num(vir[k], k ? ", " : "");
  std::printf("], \"force_head\": [");
  for (int i = 0; i < h.nforce; i++)
    for (int d = 0; d < 3; d++) put_num(f[i + (size_t)d * stride], i || d ? ", " : "");
  std::printf("]}\n");
  for (auto& e : ev) cudaEventDestroy(e);
  cudaFree(d_xyzq);
  cudaFree(d_force);
  cudaFree(d_flush);
  cudaStreamDestroy(stream);
  return 0;
}

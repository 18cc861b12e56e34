// looper_driver.cpp -- a C++ recip node built on the C ABI's request loop (pme_recip_loop_run,
// the role of CudaDomdecRecipLooper::run, CudaDomdecRecipLooper.cu:3-36).  The transport is a
// scripted in-process direct side: three steps with changing box scale, coordinate count and
// energy/virial flags, then STOP.  Each step's coordinates are copied to the device on the loop's
// stream by recv_coord; send_force copies the forces back and records the step's energy/virial.
//
// Input (binary, little endian): int32 natom, order, nx, ny, nz; float64 box[3], kappa;
// float32 xyzq[natom][4].  Output (binary): int64 steps; per step int32 ncoord, float64 record[11],
// float32 forces[ncoord][3].  Exit status 0 on success.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <vector>

#include "pme_recip.h"

namespace {

struct Step {
  double scale;
  int ncoord, calc_energy, calc_virial;
};

const Step kSteps[3] = {{1.0, 0, 1, 1}, {1.01, 7, 0, 1}, {0.995, 14, 1, 0}};   // ncoord = natom - this

struct DirectSide {
  std::vector<float> xyzq;
  int natom = 0;
  double box[3] = {0, 0, 0};
  int step = 0;                  // next header to send
  float* d_xyzq = nullptr;
  std::vector<int> counts;
  std::vector<double> records;
  std::vector<float> forces;
};

int recv_header(void* user, pme_recip_header* h) {
  DirectSide* d = (DirectSide*)user;
  if (d->step >= 3) {
    h->ncoord = -1;   // STOP
    return 0;
  }
  const Step& s = kSteps[d->step];
  h->inv_boxx = 1.0 / (d->box[0] * s.scale);
  h->inv_boxy = 1.0 / (d->box[1] * s.scale);
  h->inv_boxz = 1.0 / (d->box[2] * s.scale);
  h->ncoord = d->natom - s.ncoord;
  h->calc_energy = s.calc_energy;
  h->calc_virial = s.calc_virial;
  return 0;
}

int recv_coord(void* user, int ncoord, void* stream, const void** xyzq) {
  DirectSide* d = (DirectSide*)user;
  if (cudaMemcpyAsync(d->d_xyzq, d->xyzq.data(), (size_t)ncoord * 4 * sizeof(float), cudaMemcpyHostToDevice,
                      (cudaStream_t)stream) != cudaSuccess)
    return 1;
  *xyzq = d->d_xyzq;
  return 0;
}

int send_force(void* user, int ncoord, const void* force, const double* ev) {
  DirectSide* d = (DirectSide*)user;
  const size_t off = d->forces.size();
  d->forces.resize(off + 3 * (size_t)ncoord);
  if (cudaMemcpy(d->forces.data() + off, force, 3 * sizeof(float) * (size_t)ncoord, cudaMemcpyDeviceToHost) !=
      cudaSuccess)
    return 1;
  d->counts.push_back(ncoord);
  d->records.insert(d->records.end(), ev, ev + PME_EV_COUNT);
  d->step++;
  return 0;
}

}  // namespace

int main(int argc, char** argv) {
  if (argc != 3) {
    std::fprintf(stderr, "usage: %s input.bin output.bin\n", argv[0]);
    return 2;
  }
  FILE* in = std::fopen(argv[1], "rb");
  if (!in) return 2;
  int hdr[5];
  double kappa;
  DirectSide d;
  if (std::fread(hdr, sizeof(int), 5, in) != 5 || std::fread(d.box, sizeof(double), 3, in) != 3 ||
      std::fread(&kappa, sizeof(double), 1, in) != 1)
    return 2;
  d.natom = hdr[0];
  d.xyzq.resize((size_t)d.natom * 4);
  if (std::fread(d.xyzq.data(), sizeof(float), d.xyzq.size(), in) != d.xyzq.size()) return 2;
  std::fclose(in);
  if (cudaMalloc(&d.d_xyzq, d.xyzq.size() * sizeof(float)) != cudaSuccess) return 1;

  pme_recip* h = nullptr;
  if (pme_create(hdr[2], hdr[3], hdr[4], hdr[1], PME_FFT_BOX, 1, 0, nullptr, &h) != PME_OK) {
    std::fprintf(stderr, "pme_create: %s\n", pme_last_error_string());
    return 1;
  }
  pme_recip_comm comm;
  std::memset(&comm, 0, sizeof(comm));
  comm.user = &d;
  comm.recv_header = recv_header;
  comm.recv_coord = recv_coord;
  comm.send_force = send_force;
  long long steps = 0;
  if (pme_recip_loop_run(h, kappa, &comm, &steps) != PME_OK) {
    std::fprintf(stderr, "pme_recip_loop_run: %s\n", pme_last_error_string());
    return 1;
  }
  pme_destroy(h);
  cudaFree(d.d_xyzq);

  FILE* out = std::fopen(argv[2], "wb");
  if (!out) return 2;
  std::fwrite(&steps, sizeof(steps), 1, out);
  size_t f = 0;
  for (size_t k = 0; k < d.counts.size(); k++) {
    const int n = d.counts[k];
    std::fwrite(&n, sizeof(int), 1, out);
    std::fwrite(d.records.data() + k * PME_EV_COUNT, sizeof(double), PME_EV_COUNT, out);
    std::fwrite(d.forces.data() + f, sizeof(float), 3 * (size_t)n, out);
    f += 3 * (size_t)n;
  }
  std::fclose(out);
  return 0;
}

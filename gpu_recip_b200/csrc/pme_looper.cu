// pme_looper.cu -- the recip node's request loop behind the C ABI.
//
// The reference runs the reciprocal part on pure recip nodes: CudaDomdecRecipLooper::run
// (CudaDomdecRecipLooper.cu:3-36) receives a header from the direct nodes (inverse box edges,
// coordinate count, whether to compute energy and virial; DomdecRecipComm.h:11-15, a negative
// count is STOP), then the coordinates, runs CudaDomdecRecip::calc into a float3 force buffer that
// grows with the coordinate count, and sends the forces back, until STOP.  Here the transport is
// the caller's (the role of CudaDomdecRecipComm): three callbacks of pme_recip_comm.  Each step is
// one fused evaluation on the handle's stream; the step's own energy/virial record travels with
// the forces.
#include <cuda_runtime.h>

#include <cstring>
#include <string>

#include "../../include/pme_recip.h"
#include "pme_internal.h"

using namespace pme;

namespace {

int loop_fail(int status, const std::string& msg) {
  set_last_error(msg.c_str());
  return status;
}

}  // namespace

extern "C" {

int pme_recip_loop_run(pme_recip* h, double kappa, const pme_recip_comm* comm, long long* steps) {
  if (!h || !comm || !comm->recv_header || !comm->recv_coord || !comm->send_force)
    return loop_fail(PME_EINVAL, "recip loop: handle, comm or a callback is NULL");
  if (!(kappa > 0.0)) return loop_fail(PME_EINVAL, "recip loop: kappa must be positive");
  void* stream = nullptr;
  if (int rc = pme_get_stream(h, &stream)) return rc;
  cudaStream_t s = (cudaStream_t)stream;
  float* force = nullptr;       // device float3[cap], grown like reallocate<float3>
  size_t cap = 0;
  double* rec = nullptr;        // pinned host record of the step
  if (cudaMallocHost(&rec, PME_EV_COUNT * sizeof(double)) != cudaSuccess) {
    cudaGetLastError();
    return loop_fail(PME_ENOMEM, "recip loop: pinned record allocation failed");
  }
  long long done = 0;
  int rc = PME_OK;
  while (true) {
    pme_recip_header hdr;
    std::memset(&hdr, 0, sizeof(hdr));
    if (comm->recv_header(comm->user, &hdr) != 0) {
      rc = loop_fail(PME_ESTATE, "recip loop: recv_header failed");
      break;
    }
    if (hdr.ncoord < 0) break;   // STOP
    const int n = hdr.ncoord;
    if ((size_t)n > cap) {
      const cudaError_t e = cudaStreamSynchronize(s);
      cudaFree(force);
      force = nullptr;
      cap = 0;
      if (e != cudaSuccess || cudaMalloc(&force, 3 * sizeof(float) * (size_t)n) != cudaSuccess) {
        cudaGetLastError();
        rc = loop_fail(PME_ENOMEM, "recip loop: force buffer allocation failed");
        break;
      }
      cap = (size_t)n;
    }
    const void* xyzq = nullptr;
    if (comm->recv_coord(comm->user, n, stream, &xyzq) != 0 || (n > 0 && !xyzq)) {
      rc = loop_fail(PME_ESTATE, "recip loop: recv_coord failed");
      break;
    }
    if ((rc = pme_clear_energy_virial(h))) break;
    if ((rc = pme_eval_ortho(h, hdr.inv_boxx, hdr.inv_boxy, hdr.inv_boxz, xyzq, n, kappa, hdr.calc_energy,
                             hdr.calc_virial, PME_FORCE_F32X3, force, n)))
      break;
    if ((rc = pme_copy_energy_virial_async(h, rec))) break;
    const cudaError_t e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
      cudaGetLastError();
      rc = loop_fail(PME_ECUDA, std::string("recip loop: ") + cudaGetErrorString(e));
      break;
    }
    int status = 0;
    if ((rc = pme_get_status(h, &status))) break;
    if (comm->send_force(comm->user, n, force, rec) != 0) {
      rc = loop_fail(PME_ESTATE, "recip loop: send_force failed");
      break;
    }
    done++;
  }
  cudaStreamSynchronize(s);
  cudaFree(force);
  cudaFreeHost(rec);
  if (steps) *steps = done;
  return rc;
}

}  // extern "C"

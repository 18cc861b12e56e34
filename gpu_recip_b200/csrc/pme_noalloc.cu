// pme_noalloc.cu -- charge spreading that allocates no device memory.
//
// Some callers cannot allocate device memory at the moment they need a charge grid: hosts whose
// own memory manager owns every device byte and forbids plug-ins from calling cudaMalloc behind
// its back, and time-critical loops that must not take the allocator's locks or let an
// allocation synchronise the device.  For them this entry point spreads the charges with the
// same kernel as pme_spread_charge, but accumulates the exact int64 grid in a fixed device array
// compiled into this library instead of in memory the library allocates.
//
// The array lives as long as the library is loaded and costs kNoAllocMaxPoints * 8 bytes
// (8 MiB) on every GPU that loads it.  It is shared by every call: each call clears the part it
// uses before spreading, and two calls whose work overlaps on the GPU (different streams, no
// ordering between them) race on it.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <mutex>
#include <string>

#include "../../include/pme_recip.h"
#include "pme_internal.h"

using namespace pme;

namespace {

constexpr size_t kNoAllocMaxPoints = (size_t)1 << 20;   // nfftx * nffty * nfftz limit
constexpr int kMaxDevices = 64;

}  // namespace

static __device__ __align__(256) unsigned long long g_noalloc_grid[kNoAllocMaxPoints];

namespace {

// Driver calls reached through the runtime (no link-time dependency on the driver library).
typedef int (*CtxGetCurrentFn)(void** ctx);
typedef int (*CtxGetIdFn)(void* ctx, unsigned long long* id);

struct ScratchSlot {
  unsigned long long ctx_id = 0;   // unique ID of the context the address belongs to (0: none)
  void* addr = nullptr;
};

std::mutex g_symbol_mutex;
ScratchSlot g_symbol_slot[kMaxDevices];

int noalloc_fail(int status, const std::string& msg) {
  set_last_error(msg.c_str());   // reported by pme_last_error_string()
  return status;
}

// Unique ID of the calling thread's current context (0 when there is none yet).  IDs are never
// reused within a process, so an address looked up in a context that a device reset destroyed is
// never taken for one in the context that replaced it.
unsigned long long current_context_id() {
  static CtxGetCurrentFn get_current = nullptr;
  static CtxGetIdFn get_id = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_current = (CtxGetCurrentFn)f;
    f = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_id = (CtxGetIdFn)f;
    cudaGetLastError();
  });
  void* ctx = nullptr;
  unsigned long long id = 0;
  if (!get_current || !get_id || get_current(&ctx) != 0 || ctx == nullptr || get_id(ctx, &id) != 0) return 0;
  return id;
}

// Set-up of the scratch array on the current device: its device address, looked up once per
// device (and again only if the device's context has been replaced, e.g. after cudaDeviceReset).
// In host code the array's name is only a host-side stand-in, never a usable device address.
cudaError_t scratch_address(int dev, void** out) {
  std::lock_guard<std::mutex> lock(g_symbol_mutex);
  ScratchSlot& slot = g_symbol_slot[dev];
  const unsigned long long id = current_context_id();
  if (slot.addr == nullptr || id == 0 || id != slot.ctx_id) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_grid);   // creates the context if needed
    if (e != cudaSuccess) return e;
    slot.addr = p;
    slot.ctx_id = current_context_id();
  }
  *out = slot.addr;
  return cudaSuccess;
}

__global__ void k_fixed_to_float(const unsigned long long* __restrict__ in, float* __restrict__ out,
                                 size_t count) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < count; i += (size_t)gridDim.x * blockDim.x)
    out[i] = fixed_to_float((long long)in[i]);
}

bool smooth235(int n) {
  for (int f : {2, 3, 5})
    while (n % f == 0) n /= f;
  return n == 1;
}

}  // namespace

extern "C" {

int pme_spread_charge_noalloc(const void* xyzq, int ncoord, const double* recip, int nfftx, int nffty,
                              int nfftz, int order, float* grid_out, void* stream) {
  if (order != 4 && order != 6 && order != 8) return noalloc_fail(PME_EINVAL, "order must be 4, 6 or 8");
  const int n3[3] = {nfftx, nffty, nfftz};
  for (int d = 0; d < 3; d++) {
    if (n3[d] < order || n3[d] > kMaxFftLen) return noalloc_fail(PME_EINVAL, "grid lengths must be in [order, 512]");
    if (!smooth235(n3[d])) return noalloc_fail(PME_EUNSUPPORTED, "grid lengths must factor into 2, 3 and 5");
  }
  const size_t G = (size_t)nfftx * nffty * nfftz;
  if (G > kNoAllocMaxPoints)
    return noalloc_fail(PME_EINVAL, "grid too large for the no-allocation spread: nfftx*nffty*nfftz must be <= 1048576");
  if (ncoord < 0 || (ncoord > 0 && !xyzq)) return noalloc_fail(PME_EINVAL, "bad xyzq/ncoord");
  if (!grid_out) return noalloc_fail(PME_EINVAL, "grid_out is NULL");
  if (!recip) return noalloc_fail(PME_EINVAL, "recip is NULL");
  if (!(recip[1] == 0.0 && recip[2] == 0.0 && recip[3] == 0.0 && recip[5] == 0.0 && recip[6] == 0.0 &&
        recip[7] == 0.0))
    return noalloc_fail(PME_EINVAL, "only orthorhombic boxes are supported (recip off-diagonals must be 0)");
  for (int i : {0, 4, 8})
    if (!(recip[i] > 0.0) || !std::isfinite(recip[i]))
      return noalloc_fail(PME_EINVAL, "recip diagonal must be finite and positive");

  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess || dev < 0 || dev >= kMaxDevices)
    return noalloc_fail(PME_ECUDA, "no usable current device");
  void* scratch = nullptr;
  e = scratch_address(dev, &scratch);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return noalloc_fail(PME_ECUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
  }
  cudaStream_t s = (cudaStream_t)stream;

  // the array keeps the previous call's grid: clear the part this call accumulates into
  e = cudaMemsetAsync(scratch, 0, G * sizeof(unsigned long long), s);
  if (e != cudaSuccess) return noalloc_fail(PME_ECUDA, std::string("clear scratch: ") + cudaGetErrorString(e));

  SysDesc d;
  std::memset(&d, 0, sizeof(d));
  Geom& g = d.g;
  g.nx = nfftx; g.ny = nffty; g.nz = nfftz;
  g.hx = nfftx / 2 + 1;
  const double r3[3] = {recip[0], recip[4], recip[8]};
  g.rx = (float)r3[0]; g.ry = (float)r3[1]; g.rz = (float)r3[2];
  float hi[3], lo[3];
  for (int i = 0; i < 3; i++) {
    const double sc = r3[i] * n3[i];
    hi[i] = (float)sc;
    lo[i] = (float)(sc - (double)hi[i]);
  }
  g.sx_hi = hi[0]; g.sy_hi = hi[1]; g.sz_hi = hi[2];
  g.sx_lo = lo[0]; g.sy_lo = lo[1]; g.sz_lo = lo[2];
  d.order = order;
  d.natom = ncoord;
  d.xyzq = (const float4*)xyzq;
  d.accum = (unsigned long long*)scratch;
  e = staged_spread(d, s);
  if (e != cudaSuccess) return noalloc_fail(PME_ECUDA, std::string("spread: ") + cudaGetErrorString(e));
  int blocks = (int)((G + 255) / 256);
  if (blocks > 4096) blocks = 4096;
  k_fixed_to_float<<<blocks, 256, 0, s>>>((const unsigned long long*)scratch, grid_out, G);
  e = cudaGetLastError();
  if (e != cudaSuccess) return noalloc_fail(PME_ECUDA, std::string("convert: ") + cudaGetErrorString(e));
  return PME_OK;
}

}  // extern "C"

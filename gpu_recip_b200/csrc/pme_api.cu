// pme_api.cu -- host engine and C ABI of the B200 smooth-PME reciprocal-space operator.
//
// A pme_recip instance mirrors one CudaPMERecip<long long, float, float2> of the reference
// (CudaPMERecip.h:37-205); a pme_batch holds many independent systems evaluated by one
// persistent launch.  Both own, per system, the int64 accumulation grid, the half-complex grid,
// the solved real grid, FFT plans with FP64-accurate twiddles, FP64 B-spline moduli, the FP64
// influence tables, the fixed-point energy/virial accumulators and the FP64 energy/virial record,
// carved from one device allocation.  Compute calls only enqueue work on the instance's stream
// (no allocation, no host synchronisation), so evaluations can be captured in CUDA graphs.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <new>
#include <tuple>
#include <string>
#include <vector>

#include "../../include/pme_recip.h"
#include "pme_internal.h"
#include "pme_state.h"

using namespace pme;

namespace {

thread_local std::string g_err;

}  // namespace

namespace pme {
void set_last_error(const char* msg) { g_err = msg ? msg : ""; }
}  // namespace pme

struct pme_recip {
  int fft_type = PME_FFT_BOX;
  int* d_bins = nullptr;
  int device = 0;
  cudaStream_t stream = nullptr;
  SystemState st;
  char* d_block = nullptr;
  unsigned long long* d_bar = nullptr;
  int* d_status = nullptr;
  size_t max_smem = 0;
  unsigned int spin_limit = 1u << 22;
  int inject = 0;
  unsigned long long* trace = nullptr;
  int trace_ctas = 0;
  double* ev_mirror = nullptr;   // device-mapped pinned host memory, or null
  int plane_mode = 0;   // 0 automatic, 1 whole-plane tiles where they fit, 2 separate passes
  int grid_cap = 0;     // CTAs of the persistent launch (0: as many as are resident)
  int x_gather = PME_XGATHER_AUTO;   // PME_XGATHER_*
  bool accum_zero = true;
  bool no_cluster = false;   // the cluster launch of the plane phase could not be shaped here    // the int64 charge grid is known to be all zero (staged spread skips its clear)
  float* d_force = nullptr;      // pme_eval_host: device forces before the copy to the host
  size_t force_bytes = 0;
};

struct pme_batch {
  int device = 0;
  cudaStream_t stream = nullptr;
  std::vector<SystemState> st;
  std::vector<SysDesc> desc;
  SysDesc* d_desc = nullptr;
  int* d_prefix = nullptr;
  int total[kPhases] = {0};
  char* d_block = nullptr;
  unsigned long long* d_bar = nullptr;
  int* d_status = nullptr;
  size_t smem = 0;
  FusedShape shape{kFusedLatency, 0};
  unsigned int spin_limit = 1u << 22;
  size_t bytes = 0;
  unsigned long long* trace = nullptr;
  int trace_ctas = 0;
  int plane_mode = 0;   // PME_SCHED_*: AUTO and PLANES use planes where they fit
  int grid_cap = 0;
  int line_scale = 1;   // lines per x/y/z pass tile: each system's default times this (budget permitting)
};

namespace {

void release(pme_recip* h) {
  if (!h) return;
  cudaFree(h->d_force);
  cudaFree(h->d_bins);
  cudaFree(h->d_block);
  cudaFree(h->d_bar);
  delete h;
}

int handle_ok(const pme_recip* h) { return h ? PME_OK : fail(PME_EINVAL, "handle is NULL"); }

// Barrier words of a handle: [0] arrival counter, [1] its value at launch start, [2] device status
// (int), [3] launch counter (bin parity), [4] arrival counter of the self-energy launch.
constexpr int kBarWords = 6;

StagedCtx staged_ctx(const pme_recip* h) { return StagedCtx{h->d_bar, h->d_status, h->spin_limit}; }

unsigned int* self_counter(const pme_recip* h) { return (unsigned int*)(h->d_bar + 4); }

// Size the fused path's atom bins for natom atoms (allocates only when the count grows).
int ensure_bins(pme_recip* h, int natom) {
  SystemState& s = h->st;
  if (h->d_bins && natom <= s.atom_cap) return PME_OK;
  const int cap = std::max(natom, 1024);
  const size_t ints = s.bin_ints(cap);
  cudaError_t e = cudaStreamSynchronize(h->stream);
  if (e != cudaSuccess) return cuda_fail(e, "bins: sync");
  cudaFree(h->d_bins);
  h->d_bins = nullptr;
  if (cudaMalloc(&h->d_bins, ints * sizeof(int)) != cudaSuccess) {
    cudaGetLastError();
    s.bins = nullptr;
    s.atom_cap = 0;
    return fail(PME_ENOMEM, "device allocation of the atom bins failed");
  }
  e = cudaMemset(h->d_bins, 0, ints * sizeof(int));
  if (e != cudaSuccess) return cuda_fail(e, "bins: clear");
  s.bins = h->d_bins;
  s.atom_cap = cap;
  s.bin_cap = SystemState::cap_for(cap, s.nbins());
  return PME_OK;
}

int launch_fused_single(pme_recip* h, const SysDesc& d_in) {
  SysDesc d = d_in;
  FusedArgs a;
  std::memset(&a, 0, sizeof(a));
  a.table = nullptr;
  a.nsys = 1;
  a.prefix = nullptr;
  a.bar = h->d_bar;
  a.status = h->d_status;
  a.spin_limit = h->spin_limit;
  a.inject = h->inject;
  a.trace = h->trace;
  a.trace_ctas = h->trace_ctas;
  if (h->trace) d.steps = h->trace + (size_t)h->trace_ctas * kPhases * 2;
  // whole-plane tiles only pay when there are enough planes to occupy the GPU; otherwise the
  // separate y and z passes spread the same work over many more CTAs
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, h->device);
  if (h->plane_mode == 0) d.plane = (d.plane && d.g.hx >= sms) ? 1 : 0;
  else d.plane = (d.plane && h->plane_mode == 1) ? 1 : 0;
  // fewer full bin tiles than SMs: half-size tiles, so that no SM bins more than kThreads atoms
  // where the hardware doubles CTAs up (measured on 24,000 atoms: 0.9 us faster; 64-atom tiles
  // were 2 us slower)
  d.bin_atoms = (d.natom + kThreads - 1) / kThreads < sms ? kThreads / 2 : kThreads;
  // inverse x pass inside the gather tiles where its rows fit in the shared memory the other
  // phases already take (so that the launch keeps its CTAs per SM)
  // (latency build only: the throughput build, for launches with many tiles per CTA, keeps the
  // separate phase and is compiled without the fused variant)
  d.gx = 0;
  if (h->x_gather == PME_XGATHER_AUTO && gx_smem_bytes(d.g.nx, d.bry, d.brz, d.order) <= fused_smem_bytes(d)) d.gx = 1;
  fused_tile_counts(d, a.total);
  size_t smem = fused_smem_bytes(d);
  FusedShape shape;
  cudaError_t e = fused_shape(a.total, smem, h->grid_cap, &shape);
  if (e == cudaSuccess && d.gx && shape.variant != kFusedLatency) {
    d.gx = 0;
    fused_tile_counts(d, a.total);
    smem = fused_smem_bytes(d);
    e = fused_shape(a.total, smem, h->grid_cap, &shape);
  }
  if (e != cudaSuccess) return cuda_fail(e, "fused: launch shape (does the kernel fit on an SM?)");
  // y, z, the solve and both inverses as kx planes split over 4-CTA clusters, where the plane
  // count alone would leave most SMs idle (latency build, orthorhombic, line counts divisible);
  // by default from 32 planes up (64^3: 55.8 against 61.9 us with passes; 32^3 with 17 planes:
  // 43.5 against 41.5 us with one CTA per plane)
  const bool want_cluster = h->plane_mode == PME_SCHED_CLUSTER ||
                            (h->plane_mode == PME_SCHED_AUTO && !d.plane && d.g.hx >= 32);
  if (want_cluster && !h->no_cluster && shape.variant == kFusedLatency && !d.g.tric && d.g.ny % kClusterPlane == 0 &&
      d.g.nz % kClusterPlane == 0 && cplane_smem_bytes(d.g.ny, d.g.nz, kClusterPlane) <= kTileSmemBudget) {
    SysDesc c = d;
    c.plane = 0;
    c.cplane = kClusterPlane;
    int tot[kPhases];
    fused_tile_counts(c, tot);
    const size_t csmem = fused_smem_bytes(c);
    FusedShape cshape;
    if (fused_shape_cluster(tot, csmem, h->grid_cap, kClusterPlane, &cshape) == cudaSuccess) {
      d = c;
      std::memcpy(a.total, tot, sizeof(tot));
      smem = csmem;
      shape = cshape;
    } else {
      cudaGetLastError();
      h->no_cluster = true;   // this device cannot hold the cluster launch: never try again
    }
  }
  d.gsort = gather_sorts(d, smem);
  a.nbar = fused_barriers(a.total);
  a.single = d;
  e = fused_launch(a, shape, smem, h->stream);
  if (e != cudaSuccess) return cuda_fail(e, "fused eval launch");
  return PME_OK;
}

// ---- launch shapes (autotuner) ----
struct TuneKey {
  int dev, nx, ny, nz, order;
  bool operator<(const TuneKey& o) const {
    return std::tie(dev, nx, ny, nz, order) < std::tie(o.dev, o.nx, o.ny, o.nz, o.order);
  }
};
std::mutex g_tune_mutex;
std::map<TuneKey, pme_tune_config> g_tune_cache;

TuneKey tune_key(const pme_recip* h) { return TuneKey{h->device, h->st.nx, h->st.ny, h->st.nz, h->st.order}; }

void get_config(const pme_recip* h, pme_tune_config* c) {
  std::memset(c, 0, sizeof(*c));
  c->schedule = h->plane_mode;
  c->x_lines = h->st.tx_rows;
  c->y_lines = h->st.tx_y;
  c->z_columns = h->st.tx_z;
  c->grid_ctas = h->grid_cap;
}

// Does a shape fit the fused kernel's per-tile shared-memory budget?
bool config_fits(const SystemState& st, const pme_tune_config& c) {
  if (c.schedule < PME_SCHED_AUTO || c.schedule > PME_SCHED_CLUSTER) return false;
  if (c.x_lines < 1 || c.y_lines < 1 || c.z_columns < 1 || c.grid_ctas < 0) return false;
  if (c.x_lines > 64 || c.y_lines > 64 || c.z_columns > 64) return false;
  return tile_smem_bytes(st.nx, c.x_lines) <= kTileSmemBudget && tile_smem_bytes(st.ny, c.y_lines) <= kTileSmemBudget &&
         tile_smem_bytes(st.nz, c.z_columns) + ktab_smem_bytes(st.ny, st.nz) <= kTileSmemBudget;
}

void set_config(pme_recip* h, const pme_tune_config& c) {
  h->plane_mode = c.schedule;
  h->st.tx_rows = c.x_lines;
  h->st.tx_y = c.y_lines;
  h->st.tx_z = c.z_columns;
  h->grid_cap = c.grid_ctas;
}

// base * scale lines per pass tile, at most limit, shrunk (not below base) until the tile's
// shared memory (plus `extra` bytes) fits the budget.
int scaled_lines(int L, int base, int scale, int limit, size_t extra) {
  int t = std::min(base * scale, std::max(limit, base));
  while (t > base && tile_smem_bytes(L, t) + extra > kTileSmemBudget) t--;
  return t;
}

void apply_cached_config(pme_recip* h) {
  std::lock_guard<std::mutex> lock(g_tune_mutex);
  auto it = g_tune_cache.find(tune_key(h));
  if (it != g_tune_cache.end() && config_fits(h->st, it->second)) set_config(h, it->second);
}

}  // namespace

extern "C" {

int pme_create(int nfftx, int nffty, int nfftz, int order, int fft_type, int nnode, int mynode,
               void* stream, pme_recip** out) {
  if (!out) return fail(PME_EINVAL, "out is NULL");
  *out = nullptr;
  if (nnode != 1 || mynode != 0)
    return fail(PME_EUNSUPPORTED, "multi-node grid decomposition is not supported (nnode must be 1)");
  if (fft_type != PME_FFT_COLUMN && fft_type != PME_FFT_SLAB && fft_type != PME_FFT_BOX)
    return fail(PME_EINVAL, "invalid fft_type");
  int rc = check_grid(nfftx, nffty, nfftz, order);
  if (rc) return rc;
  pme_recip* h = new (std::nothrow) pme_recip();
  if (!h) return fail(PME_ENOMEM, "host allocation failed");
  h->fft_type = fft_type;
  h->stream = (cudaStream_t)stream;
  cudaError_t e = cudaGetDevice(&h->device);
  if (e != cudaSuccess) { delete h; return cuda_fail(e, "cudaGetDevice"); }
  e = configure_kernels(&h->max_smem);
  if (e != cudaSuccess) { delete h; return cuda_fail(e, "configure kernels"); }
  h->st.setup(nfftx, nffty, nfftz, order);
  apply_cached_config(h);
  const size_t bytes = SystemState::bytes(nfftx, nffty, nfftz);
  if (cudaMalloc(&h->d_block, bytes) != cudaSuccess ||
      cudaMalloc(&h->d_bar, kBarWords * sizeof(unsigned long long)) != cudaSuccess) {
    cudaGetLastError();
    release(h);
    return fail(PME_ENOMEM, "device allocation failed");
  }
  h->d_status = (int*)(h->d_bar + 2);
  h->st.carve(h->d_block);
  e = cudaMemset(h->d_block, 0, bytes);
  if (e == cudaSuccess) e = cudaMemset(h->d_bar, 0, kBarWords * sizeof(unsigned long long));
  if (e == cudaSuccess) e = h->st.upload_tables();
  if (e != cudaSuccess) {
    release(h);
    return cuda_fail(e, "pme_create: initialise buffers");
  }
  *out = h;
  return PME_OK;
}

int pme_destroy(pme_recip* h) {
  if (!h) return PME_OK;
  DeviceGuard dg(h->device);
  release(h);
  return PME_OK;
}

int pme_set_stream(pme_recip* h, void* stream) {
  if (int rc = handle_ok(h)) return rc;
  h->stream = (cudaStream_t)stream;
  return PME_OK;
}

int pme_get_stream(const pme_recip* h, void** stream) {
  if (!h || !stream) return fail(PME_EINVAL, "NULL argument");
  *stream = (void*)h->stream;
  return PME_OK;
}

int pme_set_order(pme_recip* h, int order) {
  if (int rc = handle_ok(h)) return rc;
  if (int rc = check_grid(h->st.nx, h->st.ny, h->st.nz, order)) return rc;
  DeviceGuard dg(h->device);
  cudaError_t e = cudaStreamSynchronize(h->stream);   // tables are replaced synchronously
  if (e != cudaSuccess) return cuda_fail(e, "set_order");
  h->st.order = order;
  e = h->st.upload_tables();
  if (e != cudaSuccess) return cuda_fail(e, "set_order: upload moduli");
  return PME_OK;
}

int pme_get_nfft(const pme_recip* h, int* nx, int* ny, int* nz) {
  if (int rc = handle_ok(h)) return rc;
  if (nx) *nx = h->st.nx;
  if (ny) *ny = h->st.ny;
  if (nz) *nz = h->st.nz;
  return PME_OK;
}

int pme_get_order(const pme_recip* h, int* order) {
  if (!h || !order) return fail(PME_EINVAL, "NULL argument");
  *order = h->st.order;
  return PME_OK;
}

int pme_print_info(const pme_recip* h) {
  if (int rc = handle_ok(h)) return rc;
  const SystemState& s = h->st;
  const char* ft = h->fft_type == PME_FFT_COLUMN ? "COLUMN" : (h->fft_type == PME_FFT_SLAB ? "SLAB" : "BOX");
  std::printf("fft_type = %s computed using the built-in sm_100a 2/3/5-radix FFT\n", ft);
  std::printf("order = %d\n", s.order);
  std::printf("nfftx, nffty, nfftz = %d %d %d\n", s.nx, s.ny, s.nz);
  std::printf("x0...x1   = 0 ... %d\ny0...y1   = 0 ... %d\nz0...z1   = 0 ... %d\n", s.nx - 1, s.ny - 1,
              s.nz - 1);
  std::printf("xsize, ysize, zsize = %d %d %d\n", s.nx, s.ny, s.nz);
  std::printf("data_size = %d\n", 2 * (s.nx / 2 + 1) * s.ny * s.nz);
  std::printf("tiles: x %d rows, y %d, z %d columns per CTA\n", s.tx_rows, s.tx_y, s.tx_z);
  std::fflush(stdout);
  return PME_OK;
}

int pme_spread_charge(pme_recip* h, const void* xyzq, int ncoord, const double* recip) {
  if (int rc = handle_ok(h)) return rc;
  if (ncoord < 0 || (ncoord > 0 && !xyzq)) return fail(PME_EINVAL, "bad xyzq/ncoord");
  if (int rc = check_recip(recip)) return rc;
  DeviceGuard dg(h->device);
  // the atomic spread adds into the int64 grid: clear it unless it is known to be zero (after
  // creation and after r2c_fft, which clears it behind its read)
  if (!h->accum_zero) {
    cudaError_t e = cudaMemsetAsync(h->st.accum, 0, h->st.G() * 8, h->stream);
    if (e != cudaSuccess) return cuda_fail(e, "spread_charge: clear grid");
  }
  h->accum_zero = false;
  cudaError_t e = staged_spread(h->st.desc9(recip, 0.0, xyzq, ncoord, nullptr, 0, 0, 0, 0), h->stream);
  if (e != cudaSuccess) return cuda_fail(e, "spread_charge");
  return PME_OK;
}

int pme_r2c_fft(pme_recip* h) {
  if (int rc = handle_ok(h)) return rc;
  DeviceGuard dg(h->device);
  cudaError_t e = staged_r2c(h->st.desc(nullptr, 0.0, nullptr, 0, nullptr, 0, 0, 0, 0), staged_ctx(h), h->stream);
  if (e != cudaSuccess) return cuda_fail(e, "r2c_fft");
  h->accum_zero = true;
  return PME_OK;
}

int pme_scalar_sum(pme_recip* h, const double* recip, double kappa, int calc_energy, int calc_virial) {
  if (int rc = handle_ok(h)) return rc;
  if (int rc = check_recip(recip)) return rc;
  if (!(kappa > 0.0) || !std::isfinite(kappa)) return fail(PME_EINVAL, "kappa must be positive");
  DeviceGuard dg(h->device);
  const int ev = (calc_energy || calc_virial) ? 1 : 0;
  cudaError_t e = staged_solve(h->st.desc9(recip, kappa, nullptr, 0, nullptr, 0, 0, ev, 0), staged_ctx(h), h->stream);
  if (e != cudaSuccess) return cuda_fail(e, "scalar_sum");
  return PME_OK;
}

int pme_c2r_fft(pme_recip* h) {
  if (int rc = handle_ok(h)) return rc;
  DeviceGuard dg(h->device);
  cudaError_t e = staged_c2r(h->st.desc(nullptr, 0.0, nullptr, 0, nullptr, 0, 0, 0, 0), staged_ctx(h), h->stream);
  if (e != cudaSuccess) return cuda_fail(e, "c2r_fft");
  return PME_OK;
}

int pme_gather_force(pme_recip* h, const void* xyzq, int ncoord, const double* recip, int stride,
                     int kind, void* force) {
  if (int rc = handle_ok(h)) return rc;
  if (ncoord < 0 || (ncoord > 0 && !xyzq)) return fail(PME_EINVAL, "bad xyzq/ncoord");
  if (int rc = check_recip(recip)) return rc;
  if (int rc = check_force_args(ncoord, stride, kind, force)) return rc;
  DeviceGuard dg(h->device);
  cudaError_t e = staged_gather(h->st.desc9(recip, 0.0, xyzq, ncoord, force, kind, stride, 0, 0), h->stream);
  if (e != cudaSuccess) return cuda_fail(e, "gather_force");
  return PME_OK;
}

int pme_calc_self_energy(pme_recip* h, const void* xyzq, int ncoord, double kappa) {
  if (int rc = handle_ok(h)) return rc;
  if (ncoord < 0 || (ncoord > 0 && !xyzq)) return fail(PME_EINVAL, "bad xyzq/ncoord");
  if (!std::isfinite(kappa)) return fail(PME_EINVAL, "kappa must be finite");
  DeviceGuard dg(h->device);
  cudaError_t e = staged_self(h->st.desc(nullptr, kappa, xyzq, ncoord, nullptr, 0, 0, 0, 1), self_counter(h), h->stream);
  if (e != cudaSuccess) return cuda_fail(e, "calc_self_energy");
  return PME_OK;
}

int pme_clear_energy_virial(pme_recip* h) {
  if (int rc = handle_ok(h)) return rc;
  DeviceGuard dg(h->device);
  cudaError_t e = cudaMemsetAsync(h->st.ev, 0, kEvCount * sizeof(double), h->stream);
  if (e != cudaSuccess) return cuda_fail(e, "clear_energy_virial");
  return PME_OK;
}

int pme_get_energy_virial(pme_recip* h, double* energy_recip, double* energy_self, double* virial9) {
  if (int rc = handle_ok(h)) return rc;
  DeviceGuard dg(h->device);
  double buf[kEvCount];
  int status = 0;
  cudaError_t e = cudaMemcpyAsync(buf, h->st.ev, sizeof(buf), cudaMemcpyDeviceToHost, h->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(&status, h->d_status, sizeof(int), cudaMemcpyDeviceToHost, h->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  if (e != cudaSuccess) return cuda_fail(e, "get_energy_virial");
  if (energy_recip) *energy_recip = buf[kEvRecip];
  if (energy_self) *energy_self = buf[kEvSelf];
  if (virial9) for (int i = 0; i < 9; i++) virial9[i] = buf[kEvVirial + i];
  if (status != kStatusOk)
    return fail(PME_ETIMEOUT, "a grid barrier of the fused evaluation timed out; results are incomplete");
  return PME_OK;
}

int pme_copy_energy_virial_async(pme_recip* h, double* dst) {
  if (!h || !dst) return fail(PME_EINVAL, "NULL argument");
  DeviceGuard dg(h->device);
  cudaError_t e = cudaMemcpyAsync(dst, h->st.ev, kEvCount * sizeof(double), cudaMemcpyDefault, h->stream);
  if (e != cudaSuccess) return cuda_fail(e, "copy_energy_virial_async");
  return PME_OK;
}

int pme_energy_virial_device_ptr(pme_recip* h, double** dev_ptr) {
  if (!h || !dev_ptr) return fail(PME_EINVAL, "NULL argument");
  *dev_ptr = h->st.ev;
  return PME_OK;
}

int pme_set_energy_virial_mirror(pme_recip* h, double* host_mapped) {
  if (int rc = handle_ok(h)) return rc;
  if (host_mapped) {
    cudaPointerAttributes a;
    cudaError_t e = cudaPointerGetAttributes(&a, host_mapped);
    if (e != cudaSuccess || a.type != cudaMemoryTypeHost || a.devicePointer != (void*)host_mapped) {
      cudaGetLastError();
      return fail(PME_EINVAL, "energy/virial mirror must be pinned host memory mapped at the same address");
    }
  }
  h->ev_mirror = host_mapped;
  return PME_OK;
}

int pme_eval_ortho(pme_recip* h, double inv_boxx, double inv_boxy, double inv_boxz, const void* xyzq,
                   int ncoord, double kappa, int calc_energy, int calc_virial, int kind, void* force,
                   int stride) {
  const double recip[9] = {inv_boxx, 0, 0, 0, inv_boxy, 0, 0, 0, inv_boxz};
  return pme_eval(h, recip, xyzq, ncoord, kappa, calc_energy, calc_virial, kind, force, stride);
}

int pme_eval(pme_recip* h, const double* recip, const void* xyzq, int ncoord, double kappa,
             int calc_energy, int calc_virial, int kind, void* force, int stride) {
  if (int rc = handle_ok(h)) return rc;
  if (ncoord < 0 || (ncoord > 0 && !xyzq)) return fail(PME_EINVAL, "bad xyzq/ncoord");
  if (int rc = check_recip(recip)) return rc;
  if (!(kappa > 0.0) || !std::isfinite(kappa)) return fail(PME_EINVAL, "kappa must be positive");
  if (int rc = check_force_args(ncoord, stride, kind, force)) return rc;
  DeviceGuard dg(h->device);
  if (int rc = ensure_bins(h, ncoord)) return rc;
  const int ev = (calc_energy || calc_virial) ? 1 : 0;
  SysDesc d = h->st.desc9(recip, kappa, xyzq, ncoord, force, kind, stride, ev, calc_energy ? 1 : 0);
  d.ev_mirror = h->ev_mirror;
  return launch_fused_single(h, d);
}

// True when p is page-locked host memory that the device reads at the same address.
static bool host_mapped(const void* p) {
  cudaPointerAttributes a;
  const cudaError_t e = cudaPointerGetAttributes(&a, p);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeHost && a.devicePointer == p;
}

int pme_eval_host(pme_recip* h, const double* recip, const void* xyzq_host, int ncoord, double kappa,
                  int calc_energy, int calc_virial, int kind, void* force_host, int stride) {
  if (int rc = handle_ok(h)) return rc;
  if (ncoord < 0 || (ncoord > 0 && !xyzq_host)) return fail(PME_EINVAL, "bad xyzq/ncoord");
  if (int rc = check_recip(recip)) return rc;
  if (!(kappa > 0.0) || !std::isfinite(kappa)) return fail(PME_EINVAL, "kappa must be positive");
  if (int rc = check_force_args(ncoord, stride, kind, force_host)) return rc;
  if (kind == PME_FORCE_I64_SOA_ACCUM)
    return fail(PME_EUNSUPPORTED, "eval_host writes float forces; accumulate int64 forces with pme_eval");
  if (ncoord == 0) return PME_OK;
  DeviceGuard dg(h->device);
  if (!host_mapped(xyzq_host))
    return fail(PME_EINVAL, "xyzq must be pinned host memory mapped at the same address");
  cudaPointerAttributes fa;
  if (cudaPointerGetAttributes(&fa, force_host) != cudaSuccess || fa.type != cudaMemoryTypeHost) {
    cudaGetLastError();
    return fail(PME_EINVAL, "force must be pinned host memory");
  }
  // device layout as the caller's: float3[ncoord], or three rows of `stride` floats
  const size_t bytes = 3 * (kind == PME_FORCE_F32X3 ? (size_t)ncoord : (size_t)stride) * sizeof(float);
  if (bytes > h->force_bytes) {
    cudaError_t e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) return cuda_fail(e, "eval_host: sync");
    cudaFree(h->d_force);
    h->d_force = nullptr;
    h->force_bytes = 0;
    if (cudaMalloc(&h->d_force, bytes) != cudaSuccess) {
      cudaGetLastError();
      return fail(PME_ENOMEM, "device allocation of the force buffer failed");
    }
    h->force_bytes = bytes;
  }
  if (int rc = ensure_bins(h, ncoord)) return rc;
  const int ev = (calc_energy || calc_virial) ? 1 : 0;
  SysDesc d = h->st.desc9(recip, kappa, xyzq_host, ncoord, h->d_force, kind, stride, ev, calc_energy ? 1 : 0);
  d.ev_mirror = h->ev_mirror;
  d.xyzq_host = 1;
  if (int rc = launch_fused_single(h, d)) return rc;
  // only the written forces travel (the caller's stride padding is left alone), in one copy
  const cudaError_t e =
      kind == PME_FORCE_F32X3
          ? cudaMemcpyAsync(force_host, h->d_force, bytes, cudaMemcpyDeviceToHost, h->stream)
          : cudaMemcpy2DAsync(force_host, (size_t)stride * sizeof(float), h->d_force, (size_t)stride * sizeof(float),
                              (size_t)ncoord * sizeof(float), 3, cudaMemcpyDeviceToHost, h->stream);
  if (e != cudaSuccess) return cuda_fail(e, "eval_host: copy forces");
  return PME_OK;
}

static int copy_back(pme_recip* h, void* dst, const void* src, size_t bytes, const char* what) {
  if (!h || !dst) return fail(PME_EINVAL, "NULL argument");
  DeviceGuard dg(h->device);
  cudaError_t e = cudaStreamSynchronize(h->stream);
  if (e == cudaSuccess) e = cudaMemcpy(dst, src, bytes, cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return cuda_fail(e, what);
  return PME_OK;
}

int pme_copy_charge_grid_fixed(pme_recip* h, long long* host_out) {
  if (int rc = handle_ok(h)) return rc;
  return copy_back(h, host_out, h->st.accum, h->st.G() * 8, "copy_charge_grid_fixed");
}

int pme_copy_charge_grid(pme_recip* h, float* host_out) {
  if (!h || !host_out) return fail(PME_EINVAL, "NULL argument");
  std::vector<long long> tmp(h->st.G());
  int rc = copy_back(h, tmp.data(), h->st.accum, h->st.G() * 8, "copy_charge_grid");
  if (rc) return rc;
  for (size_t i = 0; i < tmp.size(); i++) host_out[i] = (float)tmp[i] * kInvFixedScaleF;   // as fixed_to_float
  return PME_OK;
}

int pme_copy_fft_grid(pme_recip* h, float* host_out) {
  if (!h || !host_out) return fail(PME_EINVAL, "NULL argument");
  const SystemState& s = h->st;
  std::vector<float2> tmp(s.H());
  int rc = copy_back(h, tmp.data(), s.cgrid, s.H() * 8, "copy_fft_grid");
  if (rc) return rc;
  const int hx = s.nx / 2 + 1;
  float2* out = (float2*)host_out;
  for (int kx = 0; kx < hx; kx++)
    for (int z = 0; z < s.nz; z++)
      for (int y = 0; y < s.ny; y++)
        out[((size_t)z * s.ny + y) * hx + kx] = tmp[((size_t)kx * s.nz + z) * s.ny + y];
  return PME_OK;
}

int pme_copy_solved_grid(pme_recip* h, float* host_out) {
  if (int rc = handle_ok(h)) return rc;
  return copy_back(h, host_out, h->st.rgrid, h->st.G() * 4, "copy_solved_grid");
}

int pme_load_charge_grid(pme_recip* h, const float* host_in) {
  if (!h || !host_in) return fail(PME_EINVAL, "NULL argument");
  std::vector<long long> tmp(h->st.G());
  for (size_t i = 0; i < tmp.size(); i++) {
    const double v = (double)host_in[i] * 1099511627776.0;
    if (!(std::fabs(v) < 9.0e18)) return fail(PME_EINVAL, "grid value out of fixed-point range");
    tmp[i] = std::llrint(v);
  }
  DeviceGuard dg(h->device);
  cudaError_t e = cudaStreamSynchronize(h->stream);
  if (e == cudaSuccess) e = cudaMemcpy(h->st.accum, tmp.data(), tmp.size() * 8, cudaMemcpyHostToDevice);
  if (e != cudaSuccess) return cuda_fail(e, "load_charge_grid");
  h->accum_zero = false;
  return PME_OK;
}

int pme_get_status(pme_recip* h, int* device_status) {
  if (int rc = handle_ok(h)) return rc;
  DeviceGuard dg(h->device);
  int status = 0;
  cudaError_t e = cudaMemcpyAsync(&status, h->d_status, sizeof(int), cudaMemcpyDeviceToHost, h->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  if (e != cudaSuccess) return cuda_fail(e, "get_status");
  if (device_status) *device_status = status;
  if (status != kStatusOk) {
    // clear the sticky status, the barrier words, the accumulation grid and the accumulators
    // (an interrupted evaluation leaves them partly filled) so the handle is usable again
    e = cudaMemsetAsync(h->d_bar, 0, kBarWords * sizeof(unsigned long long), h->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(h->st.accum, 0, h->st.G() * 8, h->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(h->st.acc, 0, kAccCount * sizeof(long long), h->stream);
    if (e == cudaSuccess && h->d_bins)
      e = cudaMemsetAsync(h->d_bins, 0, h->st.bin_ints(h->st.atom_cap) * sizeof(int), h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) return cuda_fail(e, "get_status: reset");
    h->accum_zero = true;
    return fail(PME_ETIMEOUT, "a grid barrier of the fused evaluation timed out");
  }
  return PME_OK;
}

int pme_reserve_atoms(pme_recip* h, int natom) {
  if (int rc = handle_ok(h)) return rc;
  if (natom < 0) return fail(PME_EINVAL, "natom must be >= 0");
  DeviceGuard dg(h->device);
  return ensure_bins(h, natom);
}

int pme_set_barrier_spin_limit(pme_recip* h, unsigned int polls) {
  if (int rc = handle_ok(h)) return rc;
  h->spin_limit = polls == 0 ? 1u : polls;
  return PME_OK;
}

int pme_set_fft_schedule(pme_recip* h, int schedule) {
  if (int rc = handle_ok(h)) return rc;
  if (schedule < PME_SCHED_AUTO || schedule > PME_SCHED_CLUSTER) return fail(PME_EINVAL, "unknown schedule");
  h->plane_mode = schedule;
  return PME_OK;
}

int pme_set_x_gather_fusion(pme_recip* h, int mode) {
  if (int rc = handle_ok(h)) return rc;
  if (mode != PME_XGATHER_AUTO && mode != PME_XGATHER_OFF) return fail(PME_EINVAL, "unknown x-gather fusion mode");
  h->x_gather = mode;
  return PME_OK;
}

int pme_set_fault_injection(pme_recip* h, int what) {
  if (int rc = handle_ok(h)) return rc;
  if (what != PME_INJECT_NONE && what != PME_INJECT_SKIP_BARRIER) return fail(PME_EINVAL, "unknown injection");
  h->inject = what;
  return PME_OK;
}

int pme_set_trace(pme_recip* h, unsigned long long* dev_buf, int max_ctas) {
  if (int rc = handle_ok(h)) return rc;
  if (dev_buf && max_ctas <= 0) return fail(PME_EINVAL, "max_ctas must be positive");
  h->trace = dev_buf;
  h->trace_ctas = dev_buf ? max_ctas : 0;
  return PME_OK;
}

const char* pme_last_error_string(void) { return g_err.c_str(); }

const char* pme_status_string(int status) {
  switch (status) {
    case PME_OK: return "PME_OK";
    case PME_EINVAL: return "PME_EINVAL";
    case PME_EUNSUPPORTED: return "PME_EUNSUPPORTED";
    case PME_ECUDA: return "PME_ECUDA";
    case PME_ETIMEOUT: return "PME_ETIMEOUT";
    case PME_ENOMEM: return "PME_ENOMEM";
    case PME_ESTATE: return "PME_ESTATE";
    default: return "PME_UNKNOWN";
  }
}

int pme_version(void) { return 200; }

// ---------------------------------------------------------------------------------------------
// Batches: many independent systems, one persistent launch per evaluation.
// ---------------------------------------------------------------------------------------------
int pme_batch_commit(pme_batch* b);

int pme_batch_destroy(pme_batch* b) {
  if (!b) return PME_OK;
  DeviceGuard dg(b->device);
  cudaFree(b->d_block);
  cudaFree(b->d_desc);
  cudaFree(b->d_bar);
  delete b;
  return PME_OK;
}

int pme_batch_create(const pme_system_desc* systems, int nsys, void* stream, pme_batch** out) {
  if (!out) return fail(PME_EINVAL, "out is NULL");
  *out = nullptr;
  if (!systems || nsys <= 0) return fail(PME_EINVAL, "need at least one system");
  for (int i = 0; i < nsys; i++) {
    const pme_system_desc& s = systems[i];
    if (int rc = check_grid(s.nfftx, s.nffty, s.nfftz, s.order)) return rc;
    if (s.natom < 0 || (s.natom > 0 && !s.xyzq)) return fail(PME_EINVAL, "bad xyzq/natom in a batch system");
    if (!(s.box[0] > 0 && s.box[1] > 0 && s.box[2] > 0) || !(s.kappa > 0))
      return fail(PME_EINVAL, "box edges and kappa must be positive");
    if (int rc = check_force_args(s.natom, s.stride, s.force_kind, s.force)) return rc;
  }
  pme_batch* b = new (std::nothrow) pme_batch();
  if (!b) return fail(PME_ENOMEM, "host allocation failed");
  b->stream = (cudaStream_t)stream;
  cudaError_t e = cudaGetDevice(&b->device);
  size_t max_smem = 0;
  if (e == cudaSuccess) e = configure_kernels(&max_smem);
  if (e != cudaSuccess) { delete b; return cuda_fail(e, "batch: configure kernels"); }
  b->st.resize(nsys);
  std::vector<size_t> off(nsys), boff(nsys);
  size_t total = 0;
  for (int i = 0; i < nsys; i++) {
    b->st[i].setup(systems[i].nfftx, systems[i].nffty, systems[i].nfftz, systems[i].order);
    off[i] = total;
    total += SystemState::bytes(systems[i].nfftx, systems[i].nffty, systems[i].nfftz);
  }
  for (int i = 0; i < nsys; i++) {
    boff[i] = total;
    total += align256(b->st[i].bin_ints(systems[i].natom) * sizeof(int));
  }
  b->bytes = total;
  const size_t table_bytes = align256(sizeof(SysDesc) * nsys) + align256(sizeof(int) * kPhases * (nsys + 1));
  if (cudaMalloc(&b->d_block, total) != cudaSuccess || cudaMalloc(&b->d_desc, table_bytes) != cudaSuccess ||
      cudaMalloc(&b->d_bar, 4 * sizeof(unsigned long long)) != cudaSuccess) {
    cudaGetLastError();
    pme_batch_destroy(b);
    return fail(PME_ENOMEM, "batch: device allocation failed");
  }
  b->d_prefix = (int*)((char*)b->d_desc + align256(sizeof(SysDesc) * nsys));
  b->d_status = (int*)(b->d_bar + 2);
  e = cudaMemset(b->d_block, 0, total);
  if (e == cudaSuccess) e = cudaMemset(b->d_bar, 0, 4 * sizeof(unsigned long long));
  for (int i = 0; i < nsys && e == cudaSuccess; i++) {
    b->st[i].carve(b->d_block + off[i]);
    b->st[i].bins = (int*)(b->d_block + boff[i]);
    b->st[i].atom_cap = std::max(systems[i].natom, 1);
    b->st[i].bin_cap = SystemState::cap_for(b->st[i].atom_cap, b->st[i].nbins());
    e = b->st[i].upload_tables();
  }
  if (e != cudaSuccess) {
    pme_batch_destroy(b);
    return cuda_fail(e, "batch: initialise buffers");
  }
  b->desc.resize(nsys);
  for (int i = 0; i < nsys; i++) {
    const pme_system_desc& s = systems[i];
    const double r3[3] = {1.0 / s.box[0], 1.0 / s.box[1], 1.0 / s.box[2]};
    const int ev = (s.calc_energy || s.calc_virial) ? 1 : 0;
    b->desc[i] = b->st[i].desc(r3, s.kappa, s.xyzq, s.natom, s.force, s.force_kind, s.stride, ev,
                               s.calc_energy ? 1 : 0);
  }
  int rc = pme_batch_commit(b);
  if (rc) {
    pme_batch_destroy(b);
    return rc;
  }
  *out = b;
  return PME_OK;
}

int pme_batch_commit(pme_batch* b) {
  if (!b) return fail(PME_EINVAL, "batch is NULL");
  DeviceGuard dg(b->device);
  const int nsys = (int)b->desc.size();
  std::vector<int> prefix((size_t)kPhases * (nsys + 1), 0);
  size_t smem = 0;
  for (int i = 0; i < nsys; i++) {
    const SystemState& st = b->st[i];
    b->desc[i].plane = (st.plane && b->plane_mode != PME_SCHED_PASSES) ? 1 : 0;
    b->desc[i].tx_rows = scaled_lines(st.nx, st.tx_rows, b->line_scale, 64, 0);
    b->desc[i].tx_y = scaled_lines(st.ny, st.tx_y, b->line_scale, 64, 0);
    b->desc[i].tx_z = scaled_lines(st.nz, st.tx_z, b->line_scale, std::max(st.tx_z, st.ny),
                                   ktab_smem_bytes(st.ny, st.nz));
    int cnt[kPhases];
    fused_tile_counts(b->desc[i], cnt);
    for (int p = 0; p < kPhases; p++)
      prefix[(size_t)p * (nsys + 1) + i + 1] = prefix[(size_t)p * (nsys + 1) + i] + cnt[p];
    smem = std::max(smem, fused_smem_bytes(b->desc[i]));
  }
  for (int p = 0; p < kPhases; p++) b->total[p] = prefix[(size_t)p * (nsys + 1) + nsys];
  for (int i = 0; i < nsys; i++) b->desc[i].gsort = gather_sorts(b->desc[i], smem);
  cudaError_t e = cudaStreamSynchronize(b->stream);
  if (e == cudaSuccess) e = cudaMemcpy(b->d_desc, b->desc.data(), sizeof(SysDesc) * nsys, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(b->d_prefix, prefix.data(), prefix.size() * sizeof(int), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) return cuda_fail(e, "batch: upload descriptors");
  b->smem = smem;
  e = fused_shape(b->total, smem, b->grid_cap, &b->shape);
  if (e != cudaSuccess) return cuda_fail(e, "batch: launch shape (does the kernel fit on an SM?)");
  return PME_OK;
}

int pme_batch_set_system(pme_batch* b, int sys, const double* box3, const void* xyzq, void* force) {
  if (!b || sys < 0 || sys >= (int)b->desc.size()) return fail(PME_EINVAL, "bad batch or system index");
  SysDesc& d = b->desc[sys];
  if (box3) {
    if (!(box3[0] > 0 && box3[1] > 0 && box3[2] > 0)) return fail(PME_EINVAL, "box edges must be positive");
    const double r3[3] = {1.0 / box3[0], 1.0 / box3[1], 1.0 / box3[2]};
    const double kappa = kPi / std::sqrt(d.fac);
    d = b->st[sys].desc(r3, kappa, d.xyzq, d.natom, d.force, d.force_kind, d.stride, d.calc_ev, d.calc_self);
  }
  if (xyzq) d.xyzq = (const float4*)xyzq;
  if (force) d.force = force;
  return PME_OK;
}

int pme_batch_eval(pme_batch* b) {
  if (!b) return fail(PME_EINVAL, "batch is NULL");
  DeviceGuard dg(b->device);
  FusedArgs a;
  std::memset(&a, 0, sizeof(a));
  a.table = b->d_desc;
  a.nsys = (int)b->desc.size();
  a.prefix = b->d_prefix;
  for (int p = 0; p < kPhases; p++) a.total[p] = b->total[p];
  a.nbar = fused_barriers(a.total);
  a.bar = b->d_bar;
  a.status = b->d_status;
  a.spin_limit = b->spin_limit;
  a.trace = b->trace;
  a.trace_ctas = b->trace_ctas;
  cudaError_t e = fused_launch(a, b->shape, b->smem, b->stream);
  if (e != cudaSuccess) return cuda_fail(e, "batch eval launch");
  return PME_OK;
}

int pme_batch_clear_energy_virial(pme_batch* b) {
  if (!b) return fail(PME_EINVAL, "batch is NULL");
  DeviceGuard dg(b->device);
  cudaError_t e = clear_records(b->d_desc, (int)b->desc.size(), b->stream);
  if (e != cudaSuccess) return cuda_fail(e, "batch clear");
  return PME_OK;
}

int pme_batch_get_energy_virial(pme_batch* b, double* out) {
  if (!b || !out) return fail(PME_EINVAL, "NULL argument");
  DeviceGuard dg(b->device);
  int status = 0;
  cudaError_t e = cudaSuccess;
  for (size_t i = 0; i < b->st.size() && e == cudaSuccess; i++)
    e = cudaMemcpyAsync(out + i * kEvCount, b->st[i].ev, kEvCount * sizeof(double), cudaMemcpyDeviceToHost,
                        b->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(&status, b->d_status, sizeof(int), cudaMemcpyDeviceToHost, b->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(b->stream);
  if (e != cudaSuccess) return cuda_fail(e, "batch get energy/virial");
  if (status != kStatusOk) return fail(PME_ETIMEOUT, "a grid barrier of the batch evaluation timed out");
  return PME_OK;
}

int pme_batch_info(const pme_batch* b, int* nsys, int* grid, size_t* device_bytes) {
  if (!b) return fail(PME_EINVAL, "batch is NULL");
  if (nsys) *nsys = (int)b->desc.size();
  if (grid) *grid = b->shape.grid;
  if (device_bytes) *device_bytes = b->bytes;
  return PME_OK;
}

int pme_batch_set_stream(pme_batch* b, void* stream) {
  if (!b) return fail(PME_EINVAL, "batch is NULL");
  b->stream = (cudaStream_t)stream;
  return PME_OK;
}

int pme_batch_set_trace(pme_batch* b, unsigned long long* dev_buf, int max_ctas) {
  if (!b) return fail(PME_EINVAL, "batch is NULL");
  if (dev_buf && max_ctas <= 0) return fail(PME_EINVAL, "max_ctas must be positive");
  b->trace = dev_buf;
  b->trace_ctas = dev_buf ? max_ctas : 0;
  return PME_OK;
}

size_t pme_system_device_bytes(int nfftx, int nffty, int nfftz) {
  return SystemState::bytes(nfftx, nffty, nfftz);
}

}  // extern "C"

// ---------------------------------------------------------------------------------------------
// Autotuner: coordinate descent over the fused evaluation's launch shape, timed with CUDA events
// on the stream the evaluations run on.  Every shape computes the same bits, so the search may
// keep whichever is fastest on this GPU for this system.
// ---------------------------------------------------------------------------------------------
namespace {

struct EventPair {
  cudaEvent_t a = nullptr, b = nullptr;
  cudaError_t init() {
    cudaError_t e = cudaEventCreate(&a);
    return e == cudaSuccess ? cudaEventCreate(&b) : e;
  }
  ~EventPair() {
    if (a) cudaEventDestroy(a);
    if (b) cudaEventDestroy(b);
  }
};

// Mean time (us) of `reps` back-to-back launches of `launch` after two untimed ones; fails if a
// grid barrier of the fused kernel gave up.
template <class F>
int time_launches(F launch, cudaStream_t stream, const int* d_status, int reps, EventPair& ev, float* us) {
  for (int i = 0; i < 2; i++)
    if (int rc = launch()) return rc;
  cudaError_t e = cudaEventRecord(ev.a, stream);
  for (int i = 0; i < reps && e == cudaSuccess; i++)
    if (int rc = launch()) return rc;
  if (e == cudaSuccess) e = cudaEventRecord(ev.b, stream);
  if (e == cudaSuccess) e = cudaEventSynchronize(ev.b);
  float ms = 0.0f;
  if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, ev.a, ev.b);
  int status = 0;
  if (e == cudaSuccess) e = cudaMemcpy(&status, d_status, sizeof(int), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return cuda_fail(e, "autotune: timing");
  if (status != kStatusOk) return fail(PME_ETIMEOUT, "autotune: a grid barrier of the fused kernel timed out");
  *us = ms * 1000.0f / (float)reps;
  return PME_OK;
}

std::vector<int> line_values(int cur) {
  std::vector<int> v = {4, 8, 16, 32};
  if (std::find(v.begin(), v.end(), cur) == v.end()) v.push_back(cur);
  return v;
}

int sm_count(int dev) {
  int sms = 0;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms < 1) sms = 1;
  return sms;
}

}  // namespace

extern "C" {

int pme_get_tune_config(const pme_recip* h, pme_tune_config* out) {
  if (!h || !out) return fail(PME_EINVAL, "NULL argument");
  get_config(h, out);
  return PME_OK;
}

int pme_set_tune_config(pme_recip* h, const pme_tune_config* cfg) {
  if (!h || !cfg) return fail(PME_EINVAL, "NULL argument");
  if (!config_fits(h->st, *cfg)) return fail(PME_EINVAL, "launch shape out of range or over the shared-memory budget");
  set_config(h, *cfg);
  return PME_OK;
}

int pme_tune_cache_clear(void) {
  std::lock_guard<std::mutex> lock(g_tune_mutex);
  g_tune_cache.clear();
  return PME_OK;
}

int pme_autotune(pme_recip* h, const void* xyzq, int ncoord, double inv_boxx, double inv_boxy, double inv_boxz,
                 double kappa, int reps, pme_tune_config* out) {
  if (int rc = handle_ok(h)) return rc;
  if (ncoord < 0 || (ncoord > 0 && !xyzq)) return fail(PME_EINVAL, "bad xyzq/ncoord");
  const double recip[9] = {inv_boxx, 0, 0, 0, inv_boxy, 0, 0, 0, inv_boxz};
  if (int rc = check_recip(recip)) return rc;
  if (!(kappa > 0.0) || !std::isfinite(kappa)) return fail(PME_EINVAL, "kappa must be positive");
  if (reps < 1 || reps > 100000) return fail(PME_EINVAL, "reps must be in [1, 100000]");
  DeviceGuard dg(h->device);
  cudaError_t e = cudaSuccess;
  if (int rc = ensure_bins(h, ncoord)) return rc;
  // scratch force output and the energy/virial record to put back afterwards
  const int stride = std::max(ncoord, 1);
  float* force = nullptr;
  if (cudaMalloc(&force, 3 * (size_t)stride * sizeof(float)) != cudaSuccess) {
    cudaGetLastError();
    return fail(PME_ENOMEM, "autotune: scratch force allocation failed");
  }
  double saved[kEvCount];
  e = cudaStreamSynchronize(h->stream);
  if (e == cudaSuccess) e = cudaMemcpy(saved, h->st.ev, sizeof(saved), cudaMemcpyDeviceToHost);
  EventPair ev;
  if (e == cudaSuccess) e = ev.init();
  if (e != cudaSuccess) {
    cudaFree(force);
    return cuda_fail(e, "autotune: setup");
  }
  const double r3[3] = {inv_boxx, inv_boxy, inv_boxz};
  auto measure = [&](const pme_tune_config& c, float* us) {
    set_config(h, c);
    const SysDesc d = h->st.desc(r3, kappa, xyzq, ncoord, force, PME_FORCE_F32_SOA, stride, 1, 1);
    return time_launches([&]() { return launch_fused_single(h, d); }, h->stream, h->d_status, reps, ev, us);
  };
  pme_tune_config best;
  get_config(h, &best);
  const pme_tune_config start = best;
  float best_us = 0.0f;
  int count = 1;
  int rc = measure(best, &best_us);
  const int sms = sm_count(h->device);
  for (int sweep = 0; sweep < 2 && rc == PME_OK; sweep++) {
    bool improved = false;
    for (int knob = 0; knob < 5 && rc == PME_OK; knob++) {
      std::vector<int> vals;
      if (knob == 0) {
        vals = h->st.plane ? std::vector<int>{PME_SCHED_PLANES, PME_SCHED_PASSES} : std::vector<int>{PME_SCHED_PASSES};
        vals.push_back(PME_SCHED_CLUSTER);
      }
      else if (knob == 1) vals = line_values(best.z_columns);
      else if (knob == 2) vals = line_values(best.y_lines);
      else if (knob == 3) vals = line_values(best.x_lines);
      else vals = {0, sms};
      for (int v : vals) {
        pme_tune_config c = best;
        int* field = knob == 0 ? &c.schedule : knob == 1 ? &c.z_columns : knob == 2 ? &c.y_lines
                   : knob == 3 ? &c.x_lines : &c.grid_ctas;
        if (*field == v) continue;
        *field = v;
        if (!config_fits(h->st, c)) continue;
        float us = 0.0f;
        rc = measure(c, &us);
        if (rc) break;
        count++;
        if (us < 0.98f * best_us) {
          best = c;
          best_us = us;
          improved = true;
        }
      }
    }
    if (!improved) break;
  }
  set_config(h, rc == PME_OK ? best : start);
  e = cudaStreamSynchronize(h->stream);
  if (e == cudaSuccess) e = cudaMemcpy(h->st.ev, saved, sizeof(saved), cudaMemcpyHostToDevice);
  cudaFree(force);
  if (rc) return rc;
  if (e != cudaSuccess) return cuda_fail(e, "autotune: restore energy/virial");
  best.us_per_eval = best_us;
  best.candidates = count;
  {
    std::lock_guard<std::mutex> lock(g_tune_mutex);
    g_tune_cache[tune_key(h)] = best;
  }
  if (out) *out = best;
  return PME_OK;
}

int pme_batch_autotune(pme_batch* b, int reps, pme_tune_config* out) {
  if (!b) return fail(PME_EINVAL, "batch is NULL");
  if (reps < 1 || reps > 100000) return fail(PME_EINVAL, "reps must be in [1, 100000]");
  DeviceGuard dg(b->device);
  const size_t nsys = b->st.size();
  std::vector<double> saved(nsys * kEvCount);
  cudaError_t e = cudaStreamSynchronize(b->stream);
  for (size_t i = 0; i < nsys && e == cudaSuccess; i++)
    e = cudaMemcpy(&saved[i * kEvCount], b->st[i].ev, kEvCount * sizeof(double), cudaMemcpyDeviceToHost);
  EventPair ev;
  if (e == cudaSuccess) e = ev.init();
  if (e != cudaSuccess) return cuda_fail(e, "batch autotune: setup");
  const int sms = sm_count(b->device);
  const int start_mode = b->plane_mode, start_cap = b->grid_cap, start_scale = b->line_scale;
  int best_mode = start_mode, best_cap = start_cap, best_scale = start_scale, count = 0, rc = PME_OK;
  float best_us = 0.0f;
  for (int scale : {1, 2, 4}) {
    for (int mode : {PME_SCHED_AUTO, PME_SCHED_PASSES}) {
      for (int cap : {0, sms}) {
        b->plane_mode = mode;
        b->grid_cap = cap;
        b->line_scale = scale;
        if ((rc = pme_batch_commit(b))) break;
        float us = 0.0f;
        rc = time_launches([&]() { return pme_batch_eval(b); }, b->stream, b->d_status, reps, ev, &us);
        if (rc) break;
        if (count == 0 || us < 0.98f * best_us) {
          best_us = us;
          best_mode = mode;
          best_cap = cap;
          best_scale = scale;
        }
        count++;
      }
      if (rc) break;
    }
    if (rc) break;
  }
  b->plane_mode = rc == PME_OK ? best_mode : start_mode;
  b->grid_cap = rc == PME_OK ? best_cap : start_cap;
  b->line_scale = rc == PME_OK ? best_scale : start_scale;
  const int rc2 = pme_batch_commit(b);
  e = cudaStreamSynchronize(b->stream);
  for (size_t i = 0; i < nsys && e == cudaSuccess; i++)
    e = cudaMemcpy(b->st[i].ev, &saved[i * kEvCount], kEvCount * sizeof(double), cudaMemcpyHostToDevice);
  if (rc) return rc;
  if (rc2) return rc2;
  if (e != cudaSuccess) return cuda_fail(e, "batch autotune: restore energy/virial");
  if (out) {
    std::memset(out, 0, sizeof(*out));
    out->schedule = best_mode;
    out->grid_ctas = best_cap;
    out->x_lines = out->y_lines = out->z_columns = best_scale;   // multiplier of each system's default
    out->us_per_eval = best_us;
    out->candidates = count;
  }
  return PME_OK;
}

}  // extern "C"

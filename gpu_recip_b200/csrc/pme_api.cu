// pme_api.cu -- host engine and C ABI of the B200 smooth-PME reciprocal-space operator.
//
// One pme_recip instance mirrors one CudaPMERecip<long long, float, float2> of the reference
// (CudaPMERecip.h:37-205): it owns the int64 accumulation grid, the half-complex FFT grid, the
// solved real grid, per-axis FFT plans with FP64-accurate twiddles, the FP64-computed B-spline
// moduli (stored FP32) and the energy/virial record.  Every compute call only enqueues kernels
// on the instance's stream: no allocation, no host synchronisation, so a whole evaluation can
// be captured in a CUDA graph.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "../../include/pme_recip.h"
#include "pme_internal.h"

namespace pme {
cudaError_t configure_kernels();
}

using namespace pme;

struct pme_recip {
  int nx, ny, nz, order, fft_type, device;
  cudaStream_t stream;
  FftPlan1D px, py, pz;
  PassTiling tile_x, tile_y, tile_z;
  long long* d_accum;
  float2* d_cgrid;
  float* d_rgrid;
  float2* d_tw;
  float* d_bmod;
  double* d_ev;
  double* d_partials;
  unsigned int* d_ticket;
  int max_blocks;
};

namespace {

thread_local std::string g_err;

int fail(int status, const std::string& msg) {
  g_err = msg;
  return status;
}

int cuda_fail(cudaError_t e, const char* where) {
  return fail(PME_ECUDA, std::string(where) + ": " + cudaGetErrorString(e));
}

// Restores the caller's current device on scope exit.
struct DeviceGuard {
  int prev = -1;
  bool changed = false;
  explicit DeviceGuard(int dev) {
    if (cudaGetDevice(&prev) == cudaSuccess && prev != dev) {
      changed = (cudaSetDevice(dev) == cudaSuccess);
    }
  }
  ~DeviceGuard() {
    if (changed) cudaSetDevice(prev);
  }
};

bool factorize(int n, FftPlan1D& p) {
  p.n = n;
  p.nstages = 0;
  int m = n;
  auto push = [&](int r) {
    if (p.nstages >= kMaxStages) return false;
    p.radix[p.nstages++] = r;
    m /= r;
    return true;
  };
  while (m % 4 == 0) if (!push(4)) return false;
  while (m % 2 == 0) if (!push(2)) return false;
  while (m % 3 == 0) if (!push(3)) return false;
  while (m % 5 == 0) if (!push(5)) return false;
  return m == 1;
}

// Cardinal B-spline weights at u (FP64) by the same recursion as the kernels.
void bspline_host(int p, double u, double* th) {
  for (int i = 0; i < p; i++) th[i] = 0.0;
  th[0] = 1.0 - u;
  th[1] = u;
  for (int k = 3; k <= p; k++) {
    double d = 1.0 / (double)(k - 1);
    th[k - 1] = d * u * th[k - 2];
    for (int j = 1; j <= k - 2; j++)
      th[k - j - 1] = d * ((u + j) * th[k - j - 2] + ((k - j) - u) * th[k - j - 1]);
    th[0] = d * (1.0 - u) * th[0];
  }
}

// B-spline moduli 1/|b(k)|^2 in FP64 (CudaPMERecip.cu:2481-2505 dftmod, :2543-2579 calc_prefac):
// DFT over j = 0..n-2 of M = [0, theta_0(0), ..., theta_{p-1}(0), 0, ...]; values below 1e-10
// take the mean of their neighbours.
void bspline_moduli(int p, int n, std::vector<float>& out) {
  std::vector<double> arr((size_t)std::max(n, p + 2), 0.0), th(p), mod(n);
  bspline_host(p, 0.0, th.data());
  for (int i = 1; i <= p; i++) arr[i] = th[i - 1];
  for (int k = 0; k < n; k++) {
    double s1 = 0.0, s2 = 0.0;
    for (int j = 0; j < n - 1; j++) {
      double a = 2.0 * kPi * (double)k * (double)j / (double)n;
      s1 += arr[j] * std::cos(a);
      s2 += arr[j] * std::sin(a);
    }
    mod[k] = s1 * s1 + s2 * s2;
  }
  for (int k = 0; k < n; k++)
    if (mod[k] < 1.0e-10) mod[k] = 0.5 * (mod[(k - 1 + n) % n] + mod[(k + 1) % n]);
  out.resize(n);
  for (int k = 0; k < n; k++) out[k] = (float)(1.0 / mod[k]);
}

PassTiling pick_tiling_rows(int L) {
  PassTiling t;
  t.tx = 16;
  // keep the tile's two buffers within ~200 KB of shared memory
  while (t.tx > 1 && sizeof(float2) * ((size_t)L + 2 * (size_t)L * (t.tx + 1)) > 200 * 1024) t.tx--;
  t.ny = 0;
  return t;
}

PassTiling pick_tiling_cols(int hx, int L) {
  PassTiling best;
  best.tx = 16;
  best.ny = 0;
  int best_waste = 1 << 30;
  for (int tx = 17; tx >= 8; tx--) {
    int tiles = (hx + tx - 1) / tx;
    int waste = tiles * tx - hx;
    if (waste < best_waste) {
      best_waste = waste;
      best.tx = tx;
    }
  }
  if (hx < 8) best.tx = hx;
  while (best.tx > 1 && sizeof(float2) * ((size_t)L + 2 * (size_t)L * (best.tx + 1)) > 200 * 1024)
    best.tx--;
  return best;
}

bool is_ortho(const double* r) {
  return r[1] == 0.0 && r[2] == 0.0 && r[3] == 0.0 && r[5] == 0.0 && r[6] == 0.0 && r[7] == 0.0;
}

int check_recip(const double* recip) {
  if (!recip) return fail(PME_EINVAL, "recip is NULL");
  if (!is_ortho(recip))
    return fail(PME_EINVAL, "only orthorhombic boxes are supported (recip off-diagonals must be 0)");
  if (!(recip[0] > 0.0 && recip[4] > 0.0 && recip[8] > 0.0) || !std::isfinite(recip[0]) ||
      !std::isfinite(recip[4]) || !std::isfinite(recip[8]))
    return fail(PME_EINVAL, "recip diagonal must be finite and positive");
  return PME_OK;
}

Geom make_geom(const pme_recip* h, const double* recip) {
  Geom g;
  g.nx = h->nx; g.ny = h->ny; g.nz = h->nz;
  g.hx = h->nx / 2 + 1;
  g.rx = recip ? (float)recip[0] : 0.0f;
  g.ry = recip ? (float)recip[4] : 0.0f;
  g.rz = recip ? (float)recip[8] : 0.0f;
  return g;
}

ReduceScratch scratch(const pme_recip* h) {
  ReduceScratch rs;
  rs.partials = h->d_partials;
  rs.ticket = h->d_ticket;
  rs.max_blocks = h->max_blocks;
  return rs;
}

enum { kSiteSolve = 0, kSiteSelf = 1, kNumSites = 4 };

void release(pme_recip* h) {
  if (!h) return;
  cudaFree(h->d_accum);
  cudaFree(h->d_cgrid);
  cudaFree(h->d_rgrid);
  cudaFree(h->d_tw);
  cudaFree(h->d_bmod);
  cudaFree(h->d_ev);
  cudaFree(h->d_partials);
  cudaFree(h->d_ticket);
  delete h;
}

int upload_moduli(pme_recip* h) {
  std::vector<float> bx, by, bz;
  bspline_moduli(h->order, h->nx, bx);
  bspline_moduli(h->order, h->ny, by);
  bspline_moduli(h->order, h->nz, bz);
  std::vector<float> all;
  all.insert(all.end(), bx.begin(), bx.end());
  all.insert(all.end(), by.begin(), by.end());
  all.insert(all.end(), bz.begin(), bz.end());
  cudaError_t e = cudaMemcpy(h->d_bmod, all.data(), all.size() * sizeof(float),
                             cudaMemcpyHostToDevice);
  if (e != cudaSuccess) return cuda_fail(e, "upload moduli");
  return PME_OK;
}

SolveParams solve_params(const pme_recip* h, const double* recip, double kappa, int calc_ev) {
  SolveParams sp;
  const double inv_vol = recip[0] * recip[4] * recip[8];
  sp.fac = (float)(kPi * kPi / (kappa * kappa));
  sp.piv_inv = (float)(inv_vol / kPi);
  sp.bmx = h->d_bmod;
  sp.bmy = h->d_bmod + h->nx;
  sp.bmz = h->d_bmod + h->nx + h->ny;
  sp.calc_ev = calc_ev;
  sp.ev = h->d_ev;
  return sp;
}

int valid_order(int order) { return order == 4 || order == 6 || order == 8; }

// Enqueue helpers shared by the staged and fused paths.
int enqueue_spread(pme_recip* h, const void* xyzq, int ncoord, const Geom& g) {
  const size_t G = (size_t)h->nx * h->ny * h->nz;
  cudaError_t e = cudaMemsetAsync(h->d_accum, 0, G * sizeof(long long), h->stream);
  if (e != cudaSuccess) return cuda_fail(e, "spread_charge: clear grid");
  e = launch_spread((const float4*)xyzq, ncoord, g, h->order, (unsigned long long*)h->d_accum,
                    h->stream);
  if (e != cudaSuccess) return cuda_fail(e, "spread_charge");
  return PME_OK;
}

int enqueue_r2c(pme_recip* h, const Geom& g) {
  cudaError_t e = launch_x_r2c(h->d_accum, h->d_cgrid, g, h->px, h->d_tw, h->tile_x, h->stream);
  if (e != cudaSuccess) return cuda_fail(e, "r2c_fft: x pass");
  e = launch_c2c(h->d_cgrid, g, 1, 0, h->py, h->d_tw, h->tile_y, nullptr, scratch(h), 0, h->stream);
  if (e != cudaSuccess) return cuda_fail(e, "r2c_fft: y pass");
  return PME_OK;
}

int enqueue_c2r_tail(pme_recip* h, const Geom& g) {
  cudaError_t e =
      launch_c2c(h->d_cgrid, g, 1, 1, h->py, h->d_tw, h->tile_y, nullptr, scratch(h), 0, h->stream);
  if (e != cudaSuccess) return cuda_fail(e, "c2r_fft: y pass");
  e = launch_x_c2r(h->d_cgrid, h->d_rgrid, g, h->px, h->d_tw, h->tile_x, h->stream);
  if (e != cudaSuccess) return cuda_fail(e, "c2r_fft: x pass");
  return PME_OK;
}

int check_force_args(int ncoord, int stride, int kind, const void* force) {
  if (kind != PME_FORCE_F32_SOA && kind != PME_FORCE_F32X3 && kind != PME_FORCE_I64_SOA_ACCUM)
    return fail(PME_EINVAL, "unknown force kind");
  if (ncoord > 0 && !force) return fail(PME_EINVAL, "force is NULL");
  if (kind != PME_FORCE_F32X3 && ncoord > 0 && stride < ncoord)
    return fail(PME_EINVAL, "stride must be >= ncoord for strided force layouts");
  return PME_OK;
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
  if (!valid_order(order)) return fail(PME_EINVAL, "order must be 4, 6 or 8");
  const int n3[3] = {nfftx, nffty, nfftz};
  for (int d = 0; d < 3; d++) {
    if (n3[d] < order || n3[d] > kMaxFftLen)
      return fail(PME_EINVAL, "grid lengths must be in [order, 512]");
  }
  pme_recip* h = new (std::nothrow) pme_recip();
  if (!h) return fail(PME_ENOMEM, "host allocation failed");
  std::memset(h, 0, sizeof(*h));
  h->nx = nfftx; h->ny = nffty; h->nz = nfftz;
  h->order = order;
  h->fft_type = fft_type;
  h->stream = (cudaStream_t)stream;
  if (!factorize(nfftx, h->px) || !factorize(nffty, h->py) || !factorize(nfftz, h->pz)) {
    delete h;
    return fail(PME_EUNSUPPORTED, "grid lengths must factor into 2, 3 and 5");
  }
  cudaError_t e = cudaGetDevice(&h->device);
  if (e != cudaSuccess) { delete h; return cuda_fail(e, "cudaGetDevice"); }
  e = configure_kernels();
  if (e != cudaSuccess) { delete h; return cuda_fail(e, "configure kernels"); }

  h->px.tw_off = 0;
  h->py.tw_off = nfftx;
  h->pz.tw_off = nfftx + nffty;
  const int hx = nfftx / 2 + 1;
  h->tile_x = pick_tiling_rows(nfftx);
  h->tile_y = pick_tiling_cols(hx, nffty);
  h->tile_z = pick_tiling_cols(hx, nfftz);

  const size_t G = (size_t)nfftx * nffty * nfftz;
  const size_t H = (size_t)hx * nffty * nfftz;
  Geom g0 = make_geom(h, nullptr);
  const int zblocks = c2c_num_blocks(g0, 2, h->tile_z);
  h->max_blocks = zblocks > 1024 ? zblocks : 1024;

  bool ok = cudaMalloc(&h->d_accum, G * sizeof(long long)) == cudaSuccess &&
            cudaMalloc(&h->d_cgrid, H * sizeof(float2)) == cudaSuccess &&
            cudaMalloc(&h->d_rgrid, G * sizeof(float)) == cudaSuccess &&
            cudaMalloc(&h->d_tw, (size_t)(nfftx + nffty + nfftz) * sizeof(float2)) == cudaSuccess &&
            cudaMalloc(&h->d_bmod, (size_t)(nfftx + nffty + nfftz) * sizeof(float)) == cudaSuccess &&
            cudaMalloc(&h->d_ev, PME_EV_COUNT * sizeof(double)) == cudaSuccess &&
            cudaMalloc(&h->d_partials, (size_t)h->max_blocks * 8 * sizeof(double)) == cudaSuccess &&
            cudaMalloc(&h->d_ticket, kNumSites * sizeof(unsigned int)) == cudaSuccess;
  if (!ok) {
    cudaGetLastError();
    release(h);
    return fail(PME_ENOMEM, "device allocation failed");
  }
  // twiddles W_n^k = exp(-2 pi i k/n), FP64 -> FP32
  std::vector<float2> tw;
  for (int d = 0; d < 3; d++) {
    const int n = n3[d];
    for (int k = 0; k < n; k++) {
      const double a = -2.0 * kPi * (double)k / (double)n;
      tw.push_back(make_float2((float)std::cos(a), (float)std::sin(a)));
    }
  }
  e = cudaMemcpy(h->d_tw, tw.data(), tw.size() * sizeof(float2), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemset(h->d_ev, 0, PME_EV_COUNT * sizeof(double));
  if (e == cudaSuccess) e = cudaMemset(h->d_ticket, 0, kNumSites * sizeof(unsigned int));
  if (e == cudaSuccess) e = cudaMemset(h->d_accum, 0, G * sizeof(long long));
  if (e == cudaSuccess) e = cudaMemset(h->d_cgrid, 0, H * sizeof(float2));
  if (e == cudaSuccess) e = cudaMemset(h->d_rgrid, 0, G * sizeof(float));
  if (e != cudaSuccess) {
    release(h);
    return cuda_fail(e, "pme_create: initialise buffers");
  }
  int rc = upload_moduli(h);
  if (rc != PME_OK) {
    release(h);
    return rc;
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
  if (!h) return fail(PME_EINVAL, "handle is NULL");
  h->stream = (cudaStream_t)stream;
  return PME_OK;
}

int pme_set_order(pme_recip* h, int order) {
  if (!h) return fail(PME_EINVAL, "handle is NULL");
  if (!valid_order(order)) return fail(PME_EINVAL, "order must be 4, 6 or 8");
  if (h->nx < order || h->ny < order || h->nz < order)
    return fail(PME_EINVAL, "grid lengths must be >= order");
  DeviceGuard dg(h->device);
  // moduli are uploaded synchronously after the stream's pending work
  cudaError_t e = cudaStreamSynchronize(h->stream);
  if (e != cudaSuccess) return cuda_fail(e, "set_order");
  h->order = order;
  return upload_moduli(h);
}

int pme_get_nfft(const pme_recip* h, int* nx, int* ny, int* nz) {
  if (!h) return fail(PME_EINVAL, "handle is NULL");
  if (nx) *nx = h->nx;
  if (ny) *ny = h->ny;
  if (nz) *nz = h->nz;
  return PME_OK;
}

int pme_get_order(const pme_recip* h, int* order) {
  if (!h || !order) return fail(PME_EINVAL, "NULL argument");
  *order = h->order;
  return PME_OK;
}

int pme_print_info(const pme_recip* h) {
  if (!h) return fail(PME_EINVAL, "handle is NULL");
  const char* ft = h->fft_type == PME_FFT_COLUMN ? "COLUMN" : (h->fft_type == PME_FFT_SLAB ? "SLAB" : "BOX");
  std::printf("fft_type = %s computed using the built-in sm_100a 2/3/5-radix FFT\n", ft);
  std::printf("order = %d\n", h->order);
  std::printf("nfftx, nffty, nfftz = %d %d %d\n", h->nx, h->ny, h->nz);
  std::printf("x0...x1   = 0 ... %d\ny0...y1   = 0 ... %d\nz0...z1   = 0 ... %d\n", h->nx - 1,
              h->ny - 1, h->nz - 1);
  std::printf("xsize, ysize, zsize = %d %d %d\n", h->nx, h->ny, h->nz);
  std::printf("data_size = %d\n", 2 * (h->nx / 2 + 1) * h->ny * h->nz);
  std::printf("tiles: x %d, y %d, z %d lines per CTA\n", h->tile_x.tx, h->tile_y.tx, h->tile_z.tx);
  std::fflush(stdout);
  return PME_OK;
}

int pme_spread_charge(pme_recip* h, const void* xyzq, int ncoord, const double* recip) {
  if (!h) return fail(PME_EINVAL, "handle is NULL");
  if (ncoord < 0 || (ncoord > 0 && !xyzq)) return fail(PME_EINVAL, "bad xyzq/ncoord");
  int rc = check_recip(recip);
  if (rc) return rc;
  DeviceGuard dg(h->device);
  return enqueue_spread(h, xyzq, ncoord, make_geom(h, recip));
}

int pme_r2c_fft(pme_recip* h) {
  if (!h) return fail(PME_EINVAL, "handle is NULL");
  DeviceGuard dg(h->device);
  Geom g = make_geom(h, nullptr);
  int rc = enqueue_r2c(h, g);
  if (rc) return rc;
  cudaError_t e =
      launch_c2c(h->d_cgrid, g, 2, 0, h->pz, h->d_tw, h->tile_z, nullptr, scratch(h), 0, h->stream);
  if (e != cudaSuccess) return cuda_fail(e, "r2c_fft: z pass");
  return PME_OK;
}

int pme_scalar_sum(pme_recip* h, const double* recip, double kappa, int calc_energy,
                   int calc_virial) {
  if (!h) return fail(PME_EINVAL, "handle is NULL");
  int rc = check_recip(recip);
  if (rc) return rc;
  if (!(kappa > 0.0) || !std::isfinite(kappa)) return fail(PME_EINVAL, "kappa must be positive");
  DeviceGuard dg(h->device);
  Geom g = make_geom(h, recip);
  SolveParams sp = solve_params(h, recip, kappa, (calc_energy || calc_virial) ? 1 : 0);
  cudaError_t e =
      launch_c2c(h->d_cgrid, g, 2, 3, h->pz, h->d_tw, h->tile_z, &sp, scratch(h), kSiteSolve, h->stream);
  if (e != cudaSuccess) return cuda_fail(e, "scalar_sum");
  return PME_OK;
}

int pme_c2r_fft(pme_recip* h) {
  if (!h) return fail(PME_EINVAL, "handle is NULL");
  DeviceGuard dg(h->device);
  Geom g = make_geom(h, nullptr);
  cudaError_t e =
      launch_c2c(h->d_cgrid, g, 2, 1, h->pz, h->d_tw, h->tile_z, nullptr, scratch(h), 0, h->stream);
  if (e != cudaSuccess) return cuda_fail(e, "c2r_fft: z pass");
  return enqueue_c2r_tail(h, g);
}

int pme_gather_force(pme_recip* h, const void* xyzq, int ncoord, const double* recip, int stride,
                     int kind, void* force) {
  if (!h) return fail(PME_EINVAL, "handle is NULL");
  if (ncoord < 0 || (ncoord > 0 && !xyzq)) return fail(PME_EINVAL, "bad xyzq/ncoord");
  int rc = check_recip(recip);
  if (rc) return rc;
  rc = check_force_args(ncoord, stride, kind, force);
  if (rc) return rc;
  DeviceGuard dg(h->device);
  cudaError_t e = launch_gather((const float4*)xyzq, ncoord, make_geom(h, recip), h->order,
                                h->d_rgrid, kind, stride, force, h->stream);
  if (e != cudaSuccess) return cuda_fail(e, "gather_force");
  return PME_OK;
}

int pme_calc_self_energy(pme_recip* h, const void* xyzq, int ncoord, double kappa) {
  if (!h) return fail(PME_EINVAL, "handle is NULL");
  if (ncoord < 0 || (ncoord > 0 && !xyzq)) return fail(PME_EINVAL, "bad xyzq/ncoord");
  if (!std::isfinite(kappa)) return fail(PME_EINVAL, "kappa must be finite");
  DeviceGuard dg(h->device);
  cudaError_t e = launch_self_energy((const float4*)xyzq, ncoord, kappa, h->d_ev, scratch(h),
                                     kSiteSelf, h->stream);
  if (e != cudaSuccess) return cuda_fail(e, "calc_self_energy");
  return PME_OK;
}

int pme_clear_energy_virial(pme_recip* h) {
  if (!h) return fail(PME_EINVAL, "handle is NULL");
  DeviceGuard dg(h->device);
  cudaError_t e = cudaMemsetAsync(h->d_ev, 0, PME_EV_COUNT * sizeof(double), h->stream);
  if (e != cudaSuccess) return cuda_fail(e, "clear_energy_virial");
  return PME_OK;
}

int pme_get_energy_virial(pme_recip* h, double* energy_recip, double* energy_self,
                          double* virial9) {
  if (!h) return fail(PME_EINVAL, "handle is NULL");
  DeviceGuard dg(h->device);
  double buf[PME_EV_COUNT];
  cudaError_t e = cudaMemcpyAsync(buf, h->d_ev, sizeof(buf), cudaMemcpyDeviceToHost, h->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  if (e != cudaSuccess) return cuda_fail(e, "get_energy_virial");
  if (energy_recip) *energy_recip = buf[PME_EV_RECIP];
  if (energy_self) *energy_self = buf[PME_EV_SELF];
  if (virial9) for (int i = 0; i < 9; i++) virial9[i] = buf[PME_EV_VIRIAL + i];
  return PME_OK;
}

int pme_copy_energy_virial_async(pme_recip* h, double* dst) {
  if (!h || !dst) return fail(PME_EINVAL, "NULL argument");
  DeviceGuard dg(h->device);
  cudaError_t e = cudaMemcpyAsync(dst, h->d_ev, PME_EV_COUNT * sizeof(double), cudaMemcpyDefault,
                                  h->stream);
  if (e != cudaSuccess) return cuda_fail(e, "copy_energy_virial_async");
  return PME_OK;
}

int pme_energy_virial_device_ptr(pme_recip* h, double** dev_ptr) {
  if (!h || !dev_ptr) return fail(PME_EINVAL, "NULL argument");
  *dev_ptr = h->d_ev;
  return PME_OK;
}

int pme_eval_ortho(pme_recip* h, double inv_boxx, double inv_boxy, double inv_boxz,
                   const void* xyzq, int ncoord, double kappa, int calc_energy, int calc_virial,
                   int kind, void* force, int stride) {
  if (!h) return fail(PME_EINVAL, "handle is NULL");
  if (ncoord < 0 || (ncoord > 0 && !xyzq)) return fail(PME_EINVAL, "bad xyzq/ncoord");
  double recip[9] = {inv_boxx, 0, 0, 0, inv_boxy, 0, 0, 0, inv_boxz};
  int rc = check_recip(recip);
  if (rc) return rc;
  if (!(kappa > 0.0) || !std::isfinite(kappa)) return fail(PME_EINVAL, "kappa must be positive");
  rc = check_force_args(ncoord, stride, kind, force);
  if (rc) return rc;
  DeviceGuard dg(h->device);
  Geom g = make_geom(h, recip);
  rc = enqueue_spread(h, xyzq, ncoord, g);
  if (rc) return rc;
  rc = enqueue_r2c(h, g);
  if (rc) return rc;
  SolveParams sp = solve_params(h, recip, kappa, (calc_energy || calc_virial) ? 1 : 0);
  cudaError_t e =
      launch_c2c(h->d_cgrid, g, 2, 2, h->pz, h->d_tw, h->tile_z, &sp, scratch(h), kSiteSolve, h->stream);
  if (e != cudaSuccess) return cuda_fail(e, "eval: z pass + solve");
  rc = enqueue_c2r_tail(h, g);
  if (rc) return rc;
  e = launch_gather((const float4*)xyzq, ncoord, g, h->order, h->d_rgrid, kind, stride, force,
                    h->stream);
  if (e != cudaSuccess) return cuda_fail(e, "eval: gather");
  if (calc_energy) {
    e = launch_self_energy((const float4*)xyzq, ncoord, kappa, h->d_ev, scratch(h), kSiteSelf,
                           h->stream);
    if (e != cudaSuccess) return cuda_fail(e, "eval: self energy");
  }
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
  if (!h) return fail(PME_EINVAL, "handle is NULL");
  const size_t G = (size_t)h->nx * h->ny * h->nz;
  return copy_back(h, host_out, h->d_accum, G * sizeof(long long), "copy_charge_grid_fixed");
}

int pme_copy_charge_grid(pme_recip* h, float* host_out) {
  if (!h || !host_out) return fail(PME_EINVAL, "NULL argument");
  const size_t G = (size_t)h->nx * h->ny * h->nz;
  std::vector<long long> tmp(G);
  int rc = copy_back(h, tmp.data(), h->d_accum, G * sizeof(long long), "copy_charge_grid");
  if (rc) return rc;
  for (size_t i = 0; i < G; i++) host_out[i] = (float)((double)tmp[i] * kInvFixedScale);
  return PME_OK;
}

int pme_copy_fft_grid(pme_recip* h, float* host_out) {
  if (!h) return fail(PME_EINVAL, "handle is NULL");
  const size_t H = (size_t)(h->nx / 2 + 1) * h->ny * h->nz;
  return copy_back(h, host_out, h->d_cgrid, H * sizeof(float2), "copy_fft_grid");
}

int pme_copy_solved_grid(pme_recip* h, float* host_out) {
  if (!h) return fail(PME_EINVAL, "handle is NULL");
  const size_t G = (size_t)h->nx * h->ny * h->nz;
  return copy_back(h, host_out, h->d_rgrid, G * sizeof(float), "copy_solved_grid");
}

int pme_load_charge_grid(pme_recip* h, const float* host_in) {
  if (!h || !host_in) return fail(PME_EINVAL, "NULL argument");
  const size_t G = (size_t)h->nx * h->ny * h->nz;
  std::vector<long long> tmp(G);
  for (size_t i = 0; i < G; i++) {
    const double v = (double)host_in[i] * 1099511627776.0;
    if (!(std::fabs(v) < 9.0e18)) return fail(PME_EINVAL, "grid value out of fixed-point range");
    tmp[i] = std::llrint(v);
  }
  DeviceGuard dg(h->device);
  cudaError_t e = cudaStreamSynchronize(h->stream);
  if (e == cudaSuccess) e = cudaMemcpy(h->d_accum, tmp.data(), G * sizeof(long long), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) return cuda_fail(e, "load_charge_grid");
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

int pme_version(void) { return 100; }

}  // extern "C"

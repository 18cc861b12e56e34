// pme_state.h -- host-side state of one PME system and the helpers that build it: grid factorisation,
// B-spline moduli, launch-tile sizes, argument checks and SystemState, the per-system device
// buffers carved from one allocation.  Shared by the operator API, the batch API and the server.
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/pme_recip.h"
#include "pme_internal.h"

namespace pme {

inline int fail(int status, const std::string& msg) {
  set_last_error(msg.c_str());
  return status;
}

inline int cuda_fail(cudaError_t e, const char* where) {
  cudaGetLastError();
  return fail(PME_ECUDA, std::string(where) + ": " + cudaGetErrorString(e));
}

// Restores the caller's current device on scope exit.
struct DeviceGuard {
  int prev = -1;
  bool changed = false;
  explicit DeviceGuard(int dev) {
    if (cudaGetDevice(&prev) == cudaSuccess && prev != dev) changed = (cudaSetDevice(dev) == cudaSuccess);
  }
  ~DeviceGuard() {
    if (changed) cudaSetDevice(prev);
  }
};

inline bool factorize(int n, FftPlan1D& p) {
  p.n = n;
  p.code = fft_code(n);
  p.nstages = 0;
  p.n_div = make_fastdiv(n);
  int m = n;
  auto push = [&](int r) {
    if (p.nstages >= kMaxStages) return false;
    p.radix[p.nstages++] = r;
    m /= r;
    return true;
  };
  while (m % 8 == 0) if (!push(8)) return false;
  while (m % 4 == 0) if (!push(4)) return false;
  while (m % 2 == 0) if (!push(2)) return false;
  while (m % 3 == 0) if (!push(3)) return false;
  while (m % 5 == 0) if (!push(5)) return false;
  if (m != 1) return false;
  int ns = 1;
  for (int s = 0; s < p.nstages; s++) {
    p.ns_div[s] = make_fastdiv(ns);
    ns *= p.radix[s];
  }
  return true;
}

// Cardinal B-spline weights at u (FP64) by the recursion of CudaPMERecip.cu:2507-2537.
inline void bspline_host(int p, double u, double* th) {
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
inline void bspline_moduli(int p, int n, double* out) {
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
  for (int k = 0; k < n; k++) out[k] = 1.0 / mod[k];
}

constexpr size_t kTileSmemBudget = 100 * 1024;   // keeps >= 2 CTAs per SM for the FFT passes

inline int pick_rows_tile(int L) {
  int tx = 16;
  while (tx > 1 && tile_smem_bytes(L, tx) > kTileSmemBudget) tx--;
  return tx;
}

inline int pick_cols_tile(int hx, int L) {
  int best = 16, best_waste = 1 << 30;
  for (int tx = 17; tx >= 8; tx--) {
    const int waste = ((hx + tx - 1) / tx) * tx - hx;
    if (waste < best_waste) { best_waste = waste; best = tx; }
  }
  if (hx < 8) best = hx;
  while (best > 1 && tile_smem_bytes(L, best) > kTileSmemBudget) best--;
  return best;
}

inline int valid_order(int order) { return order == 4 || order == 6 || order == 8; }

inline int check_grid(int nx, int ny, int nz, int order) {
  if (!valid_order(order)) return fail(PME_EINVAL, "order must be 4, 6 or 8");
  const int n3[3] = {nx, ny, nz};
  for (int d = 0; d < 3; d++)
    if (n3[d] < order || n3[d] > kMaxFftLen) return fail(PME_EINVAL, "grid lengths must be in [order, 512]");
  FftPlan1D p;
  for (int d = 0; d < 3; d++)
    if (!factorize(n3[d], p)) return fail(PME_EUNSUPPORTED, "grid lengths must factor into 2, 3 and 5");
  return PME_OK;
}

inline bool recip_is_ortho(const double* recip) {
  return recip[1] == 0.0 && recip[2] == 0.0 && recip[3] == 0.0 && recip[5] == 0.0 && recip[6] == 0.0 &&
         recip[7] == 0.0;
}

inline double det3(const double* m) {
  return m[0] * (m[4] * m[8] - m[5] * m[7]) - m[1] * (m[3] * m[8] - m[5] * m[6]) +
         m[2] * (m[3] * m[7] - m[4] * m[6]);
}

// Orthorhombic recip (CudaPMERecip.cu:2042-2045 accepts only these): a finite, positive diagonal.
// Triclinic recip R[j][d] = recip[3 j + d] (the inverse of the matrix whose rows are the box
// vectors): finite entries and a finite, non-zero determinant.
inline int check_recip(const double* recip) {
  if (!recip) return fail(PME_EINVAL, "recip is NULL");
  for (int i = 0; i < 9; i++)
    if (!std::isfinite(recip[i])) return fail(PME_EINVAL, "recip entries must be finite");
  if (recip_is_ortho(recip)) {
    for (int i : {0, 4, 8})
      if (!(recip[i] > 0.0)) return fail(PME_EINVAL, "recip diagonal must be positive");
    return PME_OK;
  }
  const double det = det3(recip);
  if (!(det != 0.0) || !std::isfinite(det))
    return fail(PME_EINVAL, "recip matrix is singular (box vectors must span a volume)");
  return PME_OK;
}

inline int check_force_args(int ncoord, int stride, int kind, const void* force) {
  if (kind != PME_FORCE_F32_SOA && kind != PME_FORCE_F32X3 && kind != PME_FORCE_I64_SOA_ACCUM)
    return fail(PME_EINVAL, "unknown force kind");
  if (ncoord > 0 && !force) return fail(PME_EINVAL, "force is NULL");
  if (kind != PME_FORCE_F32X3 && ncoord > 0 && stride < ncoord)
    return fail(PME_EINVAL, "stride must be >= ncoord for strided force layouts");
  return PME_OK;
}

inline size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

// Per-system device state, carved from a caller-provided device block.
struct SystemState {
  int nx = 0, ny = 0, nz = 0, order = 0;
  FftPlan1D px{}, py{}, pz{};
  int tx_rows = 0, tx_y = 0, tx_z = 0, plane = 0;
  int bry = 4, brz = 4, nby = 1, nbz = 1;
  int bin_cap = 0, atom_cap = 0;
  int* bins = nullptr;       // counts, bin records, bookkeeping, overflow records, atom order
  unsigned long long* accum = nullptr;
  float2* cgrid = nullptr;
  float* rgrid = nullptr;
  float2* tw = nullptr;
  double* bmod = nullptr;
  double* ktab = nullptr;
  long long* acc = nullptr;
  double* ev = nullptr;

  size_t G() const { return (size_t)nx * ny * nz; }
  size_t H() const { return (size_t)(nx / 2 + 1) * ny * nz; }

  // bytes of device memory one system needs
  static size_t bytes(int nx, int ny, int nz) {
    const size_t G = (size_t)nx * ny * nz, H = (size_t)(nx / 2 + 1) * ny * nz, n = nx + ny + nz;
    return align256(G * 8) + align256(H * 8) + align256(G * 4) + align256(n * 8) + align256(n * 8) +
           align256(4 * n * 8) + align256(kAccCount * 8) + align256(kEvCount * 8);
  }

  void setup(int nx_, int ny_, int nz_, int order_) {
    nx = nx_; ny = ny_; nz = nz_; order = order_;
    factorize(nx, px);
    factorize(ny, py);
    factorize(nz, pz);
    px.tw_off = 0;
    py.tw_off = nx;
    pz.tw_off = nx + ny;
    tx_rows = pick_rows_tile(nx);
    tx_y = pick_rows_tile(ny);
    tx_z = pick_cols_tile(ny, nz);
    // whole-plane tiles need one thread per line of each orientation and the plane in smem
    plane = (plane_smem_bytes(ny, nz) <= kTileSmemBudget && ny <= kThreads && nz <= kThreads) ? 1 : 0;
    // row blocks of the fused spread + x pass: the largest square block that fits
    for (int b = kSpreadMaxBlock; b >= 1; b--) {
      bry = brz = b;
      size_t need = 0;   // the order can change later (pme_set_order): size for every order
      for (int o = 4; o <= kMaxOrder; o += 2) need = std::max(need, spread_x_smem_bytes(nx, b * b, o));
      if (need <= kTileSmemBudget) break;
    }
    nby = (ny + bry - 1) / bry;
    nbz = (nz + brz - 1) / brz;
  }

  int nbins() const { return nby * nbz; }

  // bin storage for up to natom atoms: capacity 1.5x the mean occupancy + 32 per bin
  static int cap_for(int natom, int nbins) { return std::max(32, (int)(1.5 * natom / nbins) + 32); }
  // counts (padded to 16 bytes), bin records, bookkeeping (kMetaInts), overflow records, the
  // bin-sorted atom order; records are sized for order 8
  size_t count_ints() const { return (2 * (size_t)nbins() + 3) & ~(size_t)3; }
  size_t bin_ints(int natom) const {
    const size_t n = (size_t)std::max(natom, 1);
    return count_ints() + (size_t)nbins() * cap_for(natom, nbins()) * rec_floats(kMaxOrder) + kMetaInts +
           n * rec_floats(kMaxOrder) + n;
  }

  void carve(char* base) {
    const size_t n = nx + ny + nz;
    char* p = base;
    accum = (unsigned long long*)p; p += align256(G() * 8);
    cgrid = (float2*)p; p += align256(H() * 8);
    rgrid = (float*)p; p += align256(G() * 4);
    tw = (float2*)p; p += align256(n * 8);
    bmod = (double*)p; p += align256(n * 8);
    ktab = (double*)p; p += align256(4 * n * 8);
    acc = (long long*)p; p += align256(kAccCount * 8);
    ev = (double*)p;
  }

  // twiddles exp(-2 pi i k/n) (FP64 -> FP32) and moduli (FP64) for the current order
  void host_tables(std::vector<float2>& twh, std::vector<double>& bm) const {
    const int n3[3] = {nx, ny, nz};
    twh.clear();
    bm.assign((size_t)(nx + ny + nz), 0.0);
    size_t off = 0;
    for (int d = 0; d < 3; d++) {
      for (int k = 0; k < n3[d]; k++) {
        const double a = -2.0 * kPi * (double)k / (double)n3[d];
        twh.push_back(make_float2((float)std::cos(a), (float)std::sin(a)));
      }
      bspline_moduli(order, n3[d], bm.data() + off);
      off += n3[d];
    }
  }

  cudaError_t upload_tables() const {
    std::vector<float2> twh;
    std::vector<double> bm;
    host_tables(twh, bm);
    cudaError_t e = cudaMemcpy(tw, twh.data(), twh.size() * sizeof(float2), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(bmod, bm.data(), bm.size() * sizeof(double), cudaMemcpyHostToDevice);
    return e;
  }

  SysDesc desc(const double* r3, double kappa, const void* xyzq, int natom, void* force, int kind,
               int stride, int calc_ev, int calc_self) const {
    SysDesc d;
    std::memset(&d, 0, sizeof(d));
    Geom& g = d.g;
    g.nx = nx; g.ny = ny; g.nz = nz;
    g.hx = nx / 2 + 1;
    const double r[3] = {r3 ? r3[0] : 1.0, r3 ? r3[1] : 1.0, r3 ? r3[2] : 1.0};
    g.rx = (float)r[0]; g.ry = (float)r[1]; g.rz = (float)r[2];
    const int n3[3] = {nx, ny, nz};
    float hi[3], lo[3];
    for (int i = 0; i < 3; i++) {
      const double s = r[i] * n3[i];
      hi[i] = (float)s;
      lo[i] = (float)(s - (double)hi[i]);
    }
    g.sx_hi = hi[0]; g.sy_hi = hi[1]; g.sz_hi = hi[2];
    g.sx_lo = lo[0]; g.sy_lo = lo[1]; g.sz_lo = lo[2];
    d.px = px; d.py = py; d.pz = pz;
    d.order = order;
    d.natom = natom;
    d.rxd = r[0]; d.ryd = r[1]; d.rzd = r[2];
    d.fac = kappa > 0.0 ? kPi * kPi / (kappa * kappa) : 0.0;
    d.piv_inv = r[0] * r[1] * r[2] / kPi;
    d.fac_f = (float)d.fac;
    d.piv_inv_f = (float)d.piv_inv;
    d.calc_ev = calc_ev;
    d.calc_self = calc_self;
    d.self_coef = -kappa * kCcelec / std::sqrt(kPi);
    d.force_kind = kind;
    d.stride = stride;
    d.xyzq = (const float4*)xyzq;
    d.force = force;
    d.accum = accum;
    d.cgrid = cgrid;
    d.rgrid = rgrid;
    d.bmod = bmod;
    d.ktab = ktab;
    d.tw = tw;
    d.acc = acc;
    d.ev = ev;
    d.tx_rows = tx_rows; d.tx_y = tx_y; d.tx_z = tx_z;
    d.plane = plane;
    d.bry = bry; d.brz = brz; d.nby = nby; d.nbz = nbz;
    d.bin_cap = bin_cap;
    if (bins) {
      const size_t nb = nbins();
      d.bin_count = bins;
      d.bin_recs = (float*)(bins + count_ints());
      d.bin_meta = (int*)(d.bin_recs + nb * (size_t)bin_cap * rec_floats(kMaxOrder));
      d.ovf_recs = (float*)(d.bin_meta + kMetaInts);
      d.perm = (int*)(d.ovf_recs + (size_t)std::max(atom_cap, 1) * rec_floats(kMaxOrder));
    }
    return d;
  }

  // Descriptor from a full reciprocal matrix R[j][d] = recip9[3 j + d] (or null for setup-only
  // calls).  A diagonal matrix gives exactly desc(diagonal); off-diagonals switch the tiles to
  // their triclinic forms: float-float S = n_d R[j][d] for the fractional coordinates and the force
  // transform, R and the metric G = R^T R for the influence tables, V = 1 / |det R|.
  SysDesc desc9(const double* recip9, double kappa, const void* xyzq, int natom, void* force, int kind,
                int stride, int calc_ev, int calc_self) const {
    if (!recip9) return desc(nullptr, kappa, xyzq, natom, force, kind, stride, calc_ev, calc_self);
    const double r3[3] = {recip9[0], recip9[4], recip9[8]};
    SysDesc d = desc(r3, kappa, xyzq, natom, force, kind, stride, calc_ev, calc_self);
    if (recip_is_ortho(recip9)) return d;
    Geom& g = d.g;
    g.tric = 1;
    const int n3[3] = {nx, ny, nz};
    for (int j = 0; j < 3; j++)
      for (int c = 0; c < 3; c++) {
        const double sv = recip9[3 * j + c] * n3[c];
        g.shi[3 * j + c] = (float)sv;
        g.slo[3 * j + c] = (float)(sv - (double)g.shi[3 * j + c]);
      }
    double G[9];
    for (int a = 0; a < 3; a++)
      for (int b = 0; b < 3; b++) {
        double sum = 0.0;
        for (int j = 0; j < 3; j++) sum += recip9[3 * j + a] * recip9[3 * j + b];
        G[3 * a + b] = sum;
      }
    for (int i = 0; i < 9; i++) d.rm[i] = recip9[i];
    for (int a = 0; a < 3; a++) d.gdiag[a] = G[4 * a];
    d.cross_f[0] = (float)(-2.0 * d.fac * G[1]);
    d.cross_f[1] = (float)(-2.0 * d.fac * G[2]);
    d.cross_f[2] = (float)(-2.0 * d.fac * G[5]);
    d.piv_inv = std::fabs(det3(recip9)) / kPi;
    d.piv_inv_f = (float)d.piv_inv;
    return d;
  }
};


}  // namespace pme

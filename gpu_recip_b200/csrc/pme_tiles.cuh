// pme_tiles.cuh -- per-tile device functions of the PME reciprocal path, shared by the staged
// kernels (one tile per CTA) and the persistent fused kernel (tiles of many systems, grid
// barriers between phases).  Every function assumes blockDim.x == kThreads and must be called
// by all threads of the CTA (they synchronise internally).
//
// Energy, virial and sum(q^2) are reduced in FP64 inside the CTA, then added to per-system int64
// fixed-point accumulators (scale 2^32 for energy/virial, 2^40 for sum(q^2)).  Integer addition is
// associative, so the totals are bit-identical for any tiling, launch shape or batch mix; a
// finalize step converts them into the FP64 energy/virial record.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "pme_common.cuh"
#include "pme_fft.cuh"

namespace pme {

constexpr int kThreads = 256;
constexpr double kEvScale = 4294967296.0;          // 2^32
constexpr double kQ2Scale = 1099511627776.0;       // 2^40

enum ForceKind { kForceF32Soa = 0, kForceF32x3 = 1, kForceI64SoaAccum = 2 };

// Accumulator slots (int64, per system): energy, 6 virial components, sum q^2.
enum AccSlot { kAccE = 0, kAccV0 = 1, kAccQ2 = 7, kAccCount = 8 };

// Energy/virial record layout in device memory (doubles), as include/pme_recip.h.
enum EvSlot { kEvRecip = 0, kEvSelf = 1, kEvVirial = 2, kEvCount = 11 };

// Everything a tile needs to know about one system.
struct SysDesc {
  Geom g;
  FftPlan1D px, py, pz;
  int order;
  int natom;
  double fac;                // pi^2 / kappa^2
  double piv_inv;            // 1 / (pi V)
  double rxd, ryd, rzd;      // reciprocal box diagonal, FP64
  int calc_ev;               // energy + virial in the solve
  int calc_self;             // self energy in the spread phase
  double self_coef;          // -kappa ccelec / sqrt(pi)
  int force_kind;
  int stride;
  const float4* xyzq;
  void* force;
  unsigned long long* accum; // int64 charge grid [z][y][x]
  float2* cgrid;             // half-complex grid [z][y][kx]
  float* rgrid;              // solved real grid [z][y][x]
  const double* bmod;        // B-spline moduli 1/|b|^2, x | y | z (FP64)
  double* ktab;              // influence tables: mhat x|y|z, then A = bmod exp(-fac mhat^2) x|y|z
  const float2* tw;          // twiddles x | y | z (plan.tw_off)
  long long* acc;            // kAccCount fixed-point accumulators
  double* ev;                // kEvCount record
  int tx_rows, tx_y, tx_z;   // lines per tile of the x, y, z passes
};

constexpr int kSpreadAtomsPerWarp = 8;
constexpr int kSpreadAtoms = kSpreadAtomsPerWarp * (kThreads / 32);   // atoms per spread tile
__host__ __device__ inline int tiles_spread(const SysDesc& d) { return (d.natom + kSpreadAtoms - 1) / kSpreadAtoms; }
__host__ __device__ inline int tiles_xpass(const SysDesc& d) { return (d.g.ny * d.g.nz + d.tx_rows - 1) / d.tx_rows; }
__host__ __device__ inline int tiles_ypass(const SysDesc& d) { return ((d.g.hx + d.tx_y - 1) / d.tx_y) * d.g.nz; }
__host__ __device__ inline int tiles_zpass(const SysDesc& d) { return ((d.g.hx + d.tx_z - 1) / d.tx_z) * d.g.ny; }
__host__ __device__ inline int tiles_gather(const SysDesc& d) { return (d.natom + 31) / 32; }
__host__ inline size_t tile_smem_bytes(int L, int tx) {
  return sizeof(float2) * ((size_t)L + 2 * (size_t)L * (tx + 1));
}

// ---------------------------------------------------------------------------------------------
// Block reductions
// ---------------------------------------------------------------------------------------------
template <int K>
__device__ __forceinline__ void warp_sum(double (&v)[K]) {
#pragma unroll
  for (int off = 16; off >= 1; off >>= 1)
#pragma unroll
    for (int c = 0; c < K; c++) v[c] += __shfl_down_sync(0xffffffffu, v[c], off);
}

// Deterministic block sum; the result is valid in thread 0.  `scratch` holds 32*K doubles.
template <int K>
__device__ __forceinline__ void block_sum(double (&v)[K], double* scratch) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  warp_sum<K>(v);
  __syncthreads();
  if (lane == 0)
#pragma unroll
    for (int c = 0; c < K; c++) scratch[warp * K + c] = v[c];
  __syncthreads();
  if (warp == 0) {
#pragma unroll
    for (int c = 0; c < K; c++) v[c] = lane < nw ? scratch[lane * K + c] : 0.0;
    warp_sum<K>(v);
  }
}

__device__ __forceinline__ void acc_add(long long* acc, int slot, double v, double scale) {
  atomicAdd((unsigned long long*)&acc[slot], (unsigned long long)__double2ll_rn(v * scale));
}

// ---------------------------------------------------------------------------------------------
// Spread tile: kSpreadAtoms atoms; warp w spreads atoms [8w, 8w+8) of the tile.  Lanes 0..7 each
// compute one atom's stencil origin and weights (q folded into x), then the warp covers the
// 8 atoms' P^3 stencils with its 32 lanes, adding exact fixed-point contributions with 64-bit
// integer reductions.  Also accumulates sum(q^2) when the system asks for the self energy.
// smem: kSpreadAtoms x (3 ints + 3P floats), plus 32 doubles.
// ---------------------------------------------------------------------------------------------
template <int P>
struct SplineAtom {
  int ix, iy, iz;
  float tx[P], ty[P], tz[P];
};

template <int P>
__device__ __forceinline__ void spread_tile(const SysDesc& d, int tile, void* smem) {
  constexpr int APW = kSpreadAtomsPerWarp;
  SplineAtom<P>* sh = (SplineAtom<P>*)smem;
  double* red = (double*)((char*)smem + ((sizeof(SplineAtom<P>) * kSpreadAtoms + 7) / 8) * 8);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const Geom& g = d.g;
  const int base = tile * kSpreadAtoms + warp * APW;
  const int cnt = max(0, min(APW, d.natom - base));
  double q2[1] = {0.0};
  if (lane < cnt) {
    const float4 a = __ldg(&d.xyzq[base + lane]);
    SplineAtom<P>& s = sh[warp * APW + lane];
    float ux, uy, uz, th[P];
    frac_coord(a.x, g.sx_hi, g.sx_lo, g.nx, s.ix, ux);
    frac_coord(a.y, g.sy_hi, g.sy_lo, g.ny, s.iy, uy);
    frac_coord(a.z, g.sz_hi, g.sz_lo, g.nz, s.iz, uz);
    bspline<P>(ux, th, nullptr);
#pragma unroll
    for (int i = 0; i < P; i++) s.tx[i] = __fmul_rn(a.w, th[i]);
    bspline<P>(uy, th, nullptr);
#pragma unroll
    for (int i = 0; i < P; i++) s.ty[i] = th[i];
    bspline<P>(uz, th, nullptr);
#pragma unroll
    for (int i = 0; i < P; i++) s.tz[i] = th[i];
    q2[0] = (double)a.w * (double)a.w;
  }
  __syncwarp();
  constexpr int P3 = P * P * P;
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  unsigned long long* __restrict__ accum = d.accum;
  for (int q = lane; q < cnt * P3; q += 32) {
    const int i = q / P3, r = q - i * P3;
    const int a = r % P, b = (r / P) % P, c = r / (P * P);
    const SplineAtom<P>& s = sh[warp * APW + i];
    const int x = wrap_add(s.ix, a, nx);
    const int y = wrap_add(s.iy, b, ny);
    const int z = wrap_add(s.iz, c, nz);
    const long long v = fixed_contrib(s.tx[a], s.ty[b], s.tz[c]);
    atomicAdd(&accum[x + (size_t)nx * (y + (size_t)ny * z)], (unsigned long long)v);
  }
  if (d.calc_self) {
    block_sum<1>(q2, red);
    if (threadIdx.x == 0 && d.natom > 0) acc_add(d.acc, kAccQ2, q2[0], kQ2Scale);
  }
  __syncthreads();
}

template <int P>
__host__ inline size_t spread_smem_bytes() {
  return ((sizeof(SplineAtom<P>) * kSpreadAtoms + 7) / 8) * 8 + 32 * sizeof(double);
}

// ---------------------------------------------------------------------------------------------
// x pass, forward: tx_rows consecutive grid rows (row = y + ny z); int64 -> FP32 on load (and the
// accumulation grid re-zeroed behind the read when zero_accum); complex FFT of length nx with
// zero imaginary part; the nx/2+1 non-redundant outputs go to the half-complex grid.
// ---------------------------------------------------------------------------------------------
__device__ __forceinline__ void x_fwd_tile(const SysDesc& d, int tile, float2* smem, bool zero_accum) {
  const Geom& g = d.g;
  const FftPlan1D& plan = d.px;
  const int L = g.nx, tx = d.tx_rows, ld = tx + 1;
  float2* tw = smem;
  float2* b0 = tw + L;
  float2* b1 = b0 + L * ld;
  const int tid = threadIdx.x;
  const int nrows = g.ny * g.nz, row0 = tile * tx;
  for (int i = tid; i < L; i += kThreads) tw[i] = __ldg(&d.tw[plan.tw_off + i]);
  const unsigned long long* __restrict__ src = d.accum + (size_t)row0 * L;
  const int nvalid = min(tx, nrows - row0) * L;   // rows of this tile inside the grid
#pragma unroll 4
  for (int idx = tid; idx < L * tx; idx += kThreads) {
    const int t = fdiv(idx, plan.n_div), e = idx - t * L;
    const float v = idx < nvalid ? fixed_to_float((long long)__ldcg(&src[idx])) : 0.0f;
    b0[e * ld + t] = make_float2(v, 0.0f);
  }
  if (zero_accum) {
    unsigned long long* dst = d.accum + (size_t)row0 * L;
    for (int idx = tid; idx < nvalid; idx += kThreads) __stcg(&dst[idx], 0ull);
  }
  __syncthreads();
  TileLane ln(tid, kThreads, tx);
  float2* res = fft_tile(b0, b1, plan, ld, ln, tw, false);
  const int hx = g.hx;
  const FastDiv hxd = make_fastdiv(hx);
  for (int idx = tid; idx < hx * tx; idx += kThreads) {
    const int t = fdiv(idx, hxd), k = idx - t * hx, row = row0 + t;
    if (row < nrows) __stcg(&d.cgrid[(size_t)row * hx + k], res[k * ld + t]);
  }
  __syncthreads();
}

// x pass, inverse: Hermitian rebuild X[n-k] = conj X[k] of each row, inverse FFT, real part (the
// imaginary parts of X[0] and of the Nyquist term drop out, as in a library C2R).
__device__ __forceinline__ void x_inv_tile(const SysDesc& d, int tile, float2* smem) {
  const Geom& g = d.g;
  const FftPlan1D& plan = d.px;
  const int L = g.nx, tx = d.tx_rows, ld = tx + 1, hx = g.hx;
  float2* tw = smem;
  float2* b0 = tw + L;
  float2* b1 = b0 + L * ld;
  const int tid = threadIdx.x;
  const int nrows = g.ny * g.nz, row0 = tile * tx;
  const FastDiv hxd = make_fastdiv(hx);
  for (int i = tid; i < L; i += kThreads) tw[i] = __ldg(&d.tw[plan.tw_off + i]);
  for (int idx = tid; idx < hx * tx; idx += kThreads) {
    const int t = fdiv(idx, hxd), k = idx - t * hx, row = row0 + t;
    float2 v = make_float2(0.0f, 0.0f);
    if (row < nrows) v = __ldcg(&d.cgrid[(size_t)row * hx + k]);
    b0[k * ld + t] = v;
    if (k >= 1 && L - k >= hx) b0[(L - k) * ld + t] = make_float2(v.x, -v.y);
  }
  __syncthreads();
  TileLane ln(tid, kThreads, tx);
  float2* res = fft_tile(b0, b1, plan, ld, ln, tw, true);
  for (int idx = tid; idx < L * tx; idx += kThreads) {
    const int t = fdiv(idx, plan.n_div), e = idx - t * L, row = row0 + t;
    if (row < nrows) __stcg(&d.rgrid[(size_t)row * L + e], res[e * ld + t].x);
  }
  __syncthreads();
}

// ---------------------------------------------------------------------------------------------
// Influence function (CudaPMERecip.cu:671-691): m_d = k_d or k_d - n_d, mhat = r m,
// eterm = exp(-fac |mhat|^2) piv_inv b_x b_y b_z / |mhat|^2.  exp(-fac |mhat|^2) b_x b_y b_z factors
// per axis, so ktab_tile precomputes mhat_d[k] and A_d[k] = b_d[k] exp(-fac mhat_d[k]^2) in FP64
// once per evaluation (nx+ny+nz values) and the solve evaluates eterm in FP64 from them.
// ---------------------------------------------------------------------------------------------
__device__ __forceinline__ void ktab_tile(const SysDesc& d) {
  const Geom& g = d.g;
  const int ntot = g.nx + g.ny + g.nz;
  for (int i = threadIdx.x; i < ntot; i += kThreads) {
    int n, k;
    double r;
    if (i < g.nx) { n = g.nx; k = i; r = d.rxd; }
    else if (i < g.nx + g.ny) { n = g.ny; k = i - g.nx; r = d.ryd; }
    else { n = g.nz; k = i - g.nx - g.ny; r = d.rzd; }
    const int nf = (n >> 1) + (n & 1);
    const int m = k < nf ? k : k - n;
    const double mh = r * (double)m;
    d.ktab[i] = mh;
    d.ktab[ntot + i] = d.bmod[i] * exp(-d.fac * mh * mh);
  }
}

struct KTerm {
  double eterm, m1, m2, m3, msq;
};

__device__ __forceinline__ KTerm kterm(int kx, int ky, int kz, const SysDesc& d) {
  const Geom& g = d.g;
  const double* mh = d.ktab;
  const double* A = d.ktab + g.nx + g.ny + g.nz;
  KTerm o;
  o.m1 = __ldcg(&mh[kx]);
  o.m2 = __ldcg(&mh[g.nx + ky]);
  o.m3 = __ldcg(&mh[g.nx + g.ny + kz]);
  o.msq = o.m1 * o.m1 + o.m2 * o.m2 + o.m3 * o.m3;
  o.eterm = d.piv_inv * __ldcg(&A[kx]) * __ldcg(&A[g.nx + ky]) * __ldcg(&A[g.nx + g.ny + kz]) / o.msq;
  return o;
}

// Energy and virial terms of one k (CudaPMERecip.cu:694-742), FP64:
// [t, t (v m1 m1 - 1), t v m1 m2, t v m1 m3, t (v m2 m2 - 1), t v m2 m3, t (v m3 m3 - 1)],
// t = eterm |Q|^2, v = 2 (fac + 1/|m|^2).
__device__ __forceinline__ void ev_accum(double* acc, const KTerm& k, double q2, double fac) {
  const double t1 = k.eterm * q2;
  const double vt = 2.0 * (fac + 1.0 / k.msq);
  acc[0] += t1;
  acc[1] += t1 * (vt * k.m1 * k.m1 - 1.0);
  acc[2] += t1 * vt * k.m1 * k.m2;
  acc[3] += t1 * vt * k.m1 * k.m3;
  acc[4] += t1 * (vt * k.m2 * k.m2 - 1.0);
  acc[5] += t1 * vt * k.m2 * k.m3;
  acc[6] += t1 * (vt * k.m3 * k.m3 - 1.0);
}

// Solve on a z-line tile held in smem (lines = kx0.. at fixed ky, elements = kz).  Every stored k
// contributes its own term and, for kx >= 1, the term of its mirror -k (the reference's x-mirror
// doubling, CudaPMERecip.cu:708-742).  Q(0) is zeroed.
__device__ __forceinline__ void solve_tile(float2* buf, int ld, int tx, const FastDiv& txd, int kx0,
                                           int ky, const SysDesc& d, double* acc) {
  const Geom& g = d.g;
  const int L = g.nz;
  const double facd = d.fac;
  for (int idx = threadIdx.x; idx < L * tx; idx += kThreads) {
    const int e = fdiv(idx, txd), t = idx - e * tx, kx = kx0 + t, kz = e;
    if (kx >= g.hx) continue;
    float2 q = buf[e * ld + t];
    if (kx == 0 && ky == 0 && kz == 0) {
      buf[e * ld + t] = make_float2(0.0f, 0.0f);
      continue;
    }
    const KTerm k = kterm(kx, ky, kz, d);
    if (d.calc_ev) {
      const double q2 = (double)q.x * (double)q.x + (double)q.y * (double)q.y;
      ev_accum(acc, k, q2, facd);
      if (kx >= 1) {
        const int kxs = g.nx - kx, kys = ky == 0 ? 0 : g.ny - ky, kzs = kz == 0 ? 0 : g.nz - kz;
        const KTerm ks = kterm(kxs, kys, kzs, d);
        ev_accum(acc, ks, q2, facd);
      }
    }
    const float et = (float)k.eterm;
    q.x *= et;
    q.y *= et;
    buf[e * ld + t] = q;
  }
}

// Complex pass along y (axis 1) or z (axis 2).  A tile is tx consecutive kx at one outer index
// (z for the y pass, y for the z pass), so each element row of the tile is tx contiguous complex
// values.  mode: 0 forward, 1 inverse, 2 forward + solve + inverse (z), 3 solve only (z).
// smem: twiddles, two tile buffers, 32*7 doubles.
__device__ __forceinline__ void c2c_tile(const SysDesc& d, int axis, int mode, int tile, float2* smem) {
  const Geom& g = d.g;
  const FftPlan1D& plan = axis == 1 ? d.py : d.pz;
  const int tx = axis == 1 ? d.tx_y : d.tx_z;
  const int L = plan.n, ld = tx + 1;
  float2* tw = smem;
  float2* b0 = tw + L;
  float2* b1 = b0 + L * ld;
  double* red = (double*)(b1 + L * ld);
  const int tid = threadIdx.x;
  const int tiles_x = (g.hx + tx - 1) / tx;
  const int outer = tile / tiles_x, tile_x = tile - outer * tiles_x;
  const int kx0 = tile_x * tx;
  const FastDiv txd = make_fastdiv(tx);
  size_t estride, obase;
  if (axis == 1) {
    estride = (size_t)g.hx;
    obase = (size_t)outer * g.hx * g.ny;
  } else {
    estride = (size_t)g.hx * g.ny;
    obase = (size_t)outer * g.hx;
  }
  if (mode != 3)
    for (int i = tid; i < L; i += kThreads) tw[i] = __ldg(&d.tw[plan.tw_off + i]);
  for (int idx = tid; idx < L * tx; idx += kThreads) {
    const int e = fdiv(idx, txd), t = idx - e * tx, kx = kx0 + t;
    float2 v = make_float2(0.0f, 0.0f);
    if (kx < g.hx) v = __ldcg(&d.cgrid[obase + e * estride + kx]);
    b0[e * ld + t] = v;
  }
  __syncthreads();
  TileLane ln(tid, kThreads, tx);
  float2* res = b0;
  if (mode == 0 || mode == 2) res = fft_tile(b0, b1, plan, ld, ln, tw, false);
  if (mode == 1) res = fft_tile(b0, b1, plan, ld, ln, tw, true);
  if (mode == 2 || mode == 3) {
    double acc[7] = {0, 0, 0, 0, 0, 0, 0};
    solve_tile(res, ld, tx, txd, kx0, outer, d, acc);
    __syncthreads();
    if (d.calc_ev) {
      block_sum<7>(acc, red);
      if (tid == 0)
#pragma unroll
        for (int c = 0; c < 7; c++) acc_add(d.acc, kAccE + c, acc[c], kEvScale);
    }
    if (mode == 2) {
      float2* other = (res == b0) ? b1 : b0;
      res = fft_tile(res, other, plan, ld, ln, tw, true);
    }
  }
  for (int idx = tid; idx < L * tx; idx += kThreads) {
    const int e = fdiv(idx, txd), t = idx - e * tx, kx = kx0 + t;
    if (kx < g.hx) __stcg(&d.cgrid[obase + e * estride + kx], res[e * ld + t]);
  }
  __syncthreads();
}

// Convert the accumulators into the FP64 record and clear them (one thread).
__device__ __forceinline__ void finalize_system(const SysDesc& d, bool solve, bool self) {
  long long* acc = d.acc;
  double* ev = d.ev;
  if (solve && d.calc_ev) {
    double s[7];
    for (int c = 0; c < 7; c++) {
      s[c] = (double)acc[kAccE + c] / kEvScale;
      acc[kAccE + c] = 0;
    }
    const double h = 0.5 * kCcelec;
    ev[kEvRecip] += h * s[0];
    double* vir = ev + kEvVirial;
    vir[0] -= h * s[1]; vir[1] -= h * s[2]; vir[2] -= h * s[3];
    vir[3] -= h * s[2]; vir[4] -= h * s[4]; vir[5] -= h * s[5];
    vir[6] -= h * s[3]; vir[7] -= h * s[5]; vir[8] -= h * s[6];
  }
  if (self && d.calc_self) {
    const double q2 = (double)acc[kAccQ2] / kQ2Scale;
    acc[kAccQ2] = 0;
    ev[kEvSelf] += d.self_coef * q2;
  }
}

// ---------------------------------------------------------------------------------------------
// Gather tile: 32 atoms, 8 lanes per atom; lane l takes stencil rows (b, c) = l, l+8, ... of the
// P^2 rows and sums the P points of each row; the 8 partial sums are combined with shuffles.
// F_d = q ccelec n_d r_d sum(...) (gradient convention, CudaPMERecip.cu:1234-1242).
// ---------------------------------------------------------------------------------------------
template <int P, int KIND>
__device__ __forceinline__ void gather_tile(const SysDesc& d, int tile) {
  const Geom& g = d.g;
  const int atom = tile * 32 + (threadIdx.x >> 3), gl = threadIdx.x & 7;
  const bool valid = atom < d.natom;
  const float4 a = valid ? __ldg(&d.xyzq[atom]) : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  int ix, iy, iz;
  float ux, uy, uz;
  frac_coord(a.x, g.sx_hi, g.sx_lo, g.nx, ix, ux);
  frac_coord(a.y, g.sy_hi, g.sy_lo, g.ny, iy, uy);
  frac_coord(a.z, g.sz_hi, g.sz_lo, g.nz, iz, uz);
  float thx[P], dthx[P], thy[P], dthy[P], thz[P], dthz[P];
  bspline<P>(ux, thx, dthx);
  bspline<P>(uy, thy, dthy);
  bspline<P>(uz, thz, dthz);
  int xs[P];
#pragma unroll
  for (int i = 0; i < P; i++) xs[i] = wrap_add(ix, i, g.nx);
  float f1 = 0.0f, f2 = 0.0f, f3 = 0.0f;
  constexpr int RPL = (P * P + 7) / 8;
  const float* rg = d.rgrid;
#pragma unroll
  for (int rr = 0; rr < RPL; rr++) {
    const int r = gl + 8 * rr;
    if (valid && r < P * P) {
      const int b = r % P, c = r / P;
      float wy = 0.0f, dwy = 0.0f, wz = 0.0f, dwz = 0.0f;
#pragma unroll
      for (int q = 0; q < P; q++) {
        if (q == b) { wy = thy[q]; dwy = dthy[q]; }
        if (q == c) { wz = thz[q]; dwz = dthz[q]; }
      }
      const int y = wrap_add(iy, b, g.ny), z = wrap_add(iz, c, g.nz);
      const float* row = rg + (size_t)g.nx * (y + (size_t)g.ny * z);
      float s1 = 0.0f, s2 = 0.0f;
#pragma unroll
      for (int i = 0; i < P; i++) {
        const float v = row[xs[i]];
        s1 = fmaf(dthx[i], v, s1);
        s2 = fmaf(thx[i], v, s2);
      }
      f1 = fmaf(s1, wy * wz, f1);
      f2 = fmaf(s2, dwy * wz, f2);
      f3 = fmaf(s2, wy * dwz, f3);
    }
  }
#pragma unroll
  for (int off = 4; off >= 1; off >>= 1) {
    f1 += __shfl_xor_sync(0xffffffffu, f1, off);
    f2 += __shfl_xor_sync(0xffffffffu, f2, off);
    f3 += __shfl_xor_sync(0xffffffffu, f3, off);
  }
  if (valid && gl == 0) {
    const float qc = a.w * (float)kCcelec;
    const float fx = qc * g.sx_hi * f1;
    const float fy = qc * g.sy_hi * f2;
    const float fz = qc * g.sz_hi * f3;
    const size_t st = (size_t)d.stride;
    if (KIND == kForceF32Soa) {
      float* f = (float*)d.force;
      f[atom] = fx;
      f[atom + st] = fy;
      f[atom + 2 * st] = fz;
    } else if (KIND == kForceF32x3) {
      float* f = (float*)d.force + 3 * (size_t)atom;
      f[0] = fx; f[1] = fy; f[2] = fz;
    } else {
      unsigned long long* f = (unsigned long long*)d.force;
      atomicAdd(&f[atom], (unsigned long long)__float2ll_rn(__fmul_rn(fx, kFixedScale)));
      atomicAdd(&f[atom + st], (unsigned long long)__float2ll_rn(__fmul_rn(fy, kFixedScale)));
      atomicAdd(&f[atom + 2 * st], (unsigned long long)__float2ll_rn(__fmul_rn(fz, kFixedScale)));
    }
  }
}

template <int P>
__device__ __forceinline__ void gather_tile_any(const SysDesc& d, int tile) {
  switch (d.force_kind) {
    case kForceF32Soa: gather_tile<P, kForceF32Soa>(d, tile); break;
    case kForceF32x3: gather_tile<P, kForceF32x3>(d, tile); break;
    default: gather_tile<P, kForceI64SoaAccum>(d, tile); break;
  }
}

__device__ __forceinline__ void gather_dispatch(const SysDesc& d, int tile) {
  switch (d.order) {
    case 4: gather_tile_any<4>(d, tile); break;
    case 6: gather_tile_any<6>(d, tile); break;
    default: gather_tile_any<8>(d, tile); break;
  }
}

__device__ __forceinline__ void spread_dispatch(const SysDesc& d, int tile, void* smem) {
  switch (d.order) {
    case 4: spread_tile<4>(d, tile, smem); break;
    case 6: spread_tile<6>(d, tile, smem); break;
    default: spread_tile<8>(d, tile, smem); break;
  }
}

}  // namespace pme

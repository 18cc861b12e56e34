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
  float fac_f, piv_inv_f;    // the same, FP32
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
  int plane;                 // 1: the fused path runs y, z and the solve as whole-plane tiles
  // Atom bins of the fused path: bin (by, bz) holds the atoms whose stencil origin (iy0, iz0)
  // lies in row block [by*bry, by*bry+bry) x [bz*brz, bz*brz+brz); fixed capacity bin_cap per bin,
  // surplus atoms go to an overflow list.  Counters are double-buffered by launch parity.
  int bry, brz, nby, nbz;
  int bin_cap;
  int* bin_count;            // [2][nby*nbz]
  float* bin_recs;           // [nby*nbz][bin_cap] atom records of rec_floats(order) floats
  int* ovf_count;            // [2]
  float* ovf_recs;           // [natom capacity] records of the atoms beyond a bin's capacity
  unsigned long long* steps; // profiling: %globaltimer at the steps of CTA 0's tiles (or null)
};

// Profiling stamp of one step of a tile (CTA 0, thread 0 only; no-op when steps is null).
__device__ __forceinline__ void step_mark(const SysDesc& d, int slot) {
  if (d.steps != nullptr && blockIdx.x == 0 && threadIdx.x == 0) {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    d.steps[slot] = t;
  }
}

constexpr int kSpreadAtomsPerWarp = 8;
constexpr int kSpreadAtoms = kSpreadAtomsPerWarp * (kThreads / 32);   // atoms per spread tile
__host__ __device__ inline int tiles_spread(const SysDesc& d) { return (d.natom + kSpreadAtoms - 1) / kSpreadAtoms; }
__host__ __device__ inline int tiles_xpass(const SysDesc& d) { return (d.g.ny * d.g.nz + d.tx_rows - 1) / d.tx_rows; }
__host__ __device__ inline int tiles_ypass(const SysDesc& d) { return (d.g.hx * d.g.nz + d.tx_y - 1) / d.tx_y; }
__host__ __device__ inline int tiles_zpass(const SysDesc& d) { return ((d.g.ny + d.tx_z - 1) / d.tx_z) * d.g.hx; }
__host__ __device__ inline int tiles_plane(const SysDesc& d) { return d.g.hx; }
__host__ __device__ inline int tiles_bin(const SysDesc& d) { return (d.natom + kThreads - 1) / kThreads; }
__host__ __device__ inline int tiles_blocks(const SysDesc& d) { return d.nby * d.nbz; }
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

// Block sum of one int64 per thread; the result is valid in thread 0.  `scratch`: 32 int64.
__device__ __forceinline__ long long block_sum_ll(long long v, long long* scratch) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
  for (int off = 16; off >= 1; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
  __syncthreads();
  if (lane == 0) scratch[warp] = v;
  __syncthreads();
  long long s = 0;
  if (threadIdx.x == 0)
    for (int w = 0; w < nw; w++) s += scratch[w];
  return s;
}

// q^2 of one atom in the sum-of-squares fixed point (one rounding per atom).
__device__ __forceinline__ long long q2_fixed(float q) {
  return __double2ll_rn((double)q * (double)q * kQ2Scale);
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
  long long* red = (long long*)((char*)smem + ((sizeof(SplineAtom<P>) * kSpreadAtoms + 7) / 8) * 8);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const Geom& g = d.g;
  const int base = tile * kSpreadAtoms + warp * APW;
  const int cnt = max(0, min(APW, d.natom - base));
  long long q2 = 0;
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
    q2 = q2_fixed(a.w);
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
    const long long sum = block_sum_ll(q2, red);
    if (threadIdx.x == 0 && sum != 0) atomicAdd((unsigned long long*)&d.acc[kAccQ2], (unsigned long long)sum);
  }
  __syncthreads();
}

template <int P>
__host__ inline size_t spread_smem_bytes() {
  return ((sizeof(SplineAtom<P>) * kSpreadAtoms + 7) / 8) * 8 + 32 * sizeof(double);
}

// ---------------------------------------------------------------------------------------------
// Half-complex grid layout: [kx][z][y] (y fastest), so y-lines are contiguous and each kx plane is
// one contiguous ny*nz block.
// ---------------------------------------------------------------------------------------------
__device__ __forceinline__ size_t cidx(const Geom& g, int kx, int z, int y) {
  return ((size_t)kx * g.nz + z) * g.ny + y;
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
  const int nvalid = min(tx, nrows - row0) * L;   // elements of this tile's rows inside the grid
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
  float2* res = fft_tile(b0, b1, plan, ld, 1, ln, tw, false);
  const int hx = g.hx;
  const FastDiv txd = make_fastdiv(tx), nyd = d.py.n_div;
  for (int idx = tid; idx < hx * tx; idx += kThreads) {
    const int k = fdiv(idx, txd), t = idx - k * tx, row = row0 + t;
    if (row < nrows) {
      const int z = fdiv(row, nyd), y = row - z * g.ny;
      __stcg(&d.cgrid[cidx(g, k, z, y)], res[k * ld + t]);
    }
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
  const FastDiv txd = make_fastdiv(tx), nyd = d.py.n_div;
  for (int i = tid; i < L; i += kThreads) tw[i] = __ldg(&d.tw[plan.tw_off + i]);
  for (int idx = tid; idx < hx * tx; idx += kThreads) {
    const int k = fdiv(idx, txd), t = idx - k * tx, row = row0 + t;
    float2 v = make_float2(0.0f, 0.0f);
    if (row < nrows) {
      const int z = fdiv(row, nyd), y = row - z * g.ny;
      v = __ldcg(&d.cgrid[cidx(g, k, z, y)]);
    }
    b0[k * ld + t] = v;
    if (k >= 1 && L - k >= hx) b0[(L - k) * ld + t] = make_float2(v.x, -v.y);
  }
  __syncthreads();
  TileLane ln(tid, kThreads, tx);
  float2* res = fft_tile(b0, b1, plan, ld, 1, ln, tw, true);
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

// Solve terms of one stored k.  The mirror -k that the reference adds for kx >= 1
// (CudaPMERecip.cu:708-742) has the same |m|^2 and the same eterm (the per-axis factors are
// even in m); its off-diagonal products m_i m_j change sign unless one of the two components sits
// at k = 0 or on an even-length Nyquist plane, where the mirrored index maps onto itself.
// Influence-table view for one tile: the tile's fixed kx values in registers, the y and z tables
// staged in shared memory, all rounded once from the FP64 tables to FP32.
struct KTab {
  float m1, A1;
  const float* my;   // [ny] mhat_y
  const float* mz;   // [nz] mhat_z
  const float* Ay;   // [ny] A_y
  const float* Az;   // [nz] A_z
};

__host__ __device__ inline size_t ktab_smem_bytes(int ny, int nz) { return 2 * sizeof(float) * ((size_t)ny + nz); }

// Stage mhat and A for y and z into `sm` (2 (ny + nz) floats) and load kx's.  The caller
// synchronises before use.
__device__ __forceinline__ KTab stage_ktab(const SysDesc& d, int kx, float* sm) {
  const Geom& g = d.g;
  const int ntot = g.nx + g.ny + g.nz;
  const int nyz = g.ny + g.nz;
  for (int i = threadIdx.x; i < nyz; i += kThreads) {
    sm[i] = (float)__ldcg(&d.ktab[g.nx + i]);
    sm[nyz + i] = (float)__ldcg(&d.ktab[ntot + g.nx + i]);
  }
  KTab t;
  t.m1 = (float)__ldcg(&d.ktab[kx]);
  t.A1 = (float)__ldcg(&d.ktab[ntot + kx]);
  t.my = sm;
  t.mz = sm + g.ny;
  t.Ay = sm + nyz;
  t.Az = sm + nyz + g.ny;
  return t;
}

// Solve one stored element: Q *= eterm (Q(0) = 0) and, when asked, add its energy and virial
// terms (CudaPMERecip.cu:694-742) to the fixed-point accumulators `acc`: each term is rounded to
// an integer number of 2^-32 units once, so the sums are exact and do not depend on how elements
// are split into tiles or batches.  eterm = piv_inv A_x A_y A_z / |m|^2 from the FP64-built
// tables; t = eterm |Q|^2, v = 2 (fac + 1/|m|^2); [t, t (v m1 m1 - 1), t v m1 m2, t v m1 m3,
// t (v m2 m2 - 1), t v m2 m3, t (v m3 m3 - 1)], doubled for kx >= 1 (the mirror -k, which has the
// same |m|^2 and eterm), with the mirror's off-diagonals multiplied by s_i s_j (s = -1 where the
// mirror flips m_i, +1 at k = 0 and on an even-length Nyquist plane).
__device__ __forceinline__ void solve_elem(float2& q, int kx, int ky, int kz, const SysDesc& d,
                                           const KTab& kt, long long* acc) {
  const Geom& g = d.g;
  if (kx == 0 && ky == 0 && kz == 0) {
    q = make_float2(0.0f, 0.0f);
    return;
  }
  // explicit roundings: the same bits in every kernel this is inlined into
  const float m1 = kt.m1, m2 = kt.my[ky], m3 = kt.mz[kz];
  const float inv_msq = __frcp_rn(__fmaf_rn(m3, m3, __fmaf_rn(m2, m2, __fmul_rn(m1, m1))));
  const float eterm =
      __fmul_rn(__fmul_rn(__fmul_rn(__fmul_rn(d.piv_inv_f, kt.A1), kt.Ay[ky]), kt.Az[kz]), inv_msq);
  if (d.calc_ev) {
    const float q2 = __fmaf_rn(q.y, q.y, __fmul_rn(q.x, q.x));
    const bool mirror = kx >= 1;
    const float sx = (2 * kx == g.nx) ? 1.0f : -1.0f;
    const float sy = (ky == 0 || 2 * ky == g.ny) ? 1.0f : -1.0f;
    const float sz = (kz == 0 || 2 * kz == g.nz) ? 1.0f : -1.0f;
    const float t1 = __fmul_rn(__fmul_rn(eterm, q2), (float)kEvScale);
    const float vt = __fmul_rn(2.0f, __fadd_rn(d.fac_f, inv_msq));
    const float w = mirror ? 2.0f : 1.0f;
    const float txy = mirror ? __fadd_rn(1.0f, __fmul_rn(sx, sy)) : 1.0f;
    const float txz = mirror ? __fadd_rn(1.0f, __fmul_rn(sx, sz)) : 1.0f;
    const float tyz = mirror ? __fadd_rn(1.0f, __fmul_rn(sy, sz)) : 1.0f;
    const float wt = __fmul_rn(w, t1);
    const float tv = __fmul_rn(t1, vt);
    acc[0] += __float2ll_rn(wt);
    acc[1] += __float2ll_rn(__fmul_rn(wt, __fmaf_rn(__fmul_rn(vt, m1), m1, -1.0f)));
    acc[2] += __float2ll_rn(__fmul_rn(__fmul_rn(__fmul_rn(txy, tv), m1), m2));
    acc[3] += __float2ll_rn(__fmul_rn(__fmul_rn(__fmul_rn(txz, tv), m1), m3));
    acc[4] += __float2ll_rn(__fmul_rn(wt, __fmaf_rn(__fmul_rn(vt, m2), m2, -1.0f)));
    acc[5] += __float2ll_rn(__fmul_rn(__fmul_rn(__fmul_rn(tyz, tv), m2), m3));
    acc[6] += __float2ll_rn(__fmul_rn(wt, __fmaf_rn(__fmul_rn(vt, m3), m3, -1.0f)));
  }
  q.x = __fmul_rn(q.x, eterm);
  q.y = __fmul_rn(q.y, eterm);
}

// Block-sum 7 int64 partial accumulators and add them to the system's accumulators.
__device__ __forceinline__ void flush_ev(const SysDesc& d, long long (&acc)[7], long long* red) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
  for (int off = 16; off >= 1; off >>= 1)
#pragma unroll
    for (int c = 0; c < 7; c++) acc[c] += __shfl_down_sync(0xffffffffu, acc[c], off);
  __syncthreads();
  if (lane == 0)
#pragma unroll
    for (int c = 0; c < 7; c++) red[warp * 7 + c] = acc[c];
  __syncthreads();
  if (threadIdx.x < 7) {
    long long sum = 0;
    for (int w = 0; w < nw; w++) sum += red[w * 7 + threadIdx.x];
    atomicAdd((unsigned long long*)&d.acc[kAccE + threadIdx.x], (unsigned long long)sum);
  }
}

// y pass: tx_y consecutive y-lines (line = kx nz + z, contiguous ny values).  mode 0 forward,
// 1 inverse.  smem: twiddles + two tile buffers.
__device__ __forceinline__ void y_tile(const SysDesc& d, int mode, int tile, float2* smem) {
  const Geom& g = d.g;
  const FftPlan1D& plan = d.py;
  const int L = g.ny, tx = d.tx_y, ld = tx + 1;
  float2* tw = smem;
  float2* b0 = tw + L;
  float2* b1 = b0 + L * ld;
  const int tid = threadIdx.x;
  const int nlines = g.hx * g.nz, l0 = tile * tx;
  const int nvalid = min(tx, nlines - l0) * L;
  float2* __restrict__ base = d.cgrid + (size_t)l0 * L;
  for (int i = tid; i < L; i += kThreads) tw[i] = __ldg(&d.tw[plan.tw_off + i]);
#pragma unroll 4
  for (int idx = tid; idx < L * tx; idx += kThreads) {
    const int t = fdiv(idx, plan.n_div), e = idx - t * L;
    b0[e * ld + t] = idx < nvalid ? __ldcg(&base[idx]) : make_float2(0.0f, 0.0f);
  }
  __syncthreads();
  TileLane ln(tid, kThreads, tx);
  float2* res = fft_tile(b0, b1, plan, ld, 1, ln, tw, mode == 1);
  for (int idx = tid; idx < nvalid; idx += kThreads) {
    const int t = fdiv(idx, plan.n_div), e = idx - t * L;
    __stcg(&base[idx], res[e * ld + t]);
  }
  __syncthreads();
}

// z pass: tx_z consecutive y at one kx, all z (element row of the tile = tx contiguous complex).
// mode: 0 forward, 1 inverse, 2 forward + solve + inverse, 3 solve only.
// smem: twiddles, two tile buffers, 32*7 int64.
__device__ __forceinline__ void z_tile(const SysDesc& d, int mode, int tile, float2* smem) {
  const Geom& g = d.g;
  const FftPlan1D& plan = d.pz;
  const int L = g.nz, tx = d.tx_z, ld = tx + 1;
  float2* tw = smem;
  float2* b0 = tw + L;
  float2* b1 = b0 + L * ld;
  long long* red = (long long*)(b1 + L * ld);
  float* ksm = (float*)(red + 32 * 7);
  const int tid = threadIdx.x;
  const int tpk = (g.ny + tx - 1) / tx;
  const int kx = tile / tpk, y0 = (tile - kx * tpk) * tx;
  const int nt = min(tx, g.ny - y0);
  const FastDiv txd = make_fastdiv(tx);
  float2* __restrict__ base = d.cgrid + cidx(g, kx, 0, y0);
  const size_t es = (size_t)g.ny;
  if (mode != 3)
    for (int i = tid; i < L; i += kThreads) tw[i] = __ldg(&d.tw[plan.tw_off + i]);
  for (int idx = tid; idx < L * tx; idx += kThreads) {
    const int e = fdiv(idx, txd), t = idx - e * tx;
    b0[e * ld + t] = t < nt ? __ldcg(&base[e * es + t]) : make_float2(0.0f, 0.0f);
  }
  __syncthreads();
  TileLane ln(tid, kThreads, tx);
  float2* res = b0;
  if (mode == 0 || mode == 2) res = fft_tile(b0, b1, plan, ld, 1, ln, tw, false);
  if (mode == 1) res = fft_tile(b0, b1, plan, ld, 1, ln, tw, true);
  if (mode == 2 || mode == 3) {
    const KTab kt = stage_ktab(d, kx, ksm);
    __syncthreads();
    long long acc[7] = {0, 0, 0, 0, 0, 0, 0};
    for (int idx = tid; idx < L * tx; idx += kThreads) {
      const int e = fdiv(idx, txd), t = idx - e * tx;
      if (t < nt) solve_elem(res[e * ld + t], kx, y0 + t, e, d, kt, acc);
    }
    if (d.calc_ev) flush_ev(d, acc, red);
    __syncthreads();
    if (mode == 2) {
      float2* other = (res == b0) ? b1 : b0;
      res = fft_tile(res, other, plan, ld, 1, ln, tw, true);
    }
  }
  for (int idx = tid; idx < L * tx; idx += kThreads) {
    const int e = fdiv(idx, txd), t = idx - e * tx;
    if (t < nt) __stcg(&base[e * es + t], res[e * ld + t]);
  }
  __syncthreads();
}

// Whole kx plane (ny x nz, contiguous): y forward, z forward, solve with energy/virial, z inverse,
// y inverse, all in shared memory (plane held as buf[z * (ny+1) + y]).  Used when the plane fits.
__host__ __device__ inline size_t plane_smem_bytes(int ny, int nz) {
  return sizeof(float2) * ((size_t)ny + nz + 2 * (size_t)nz * (ny + 1)) + 32 * 7 * sizeof(long long) +
         2 * sizeof(float) * ((size_t)ny + nz);
}

__device__ __forceinline__ void plane_tile(const SysDesc& d, int kx, float2* smem) {
  const Geom& g = d.g;
  const int ny = g.ny, nz = g.nz, LD = ny + 1;
  float2* twy = smem;
  float2* twz = twy + ny;
  float2* b0 = twz + nz;
  float2* b1 = b0 + (size_t)nz * LD;
  long long* red = (long long*)(b1 + (size_t)nz * LD);
  float* ksm = (float*)(red + 32 * 7);
  const int tid = threadIdx.x;
  float2* __restrict__ base = d.cgrid + cidx(g, kx, 0, 0);
  step_mark(d, 8);
  const KTab kt = stage_ktab(d, kx, ksm);
  for (int i = tid; i < ny; i += kThreads) twy[i] = __ldg(&d.tw[d.py.tw_off + i]);
  for (int i = tid; i < nz; i += kThreads) twz[i] = __ldg(&d.tw[d.pz.tw_off + i]);
  const FastDiv nyd = d.py.n_div;
#pragma unroll 4
  for (int idx = tid; idx < ny * nz; idx += kThreads) {
    const int z = fdiv(idx, nyd), y = idx - z * ny;
    b0[z * LD + y] = __ldcg(&base[idx]);
  }
  __syncthreads();
  step_mark(d, 9);
  const TileLane lz(tid, kThreads, nz);   // y-FFT: one line per z
  const TileLane ly(tid, kThreads, ny);   // z-FFT: one line per y
  float2* r = fft_tile(b0, b1, d.py, 1, LD, lz, twy, false);
  step_mark(d, 10);
  float2* o = (r == b0) ? b1 : b0;
  r = fft_tile(r, o, d.pz, LD, 1, ly, twz, false);
  step_mark(d, 11);
  long long acc[7] = {0, 0, 0, 0, 0, 0, 0};
  for (int idx = tid; idx < ny * nz; idx += kThreads) {
    const int z = fdiv(idx, nyd), y = idx - z * ny;
    solve_elem(r[z * LD + y], kx, y, z, d, kt, acc);
  }
  if (d.calc_ev) flush_ev(d, acc, red);
  __syncthreads();
  step_mark(d, 12);
  o = (r == b0) ? b1 : b0;
  r = fft_tile(r, o, d.pz, LD, 1, ly, twz, true);
  o = (r == b0) ? b1 : b0;
  r = fft_tile(r, o, d.py, 1, LD, lz, twy, true);
  step_mark(d, 13);
  for (int idx = tid; idx < ny * nz; idx += kThreads) {
    const int z = fdiv(idx, nyd), y = idx - z * ny;
    __stcg(&base[idx], r[z * LD + y]);
  }
  __syncthreads();
  step_mark(d, 14);
}

// ---------------------------------------------------------------------------------------------
// Fused path, phase 0: bin kThreads atoms by the row block of their stencil origin; sum q^2.
// A bin entry is the atom's record: stencil origin (ix, iy, iz as int bits) and atom index, then
// the FP32 spreading weights q*thx[P], thy[P], thz[P] -- the values the staged spread uses --
// padded to a multiple of 4 floats so that every record is 16-byte aligned.
// ---------------------------------------------------------------------------------------------
__host__ __device__ constexpr int rec_floats(int order) { return (4 + 3 * order + 3) & ~3; }

template <int P>
__device__ __forceinline__ void bin_tile_p(const SysDesc& d, int tile, int parity, long long* red) {
  constexpr int RF = rec_floats(P);
  const Geom& g = d.g;
  const int i = tile * kThreads + threadIdx.x;
  const int nbins = d.nby * d.nbz;
  long long q2 = 0;
  if (i < d.natom) {
    const float4 a = __ldg(&d.xyzq[i]);
    int ix, iy, iz;
    float ux, uy, uz;
    frac_coord(a.x, g.sx_hi, g.sx_lo, g.nx, ix, ux);
    frac_coord(a.y, g.sy_hi, g.sy_lo, g.ny, iy, uy);
    frac_coord(a.z, g.sz_hi, g.sz_lo, g.nz, iz, uz);
    float w[RF - 4];
#pragma unroll
    for (int k = 3 * P; k < RF - 4; k++) w[k] = 0.0f;
    bspline<P>(ux, w, nullptr);
#pragma unroll
    for (int k = 0; k < P; k++) w[k] = __fmul_rn(a.w, w[k]);
    bspline<P>(uy, w + P, nullptr);
    bspline<P>(uz, w + 2 * P, nullptr);
    const int b = iy / d.bry + d.nby * (iz / d.brz);
    const int slot = atomicAdd(&d.bin_count[parity * nbins + b], 1);
    float* rec;
    if (slot < d.bin_cap) {
      rec = d.bin_recs + ((size_t)b * d.bin_cap + slot) * RF;
    } else {
      const int o = atomicAdd(&d.ovf_count[parity], 1);
      rec = d.ovf_recs + (size_t)o * RF;
    }
    float4* r4 = (float4*)rec;
    __stcg(&r4[0], make_float4(__int_as_float(ix), __int_as_float(iy), __int_as_float(iz), __int_as_float(i)));
#pragma unroll
    for (int c = 0; c < (RF - 4) / 4; c++)
      __stcg(&r4[1 + c], make_float4(w[4 * c], w[4 * c + 1], w[4 * c + 2], w[4 * c + 3]));
    q2 = q2_fixed(a.w);
  }
  if (d.calc_self) {
    const long long sum = block_sum_ll(q2, red);
    if (threadIdx.x == 0 && sum != 0) atomicAdd((unsigned long long*)&d.acc[kAccQ2], (unsigned long long)sum);
  }
  __syncthreads();
}

__device__ __forceinline__ void bin_tile(const SysDesc& d, int tile, int parity, long long* red) {
  switch (d.order) {
    case 4: bin_tile_p<4>(d, tile, parity, red); break;
    case 6: bin_tile_p<6>(d, tile, parity, red); break;
    default: bin_tile_p<8>(d, tile, parity, red); break;
  }
}

// ---------------------------------------------------------------------------------------------
// Fused path, phase 1: spread + x forward for one row block (rows y in [Y0, Y0+bry), z in
// [Z0, Z0+brz), all x).  The block's candidate atoms are the records of the row blocks whose
// origins can reach it (origin rows Y0-P+1 .. Y0+bry-1, wrapped), plus the overflow records.
// Each contribution that lands in the block is added to an int64 row in shared memory (exact, so
// the result equals the staged spread's fixed-point grid bit for bit), then the rows are converted
// to FP32 and x-transformed in place.
//
// The work is split so that every lane does the same amount: a round takes up to kSpreadSlots
// candidates; step A tests each against the block and lists the ones that reach it (their x
// weights and their y/z weights re-indexed by block row) and one item per (atom, block row) it
// covers; step B gives each lane one item at a time, i.e. the P contributions of one stencil row.
// The accumulator rows have an odd stride, so the rows of one atom fall in different banks.
// ---------------------------------------------------------------------------------------------
constexpr int kSpreadSlots = 2 * kThreads;          // candidates per round (listed-atom slots)
constexpr int kSpreadMaxBlock = 4;                  // row-block edge limit (bry, brz)
constexpr int kSpreadItemCap = kSpreadSlots * kSpreadMaxBlock * kSpreadMaxBlock;
constexpr int kSpreadBookInts = 168;                // candidate bins, counts, offsets, counters

__host__ __device__ inline int spread_row_stride(int nx) { return nx | 1; }
__host__ __device__ inline size_t align16(size_t b) { return (b + 15) & ~(size_t)15; }

// smem of the spread + x tile: 3 x 32-bit accumulators per point, twiddles, bookkeeping, then a
// work area that holds the listed atoms and items while spreading and the FFT buffers after.
__host__ __device__ inline size_t spread_x_smem_bytes(int nx, int rows, int order) {
  const size_t acc = align16((size_t)rows * spread_row_stride(nx) * 12);
  const size_t fft = (size_t)2 * nx * (rows + 1) * sizeof(float2);
  const size_t lists = (size_t)kSpreadSlots * (1 + order + 2 * kSpreadMaxBlock) * 4 +
                       (size_t)kSpreadItemCap * sizeof(unsigned short);
  return acc + align16((size_t)nx * sizeof(float2)) + kSpreadBookInts * sizeof(int) + (fft > lists ? fft : lists);
}

// Exact int64 accumulation in shared memory with native 32-bit atomics.  A contribution
// v = p0 + p1 2^16 + p2 2^32 (p0, p1 in [0, 2^16), p2 = v >> 32 signed) is added to three 32-bit
// sums without using the atomics' return values (no dependent round trips).  The p0 and p1 sums
// cannot wrap while a point receives at most 2^16 contributions, which the tile guarantees by
// checking its candidate count; the p2 sum may wrap, harmlessly, since only its value modulo 2^32
// enters the int64 result.  Beyond that count the carry form is used: lo (u32) + hi (s32), the
// wrap of lo detected from the returned old value.
__device__ __forceinline__ void add_fixed_split3(unsigned int* s0, unsigned int* s1, int* s2, int idx,
                                                 long long v) {
  const unsigned long long u = (unsigned long long)v;
  const unsigned int p0 = (unsigned int)(u & 0xffffull), p1 = (unsigned int)((u >> 16) & 0xffffull);
  const int p2 = (int)(v >> 32);
  atomicAdd(&s0[idx], p0);
  atomicAdd(&s1[idx], p1);
  if (p2 != 0) atomicAdd(&s2[idx], p2);
}

__device__ __forceinline__ void add_fixed_carry(unsigned int* lo, int* hi, int idx, long long v) {
  const unsigned int l = (unsigned int)(unsigned long long)v;
  const int h = (int)(v >> 32);
  const unsigned int old = atomicAdd(&lo[idx], l);
  const int carry = (old + l) < old ? 1 : 0;
  if (h + carry != 0) atomicAdd(&hi[idx], h + carry);
}

// The listed atoms of a round, structure of arrays over kSpreadSlots slots:
//   ix[slot]; w[k][slot] = q thx[k] (k < P); w[P + ry][slot] = thy of block row ry;
//   w[P + kSpreadMaxBlock + rz][slot] = thz of block row rz.
// An item is slot | ry << 9 | rz << 11.
struct SpreadLists {
  int* ix;
  float* w;
  unsigned short* items;
  int* counters;   // [0] listed atoms, [1] items
};

// Step A for one candidate record per lane (rec == nullptr: no candidate).  Every lane of the
// warp calls it.
template <int P>
__device__ __forceinline__ void spread_list_atom(const SysDesc& d, const float* rec, int Y0, int Z0, int nry,
                                                 int nrz, const SpreadLists& sl) {
  constexpr int S = kSpreadSlots;
  const Geom& g = d.g;
  const int lane = threadIdx.x & 31;
  unsigned int my = 0u, mz = 0u;   // block rows covered by the stencil
  int ix = 0, ry0 = 0, rz0 = 0;
  if (rec != nullptr) {
    const float4 h = __ldcg((const float4*)rec);
    ix = __float_as_int(h.x);
    ry0 = __float_as_int(h.y) - Y0;
    if (ry0 < 0) ry0 += g.ny;
    rz0 = __float_as_int(h.z) - Z0;
    if (rz0 < 0) rz0 += g.nz;
#pragma unroll
    for (int b = 0; b < P; b++) {
      int y = ry0 + b;
      if (y >= g.ny) y -= g.ny;
      if (y < nry) my |= 1u << y;
      int z = rz0 + b;
      if (z >= g.nz) z -= g.nz;
      if (z < nrz) mz |= 1u << z;
    }
  }
  const int nrow = __popc(my) * __popc(mz);
  const unsigned int act = __ballot_sync(0xffffffffu, nrow > 0);
  if (act == 0u) return;
  int incl = nrow;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int t = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += t;
  }
  const int wtot = __shfl_sync(0xffffffffu, incl, 31);
  int sbase = 0, ibase = 0;
  if (lane == 0) {
    sbase = atomicAdd(&sl.counters[0], __popc(act));
    ibase = atomicAdd(&sl.counters[1], wtot);
  }
  sbase = __shfl_sync(0xffffffffu, sbase, 0);
  ibase = __shfl_sync(0xffffffffu, ibase, 0);
  if (nrow == 0) return;
  const int slot = sbase + __popc(act & ((1u << lane) - 1u));
  constexpr int NW = rec_floats(P) - 4;
  float w[NW];
  const float4* r4 = (const float4*)rec + 1;
#pragma unroll
  for (int c = 0; c < NW / 4; c++) {
    const float4 v = __ldcg(&r4[c]);
    w[4 * c] = v.x;
    w[4 * c + 1] = v.y;
    w[4 * c + 2] = v.z;
    w[4 * c + 3] = v.w;
  }
  sl.ix[slot] = ix;
#pragma unroll
  for (int k = 0; k < P; k++) sl.w[k * S + slot] = w[k];
#pragma unroll
  for (int b = 0; b < P; b++) {
    int y = ry0 + b;
    if (y >= g.ny) y -= g.ny;
    if (y < nry) sl.w[(P + y) * S + slot] = w[P + b];
    int z = rz0 + b;
    if (z >= g.nz) z -= g.nz;
    if (z < nrz) sl.w[(P + kSpreadMaxBlock + z) * S + slot] = w[2 * P + b];
  }
  int r = ibase + incl - nrow;
  unsigned int mzz = mz;
  while (mzz) {
    const int rz = __ffs(mzz) - 1;
    mzz &= mzz - 1;
    unsigned int myy = my;
    while (myy) {
      const int ry = __ffs(myy) - 1;
      myy &= myy - 1;
      sl.items[r++] = (unsigned short)(slot | ry << 9 | rz << 11);
    }
  }
}

// Step B: the P contributions of one (atom, block row) item per lane.
template <int P, bool SPLIT3>
__device__ __forceinline__ void spread_items(const SpreadLists& sl, int nitems, int nry, int L, int Lp,
                                             unsigned int* s0, unsigned int* s1, int* s2) {
  constexpr int S = kSpreadSlots;
  for (int j = threadIdx.x; j < nitems; j += kThreads) {
    const unsigned int it = sl.items[j];
    const int slot = it & 511u, ry = (it >> 9) & 3u, rz = it >> 11;
    const int ix = sl.ix[slot];
    const float ty = sl.w[(P + ry) * S + slot];
    const float tz = sl.w[(P + kSpreadMaxBlock + rz) * S + slot];
    const int rb = (ry + nry * rz) * Lp;
#pragma unroll
    for (int k = 0; k < P; k++) {
      int x = ix + k;
      if (x >= L) x -= L;
      const long long v = fixed_contrib(sl.w[k * S + slot], ty, tz);
      if (SPLIT3) add_fixed_split3(s0, s1, s2, rb + x, v);
      else add_fixed_carry(s0, s2, rb + x, v);
    }
  }
}

template <int P>
__device__ __forceinline__ void spread_x_tile(const SysDesc& d, int tile, int parity, char* smem_raw) {
  constexpr int RF = rec_floats(P);
  constexpr int S = kSpreadSlots;
  const Geom& g = d.g;
  const FftPlan1D& plan = d.px;
  const int L = g.nx, Lp = spread_row_stride(L);
  const int by = tile % d.nby, bz = tile / d.nby;
  const int Y0 = by * d.bry, Z0 = bz * d.brz;
  const int nry = min(d.bry, g.ny - Y0), nrz = min(d.brz, g.nz - Z0);
  const int rows = d.bry * d.brz;            // FFT lines of the tile (rows beyond nry*nrz are 0)
  const int ld = rows + 1;
  const int tid = threadIdx.x;
  unsigned int* s0 = (unsigned int*)smem_raw;
  unsigned int* s1 = s0 + (size_t)rows * Lp;
  int* s2 = (int*)(s1 + (size_t)rows * Lp);
  char* p = smem_raw + align16((size_t)rows * Lp * 12);
  float2* tw = (float2*)p;
  p += align16((size_t)L * sizeof(float2));
  int* cand = (int*)p;                         // [0..7] y bins, [8..15] z bins, [16] #y, [17] #z
  int* ccnt = cand + 32;                       // [64] counts of the candidate bins
  int* coff = ccnt + 64;                       // [65] their offsets
  p += kSpreadBookInts * sizeof(int);
  SpreadLists sl;
  sl.ix = (int*)p;
  sl.w = (float*)(sl.ix + S);
  sl.items = (unsigned short*)(sl.w + (size_t)(P + 2 * kSpreadMaxBlock) * S);
  sl.counters = cand + 18;
  float2* b0 = (float2*)p;                     // FFT view of the work area (after spreading)
  float2* b1 = b0 + (size_t)L * ld;
  const int nbins = d.nby * d.nbz;
  step_mark(d, 0);
  for (int idx = tid; idx < rows * Lp; idx += kThreads) {
    s0[idx] = 0u;
    s1[idx] = 0u;
    s2[idx] = 0;
  }
  for (int i = tid; i < L; i += kThreads) tw[i] = __ldg(&d.tw[plan.tw_off + i]);
  // Candidate bins: the origin rows Y0-P+1 .. Y0+nry-1 (wrapped) cover consecutive bins
  // b0, b0+1, ..., by (mod nby); all bins when the window spans the whole axis.  Same for z.
  // At most ceil((P-1)/bry) + 2 <= 8 bins per axis.
  if (tid < 2) {
    const int n = tid == 0 ? g.ny : g.nz, br = tid == 0 ? d.bry : d.brz;
    const int nb = tid == 0 ? d.nby : d.nbz, own = tid == 0 ? by : bz;
    const int R0 = tid == 0 ? Y0 : Z0, nr = tid == 0 ? nry : nrz;
    const int W = P - 1 + nr;
    int* out = cand + 8 * tid;
    if (W >= n) {
      for (int k = 0; k < nb; k++) out[k] = k;
      cand[16 + tid] = nb;
    } else {
      int r0 = (R0 - P + 1) % n;
      if (r0 < 0) r0 += n;
      const int b0 = r0 / br;
      int cnt = own - b0;
      if (cnt < 0) cnt += nb;
      cnt += 1;
      for (int k = 0; k < cnt; k++) {
        const int b = b0 + k;
        out[k] = b >= nb ? b - nb : b;
      }
      cand[16 + tid] = cnt;
    }
    sl.counters[tid] = 0;
  }
  __syncthreads();
  const int ncy = cand[16], ncz = cand[17], nc = ncy * ncz;
  if (tid < nc) {
    const int b = cand[tid % ncy] + d.nby * cand[8 + tid / ncy];
    ccnt[tid] = min(__ldcg(&d.bin_count[parity * nbins + b]), d.bin_cap);
  }
  __syncthreads();
  if (tid == 0) {
    int o = 0;
    for (int c = 0; c < nc; c++) { coff[c] = o; o += ccnt[c]; }
    coff[nc] = o;
  }
  __syncthreads();
  const int total = coff[nc];
  step_mark(d, 1);
  const int ncand = total + __ldcg(&d.ovf_count[parity]);
  // at most one contribution per candidate and point: up to 2^16 candidates the split form is exact
  const bool split3 = ncand <= 65536;
  for (int base0 = 0; base0 < ncand; base0 += S) {
#pragma unroll 1
    for (int h = 0; h < S; h += kThreads) {
      const int q = base0 + h + tid;
      const float* rec = nullptr;
      if (q < total) {
        int c = 0;
        while (q >= coff[c + 1]) c++;
        const int b = cand[c % ncy] + d.nby * cand[8 + c / ncy];
        rec = d.bin_recs + ((size_t)b * d.bin_cap + (q - coff[c])) * RF;
      } else if (q < ncand) {
        rec = d.ovf_recs + (size_t)(q - total) * RF;
      }
      spread_list_atom<P>(d, rec, Y0, Z0, nry, nrz, sl);
    }
    __syncthreads();
    if (base0 == 0) step_mark(d, 2);
    const int ni = sl.counters[1];
    if (split3) spread_items<P, true>(sl, ni, nry, L, Lp, s0, s1, s2);
    else spread_items<P, false>(sl, ni, nry, L, Lp, s0, s1, s2);
    __syncthreads();
    if (tid < 2) sl.counters[tid] = 0;
    __syncthreads();
  }
  step_mark(d, 3);
  // the other parity's counters are cleared for the next launch by the system's first block
  if (tile == 0) {
    for (int j = tid; j < nbins; j += kThreads) d.bin_count[(1 - parity) * nbins + j] = 0;
    if (tid == 0) d.ovf_count[1 - parity] = 0;
  }
  // rows: r = ry + nry*rz (r < nry*nrz valid); FFT line t = r
  for (int idx = tid; idx < rows * L; idx += kThreads) {
    const int t = fdiv(idx, plan.n_div), e = idx - t * L;
    const int a = t * Lp + e;
    // split: p0 + p1 2^16 + p2 2^32; carry form: s0 = lo, s1 = 0, s2 = hi -- one formula
    const unsigned long long u = (unsigned long long)s0[a] + ((unsigned long long)s1[a] << 16) +
                                 ((unsigned long long)(unsigned int)s2[a] << 32);
    b0[e * ld + t] = make_float2(fixed_to_float((long long)u), 0.0f);
  }
  __syncthreads();
  step_mark(d, 4);
  TileLane ln(tid, kThreads, rows);
  float2* res = fft_tile(b0, b1, plan, ld, 1, ln, tw, false);
  step_mark(d, 5);
  const int hx = g.hx;
  const FastDiv rd = make_fastdiv(rows), nryd = make_fastdiv(nry);
  const int nvalid = nry * nrz;
  for (int idx = tid; idx < hx * rows; idx += kThreads) {
    const int k = fdiv(idx, rd), t = idx - k * rows;
    if (t < nvalid) {
      const int rz = fdiv(t, nryd), ry = t - rz * nry;
      __stcg(&d.cgrid[cidx(g, k, Z0 + rz, Y0 + ry)], res[k * ld + t]);
    }
  }
  __syncthreads();
  step_mark(d, 6);
}

__device__ __forceinline__ void spread_x_dispatch(const SysDesc& d, int tile, int parity, char* smem) {
  switch (d.order) {
    case 4: spread_x_tile<4>(d, tile, parity, smem); break;
    case 6: spread_x_tile<6>(d, tile, parity, smem); break;
    default: spread_x_tile<8>(d, tile, parity, smem); break;
  }
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
__device__ __forceinline__ void gather_atom(const SysDesc& d, int atom, bool valid, int gl) {
  const Geom& g = d.g;
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

template <int P, int KIND>
__device__ __forceinline__ void gather_tile(const SysDesc& d, int tile) {
  const int atom = tile * 32 + (threadIdx.x >> 3), gl = threadIdx.x & 7;
  gather_atom<P, KIND>(d, atom, atom < d.natom, gl);
}

// Fused path: gather the atoms of one row-block bin (plus the overflow atoms whose origin lies in
// the block), 32 at a time, so that the tile's stencil rows (about (4+P-1)^2 grid rows) stay in L1.
template <int P, int KIND>
__device__ __forceinline__ void gather_bin_tile(const SysDesc& d, int tile, int parity) {
  constexpr int RF = rec_floats(P);
  const int nbins = d.nby * d.nbz;
  const int cnt = min(__ldcg(&d.bin_count[parity * nbins + tile]), d.bin_cap);
  const float* list = d.bin_recs + (size_t)tile * d.bin_cap * RF;
  const int gl = threadIdx.x & 7, slot = threadIdx.x >> 3;
  for (int j0 = 0; j0 < cnt; j0 += 32) {
    const int j = j0 + slot;
    const bool valid = j < cnt;
    gather_atom<P, KIND>(d, valid ? __float_as_int(__ldcg(&list[(size_t)j * RF + 3])) : 0, valid, gl);
  }
  const int novf = __ldcg(&d.ovf_count[parity]);
  for (int j0 = 0; j0 < novf; j0 += 32) {
    const int j = j0 + slot;
    int atom = 0;
    bool mine = false;
    if (j < novf) {
      const float4 h = __ldcg((const float4*)(d.ovf_recs + (size_t)j * RF));
      atom = __float_as_int(h.w);
      mine = (__float_as_int(h.y) / d.bry + d.nby * (__float_as_int(h.z) / d.brz)) == tile;
    }
    gather_atom<P, KIND>(d, atom, mine, gl);
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

template <int P>
__device__ __forceinline__ void gather_bin_any(const SysDesc& d, int tile, int parity) {
  switch (d.force_kind) {
    case kForceF32Soa: gather_bin_tile<P, kForceF32Soa>(d, tile, parity); break;
    case kForceF32x3: gather_bin_tile<P, kForceF32x3>(d, tile, parity); break;
    default: gather_bin_tile<P, kForceI64SoaAccum>(d, tile, parity); break;
  }
}

__device__ __forceinline__ void gather_bin_dispatch(const SysDesc& d, int tile, int parity) {
  switch (d.order) {
    case 4: gather_bin_any<4>(d, tile, parity); break;
    case 6: gather_bin_any<6>(d, tile, parity); break;
    default: gather_bin_any<8>(d, tile, parity); break;
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

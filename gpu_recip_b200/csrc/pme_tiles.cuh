// pme_tiles.cuh -- per-tile device functions of the PME reciprocal path, shared by the staged
// kernels (one tile per CTA) and the persistent fused kernel (tiles of many systems, grid
// barriers between phases).  Every function assumes blockDim.x == kThreads and must be called
// by all threads of the CTA (they synchronise internally).
//
// Energy and virial terms are rounded per element to integers at scale 2^32 and sum(q^2) per atom
// at 2^40; they are summed as int64 inside the CTA and added to per-system int64 accumulators.
// Integer addition is associative, so the totals are bit-identical for any tiling, launch shape
// or batch mix; a finalize step converts them into the FP64 energy/virial record.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <cooperative_groups.h>

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

// Per-system bin bookkeeping (SysDesc::bin_meta).
enum BinMeta { kMetaOvf = 0, kMetaQmax = 2, kMetaPermNatom = 4, kMetaInts = 8 };

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
  double rm[9];              // triclinic: reciprocal matrix R[j][d] (index 3 j + d), FP64
  double gdiag[3];           // triclinic: metric diagonal G_dd = sum_j R[j][d]^2
  float cross_f[3];          // triclinic: -2 fac G_xy, -2 fac G_xz, -2 fac G_yz
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
  double* ktab;              // influence tables, 4 rows of nx+ny+nz (see ktab_tile)
  const float2* tw;          // twiddles x | y | z (plan.tw_off)
  long long* acc;            // kAccCount fixed-point accumulators
  double* ev;                // kEvCount record
  double* ev_mirror;         // optional device-mapped host copy of each evaluation's own record
  int tx_rows, tx_y, tx_z;   // lines per tile of the x, y, z passes
  int plane;                 // 1: the fused path runs y, z and the solve as whole-plane tiles
  int cplane;                // > 0: ... as kx planes split over a thread-block cluster of this
                             // many CTAs (cplane_tile), in a launch with that cluster size
  int bin_atoms;             // atoms per bin tile of the fused path (0: kThreads)
  int xyzq_host;             // 1: xyzq is pinned host memory, read once in index order
  int gx;                    // 1: each gather tile runs the inverse x pass of the rows it reads
                             // (fused path; no x-inverse phase)
  int gsort;                 // 1: each gather tile (without gx) takes its atoms in order of their
                             // stencil origin along x (a counting sort in shared memory)
  // Atom bins of the fused path: bin (by, bz) holds the atoms whose stencil origin (iy0, iz0)
  // lies in row block [by*bry, by*bry+bry) x [bz*brz, bz*brz+brz); fixed capacity bin_cap per bin,
  // surplus atoms go to an overflow list.  Counters are double-buffered by launch parity.
  int bry, brz, nby, nbz;
  int bin_cap;
  int* bin_count;            // [2][nby*nbz]
  float* bin_recs;           // [nby*nbz][bin_cap] atom records of rec_floats(order) floats
  int* bin_meta;             // [8]: overflow counts [2] and max |q| as float bits [2] by launch
                             // parity, the atom count the bin-sorted order was built for
  float* ovf_recs;           // [natom capacity] records of the atoms beyond a bin's capacity
  int* perm;                 // [natom capacity] bin-sorted atom order of the previous evaluation
  unsigned long long* steps; // profiling: %globaltimer at the steps of CTA 0's tiles (or null)
};

// Profiling stamp of one step of a tile (CTA 0, thread 0 only; no-op when steps is null).
// Slots: 0-6 the spread + x tile (start, candidates counted, first round listed, spreading done,
// rows converted, x FFT done, stored), 8-14 the plane tile (or the cluster plane tile: start,
// loaded, y FFT, transposed, solved, transposed back, done), 16-21 the bin tile, 24-26 the gather
// tile; a CTA that runs several tiles of a phase leaves the stamps of its last one.
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
// atoms per bin tile: kThreads, or fewer when the host asks for more, smaller tiles (bin_atoms)
__host__ __device__ inline int bin_tile_atoms(const SysDesc& d) { return d.bin_atoms > 0 ? d.bin_atoms : kThreads; }
__host__ __device__ inline int tiles_bin(const SysDesc& d) { return (d.natom + bin_tile_atoms(d) - 1) / bin_tile_atoms(d); }
__host__ __device__ inline int tiles_blocks(const SysDesc& d) { return d.nby * d.nbz; }
// Lanes per atom of the gather (staged and fused): as few as keep the rows of one lane,
// P^2 / lanes, at 8-9, so that a bin's atoms take few passes.
__host__ __device__ constexpr int gather_lanes(int order) { return order <= 4 ? 2 : (order <= 6 ? 4 : 8); }
constexpr int kGatherAtoms = kThreads / 8;   // staged gather tile: atoms of the smallest pass
__host__ __device__ inline int tiles_gather(const SysDesc& d) {
  const int app = kThreads / gather_lanes(d.order);
  return (d.natom + app - 1) / app;
}
__host__ inline size_t tile_smem_bytes(int L, int tx) {
  return sizeof(float2) * ((size_t)L + 2 * (size_t)L * (tx + 1));
}

// ---------------------------------------------------------------------------------------------
// Block reductions
// ---------------------------------------------------------------------------------------------
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
    frac_coords(g, a.x, a.y, a.z, s.ix, s.iy, s.iz, ux, uy, uz);
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
// Triclinic boxes: k = R m = sum_d m_d R[.][d], so each axis contributes a vector; |k|^2 =
// sum_dd' G_dd' m_d m_d' (G = R^T R) keeps the per-axis factors A_d = b_d exp(-fac G_dd m_d^2) and
// adds one cross factor exp(-2 fac (G_xy m_x m_y + G_xz m_x m_z + G_yz m_y m_z)) per element.
// Table layout (ntot = nx+ny+nz entries each): [0] k_x contribution (mhat_d when orthorhombic),
// [1] A_d, and for triclinic boxes [2] k_y and [3] k_z contributions.
// ---------------------------------------------------------------------------------------------
// Table entry i (x entries, then y, then z): v[0] k contribution (mhat), v[1] A; triclinic boxes
// also v[2], v[3] (k_y and k_z contributions).
__device__ __forceinline__ void ktab_entry(const SysDesc& d, int i, double* v) {
  const Geom& g = d.g;
  int n, k, ax;
  double r;
  if (i < g.nx) { n = g.nx; k = i; r = d.rxd; ax = 0; }
  else if (i < g.nx + g.ny) { n = g.ny; k = i - g.nx; r = d.ryd; ax = 1; }
  else { n = g.nz; k = i - g.nx - g.ny; r = d.rzd; ax = 2; }
  const int nf = (n >> 1) + (n & 1);
  const int m = k < nf ? k : k - n;
  if (!g.tric) {
    const double mh = r * (double)m;
    v[0] = mh;
    v[1] = d.bmod[i] * exp(-d.fac * mh * mh);
  } else {
    const double md = (double)m;
    v[0] = d.rm[ax] * md;
    v[1] = d.bmod[i] * exp(-d.fac * d.gdiag[ax] * md * md);
    v[2] = d.rm[3 + ax] * md;
    v[3] = d.rm[6 + ax] * md;
  }
}

__device__ __forceinline__ void ktab_tile(const SysDesc& d) {
  const Geom& g = d.g;
  const int ntot = g.nx + g.ny + g.nz;
  for (int i = threadIdx.x; i < ntot; i += kThreads) {
    double v[4];
    ktab_entry(d, i, v);
    d.ktab[i] = v[0];
    d.ktab[ntot + i] = v[1];
    if (g.tric) {
      d.ktab[2 * ntot + i] = v[2];
      d.ktab[3 * ntot + i] = v[3];
    }
  }
}

// Solve terms of one stored k.  The mirror -k that the reference adds for kx >= 1
// (CudaPMERecip.cu:708-742) has the same |m|^2 and the same eterm (the per-axis factors are
// even in m); its off-diagonal products m_i m_j change sign unless one of the two components sits
// at k = 0 or on an even-length Nyquist plane, where the mirrored index maps onto itself.
// Influence-table view for one tile: the tile's fixed kx values in registers, the y and z tables
// staged in shared memory, all rounded once from the FP64 tables to FP32.  Triclinic boxes stage
// two more table rows (the k_y and k_z contributions) at my/mz + 2 (ny + nz) and + 3 (ny + nz).
struct KTab {
  float m1, A1;
  float m1b, m1c;    // triclinic: k_y and k_z contributions of kx
  const float* my;   // [ny] mhat_y
  const float* mz;   // [nz] mhat_z
  const float* Ay;   // [ny] A_y
  const float* Az;   // [nz] A_z
};

__host__ __device__ inline size_t ktab_smem_bytes(int ny, int nz) { return 4 * sizeof(float) * ((size_t)ny + nz); }

// Stage mhat and A for y and z into `sm` (4 (ny + nz) floats) and load kx's.  The caller
// synchronises before use.
__device__ __forceinline__ KTab stage_ktab(const SysDesc& d, int kx, float* sm) {
  const Geom& g = d.g;
  const int ntot = g.nx + g.ny + g.nz;
  const int nyz = g.ny + g.nz;
  const int rows = g.tric ? 4 : 2;
  for (int i = threadIdx.x; i < rows * nyz; i += kThreads) {
    const int r = i / nyz, j = i - r * nyz;
    sm[i] = (float)__ldcg(&d.ktab[r * ntot + g.nx + j]);
  }
  KTab t;
  t.m1 = (float)__ldcg(&d.ktab[kx]);
  t.A1 = (float)__ldcg(&d.ktab[ntot + kx]);
  t.m1b = g.tric ? (float)__ldcg(&d.ktab[2 * ntot + kx]) : 0.0f;
  t.m1c = g.tric ? (float)__ldcg(&d.ktab[3 * ntot + kx]) : 0.0f;
  t.my = sm;
  t.mz = sm + g.ny;
  t.Ay = sm + nyz;
  t.Az = sm + nyz + g.ny;
  return t;
}

// stage_ktab with the entries computed in place (ktab_entry, the same FP64 arithmetic as
// ktab_tile, so the same values), for a solve launch with no table phase before it.
__device__ __forceinline__ KTab stage_ktab_local(const SysDesc& d, int kx, float* sm) {
  const Geom& g = d.g;
  const int nyz = g.ny + g.nz;
  for (int j = threadIdx.x; j < nyz; j += kThreads) {
    double v[4];
    ktab_entry(d, g.nx + j, v);
    sm[j] = (float)v[0];
    sm[nyz + j] = (float)v[1];
    if (g.tric) {
      sm[2 * nyz + j] = (float)v[2];
      sm[3 * nyz + j] = (float)v[3];
    }
  }
  double vx[4];
  ktab_entry(d, kx, vx);
  KTab t;
  t.m1 = (float)vx[0];
  t.A1 = (float)vx[1];
  t.m1b = g.tric ? (float)vx[2] : 0.0f;
  t.m1c = g.tric ? (float)vx[3] : 0.0f;
  t.my = sm;
  t.mz = sm + g.ny;
  t.Ay = sm + nyz;
  t.Az = sm + nyz + g.ny;
  return t;
}

// Energy and virial terms of one k vector with weight w (1, or 2 for a stored element and its
// mirror): t = w eterm |Q|^2 2^32, v = 2 (fac + 1/|k|^2); [t, t (v k0 k0 - 1), t v k0 k1, t v k0 k2,
// t (v k1 k1 - 1), t v k1 k2, t (v k2 k2 - 1)], each rounded once to an integer.
__device__ __forceinline__ void add_ev_terms(long long* acc, float eterm, float q2, float inv_msq,
                                             float fac, float w, float k0, float k1, float k2) {
  const float wt = __fmul_rn(w, __fmul_rn(__fmul_rn(eterm, q2), (float)kEvScale));
  const float vt = __fmul_rn(2.0f, __fadd_rn(fac, inv_msq));
  const float tv = __fmul_rn(wt, vt);
  acc[0] += __float2ll_rn(wt);
  acc[1] += __float2ll_rn(__fmul_rn(wt, __fmaf_rn(__fmul_rn(vt, k0), k0, -1.0f)));
  acc[2] += __float2ll_rn(__fmul_rn(__fmul_rn(tv, k0), k1));
  acc[3] += __float2ll_rn(__fmul_rn(__fmul_rn(tv, k0), k2));
  acc[4] += __float2ll_rn(__fmul_rn(wt, __fmaf_rn(__fmul_rn(vt, k1), k1, -1.0f)));
  acc[5] += __float2ll_rn(__fmul_rn(__fmul_rn(tv, k1), k2));
  acc[6] += __float2ll_rn(__fmul_rn(wt, __fmaf_rn(__fmul_rn(vt, k2), k2, -1.0f)));
}

// Triclinic eterm of Miller indices (mx, my, mz) with k vector (k0, k1, k2) and per-axis product
// a = piv_inv A_x A_y A_z: a exp(cross) / |k|^2.
__device__ __forceinline__ float tric_eterm(const SysDesc& d, float a, float mx, float my, float mz,
                                            float k0, float k1, float k2, float& inv_msq) {
  inv_msq = __frcp_rn(__fmaf_rn(k2, k2, __fmaf_rn(k1, k1, __fmul_rn(k0, k0))));
  const float arg = __fmaf_rn(d.cross_f[2], __fmul_rn(my, mz),
                              __fmaf_rn(d.cross_f[1], __fmul_rn(mx, mz), __fmul_rn(d.cross_f[0], __fmul_rn(mx, my))));
  return __fmul_rn(__fmul_rn(a, expf(arg)), inv_msq);
}

__device__ __forceinline__ float signed_index(int k, int n) {
  return (float)(k < (n >> 1) + (n & 1) ? k : k - n);
}

// Triclinic solve of one stored element.  The x-mirror (kx >= 1) is the grid element
// (nx - kx, ny - ky, nz - kz) with its own Miller indices, as for orthorhombic boxes: m' = -m unless
// a component sits on an even-length Nyquist plane (or at 0), where m'_d = m_d.  When no component
// is on a Nyquist plane k' = -k, with the same eterm and virial products, so the element counts
// twice; otherwise the mirror's eterm and k' are evaluated separately.
__device__ __forceinline__ void solve_elem_tric(float2& q, int kx, int ky, int kz, const SysDesc& d,
                                                const KTab& kt, long long* acc) {
  const Geom& g = d.g;
  if (kx == 0 && ky == 0 && kz == 0) {
    q = make_float2(0.0f, 0.0f);
    return;
  }
  const int r2 = 2 * (g.ny + g.nz), r3 = 3 * (g.ny + g.nz);
  const float cy0 = kt.my[ky], cy1 = kt.my[r2 + ky], cy2 = kt.my[r3 + ky];
  const float cz0 = kt.mz[kz], cz1 = kt.mz[r2 + kz], cz2 = kt.mz[r3 + kz];
  const float k0 = __fadd_rn(__fadd_rn(kt.m1, cy0), cz0);
  const float k1 = __fadd_rn(__fadd_rn(kt.m1b, cy1), cz1);
  const float k2 = __fadd_rn(__fadd_rn(kt.m1c, cy2), cz2);
  const float mx = signed_index(kx, g.nx), my = signed_index(ky, g.ny), mz = signed_index(kz, g.nz);
  const float a = __fmul_rn(__fmul_rn(__fmul_rn(d.piv_inv_f, kt.A1), kt.Ay[ky]), kt.Az[kz]);
  float inv_msq;
  const float eterm = tric_eterm(d, a, mx, my, mz, k0, k1, k2, inv_msq);
  if (d.calc_ev) {
    const float q2 = __fmaf_rn(q.y, q.y, __fmul_rn(q.x, q.x));
    const bool nyq = (2 * kx == g.nx) || (2 * ky == g.ny) || (2 * kz == g.nz);
    add_ev_terms(acc, eterm, q2, inv_msq, d.fac_f, (kx >= 1 && !nyq) ? 2.0f : 1.0f, k0, k1, k2);
    if (kx >= 1 && nyq) {
      const float sx = (2 * kx == g.nx) ? 1.0f : -1.0f;
      const float sy = (ky == 0 || 2 * ky == g.ny) ? 1.0f : -1.0f;
      const float sz = (kz == 0 || 2 * kz == g.nz) ? 1.0f : -1.0f;
      const float j0 = __fadd_rn(__fadd_rn(sx * kt.m1, sy * cy0), sz * cz0);
      const float j1 = __fadd_rn(__fadd_rn(sx * kt.m1b, sy * cy1), sz * cz1);
      const float j2 = __fadd_rn(__fadd_rn(sx * kt.m1c, sy * cy2), sz * cz2);
      float inv_msq_m;
      const float eterm_m = tric_eterm(d, a, sx * mx, sy * my, sz * mz, j0, j1, j2, inv_msq_m);
      add_ev_terms(acc, eterm_m, q2, inv_msq_m, d.fac_f, 1.0f, j0, j1, j2);
    }
  }
  q.x = __fmul_rn(q.x, eterm);
  q.y = __fmul_rn(q.y, eterm);
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

// Triclinic solve of a span of stored elements held in shared memory: element (a, b), a = i div w,
// b = i - a w for i < count, at buf[a ld + b] with ky = y0 + b, kz = a (elements with b >= nb are
// padding), then the block's energy/virial flush.  Out of line so that the orthorhombic z and
// plane tiles keep their compact code (cold instruction fetch is part of a single evaluation's
// latency).  Every thread of the CTA calls it.
static __device__ __noinline__ void solve_span_tric(const SysDesc& d, float2* buf, int ld, int count, int w,
                                                    FastDiv wd, int nb, int kx, int y0, const KTab kt,
                                                    long long* red) {
  long long acc[7] = {0, 0, 0, 0, 0, 0, 0};
  for (int idx = threadIdx.x; idx < count; idx += kThreads) {
    const int a = fdiv(idx, wd), b = idx - a * w;
    if (b < nb) solve_elem_tric(buf[a * ld + b], kx, y0 + b, a, d, kt, acc);
  }
  if (d.calc_ev) flush_ev(d, acc, red);
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
// mode: 0 forward, 1 inverse, 2 forward + solve + inverse, 3 solve only (the staged scalar_sum,
// with the influence tables computed by the tile itself: no table phase before it).
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
  const bool solve = mode >= 2;
  if (mode < 3)
    for (int i = tid; i < L; i += kThreads) tw[i] = __ldg(&d.tw[plan.tw_off + i]);
  // the solve's influence tables load together with the columns (their own smem region)
  KTab kt;
  if (mode == 3) kt = stage_ktab_local(d, kx, ksm);
  else if (mode == 2) kt = stage_ktab(d, kx, ksm);
  for (int idx = tid; idx < L * tx; idx += kThreads) {
    const int e = fdiv(idx, txd), t = idx - e * tx;
    b0[e * ld + t] = t < nt ? __ldcg(&base[e * es + t]) : make_float2(0.0f, 0.0f);
  }
  __syncthreads();
  TileLane ln(tid, kThreads, tx);
  float2* res = b0;
  if (mode == 0 || mode == 2) res = fft_tile(b0, b1, plan, ld, 1, ln, tw, false);
  if (mode == 1) res = fft_tile(b0, b1, plan, ld, 1, ln, tw, true);
  if (solve) {
    if (g.tric) {
      solve_span_tric(d, res, ld, L * tx, tx, txd, nt, kx, y0, kt, red);
    } else {
      long long acc[7] = {0, 0, 0, 0, 0, 0, 0};
      for (int idx = tid; idx < L * tx; idx += kThreads) {
        const int e = fdiv(idx, txd), t = idx - e * tx;
        if (t < nt) solve_elem(res[e * ld + t], kx, y0 + t, e, d, kt, acc);
      }
      if (d.calc_ev) flush_ev(d, acc, red);
    }
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
         4 * sizeof(float) * ((size_t)ny + nz);
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
  if (g.tric) {
    solve_span_tric(d, r, LD, ny * nz, ny, nyd, ny, kx, 0, kt, red);
  } else {
    long long acc[7] = {0, 0, 0, 0, 0, 0, 0};
    for (int idx = tid; idx < ny * nz; idx += kThreads) {
      const int z = fdiv(idx, nyd), y = idx - z * ny;
      solve_elem(r[z * LD + y], kx, y, z, d, kt, acc);
    }
    if (d.calc_ev) flush_ev(d, acc, red);
  }
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
// Whole kx plane over a thread-block cluster of CS CTAs (orthorhombic boxes): y forward, z forward,
// solve with energy/virial, z inverse, y inverse in one tile, the two transposes between the y and
// z lines going through distributed shared memory instead of the global grid and two grid
// barriers.  Rank r of the cluster owns the z-lines [r nzl, (r+1) nzl) (y transforms, lines of ny
// elements, A[t (ny+1) + y]) and the y-columns [r nyl, (r+1) nyl) (z transforms and the solve,
// B[j (nz+1) + z]).  Every line goes through fft_tile and every element through solve_elem as in
// the pass and plane tiles, so the results are the same bits.  The CS CTAs of a cluster take the
// same planes in the same order (tile t = CS kx + rank, t = blockIdx.x + k gridDim.x with gridDim.x
// a multiple of CS), so each cluster barrier is reached by all of them.
// ---------------------------------------------------------------------------------------------
__host__ __device__ inline int cplane_lines(int n, int cs) { return (n + cs - 1) / cs; }
__host__ __device__ inline size_t cplane_smem_bytes(int ny, int nz, int cs) {
  const size_t A = (size_t)cplane_lines(nz, cs) * (ny + 1), B = (size_t)cplane_lines(ny, cs) * (nz + 1);
  return sizeof(float2) * ((size_t)ny + nz + 2 * A + 2 * B) + 32 * 7 * sizeof(long long) +
         4 * sizeof(float) * ((size_t)ny + nz);
}

constexpr int kClusterPlane = 4;   // CTAs per cluster of the cluster plane tiles

template <int CS>
__device__ __forceinline__ void cplane_tile(const SysDesc& d, int tile, float2* smem) {
  namespace cg = cooperative_groups;
  cg::cluster_group cl = cg::this_cluster();
  const Geom& g = d.g;
  const int ny = g.ny, nz = g.nz, kx = tile / CS, rank = tile - kx * CS;
  const int nzl = cplane_lines(nz, CS), nyl = cplane_lines(ny, CS);
  const int LDA = ny + 1, LDB = nz + 1;
  const int z0 = rank * nzl, y0 = rank * nyl;
  const int mz = min(nzl, nz - z0), my = min(nyl, ny - y0);   // lines this rank owns
  float2* twy = smem;
  float2* twz = twy + ny;
  float2* A0 = twz + nz;
  float2* A1 = A0 + (size_t)nzl * LDA;
  float2* B0 = A1 + (size_t)nzl * LDA;
  float2* B1 = B0 + (size_t)nyl * LDB;
  long long* red = (long long*)(B1 + (size_t)nyl * LDB);
  float* ksm = (float*)(red + 32 * 7);
  const int tid = threadIdx.x;
  float2* __restrict__ base = d.cgrid + cidx(g, kx, 0, 0);
  step_mark(d, 8);
  const KTab kt = stage_ktab(d, kx, ksm);
  for (int i = tid; i < ny; i += kThreads) twy[i] = __ldg(&d.tw[d.py.tw_off + i]);
  for (int i = tid; i < nz; i += kThreads) twz[i] = __ldg(&d.tw[d.pz.tw_off + i]);
  const FastDiv nyd = d.py.n_div;
  for (int idx = tid; idx < mz * ny; idx += kThreads) {       // my z-lines, contiguous in y
    const int t = fdiv(idx, nyd), y = idx - t * ny;
    A0[t * LDA + y] = __ldcg(&base[(size_t)(z0 + t) * ny + y]);
  }
  __syncthreads();
  step_mark(d, 9);
  float2* ar = fft_tile(A0, A1, d.py, 1, LDA, TileLane(tid, kThreads, nzl), twy, false);
  step_mark(d, 10);
  // transpose 1: element (z, y) to rank y / nyl, column y - owner nyl, position z
  const FastDiv nzld = make_fastdiv(nzl);
  for (int idx = tid; idx < nzl * ny; idx += kThreads) {
    const int y = fdiv(idx, nzld), t = idx - y * nzl;
    if (t < mz) {
      const int owner = y / nyl, j = y - owner * nyl;
      float2* dst = cl.map_shared_rank(B0 + (size_t)j * LDB + (z0 + t), owner);
      *dst = ar[t * LDA + y];
    }
  }
  cl.sync();
  step_mark(d, 11);
  float2* br = fft_tile(B0, B1, d.pz, 1, LDB, TileLane(tid, kThreads, nyl), twz, false);
  {
    long long acc[7] = {0, 0, 0, 0, 0, 0, 0};
    const FastDiv nzd = d.pz.n_div;
    for (int idx = tid; idx < my * nz; idx += kThreads) {
      const int j = fdiv(idx, nzd), z = idx - j * nz;
      solve_elem(br[j * LDB + z], kx, y0 + j, z, d, kt, acc);
    }
    if (d.calc_ev) flush_ev(d, acc, red);
  }
  __syncthreads();
  step_mark(d, 12);
  float2* bi = fft_tile(br, br == B0 ? B1 : B0, d.pz, 1, LDB, TileLane(tid, kThreads, nyl), twz, true);
  // transpose 2: element (y, z) back to rank z / nzl, line z - owner nzl, position y
  const FastDiv nyld = make_fastdiv(nyl);
  for (int idx = tid; idx < nyl * nz; idx += kThreads) {
    const int z = fdiv(idx, nyld), j = idx - z * nyl;
    if (j < my) {
      const int owner = z / nzl, t = z - owner * nzl;
      float2* dst = cl.map_shared_rank(A0 + (size_t)t * LDA + (y0 + j), owner);
      *dst = bi[j * LDB + z];
    }
  }
  cl.sync();
  step_mark(d, 13);
  float2* yr = fft_tile(A0, A1, d.py, 1, LDA, TileLane(tid, kThreads, nzl), twy, true);
  for (int idx = tid; idx < mz * ny; idx += kThreads) {
    const int t = fdiv(idx, nyd), y = idx - t * ny;
    __stcg(&base[(size_t)(z0 + t) * ny + y], yr[t * LDA + y]);
  }
  __syncthreads();
  step_mark(d, 14);
}


// ---------------------------------------------------------------------------------------------
// Fused path, phase 0: bin kThreads atoms by the row block of their stencil origin; sum q^2.
// A bin entry is the atom's record: stencil origin (ix, iy, iz as int bits) and atom index; the
// FP32 spreading weights q*thx[P], thy[P], thz[P] (the values the staged spread uses), padded to a
// multiple of 4 floats; then the fractional offsets ux, uy, uz and q for the gather.  Records are
// 16-byte aligned.
// ---------------------------------------------------------------------------------------------
__host__ __device__ constexpr int rec_floats(int order) { return ((4 + 3 * order + 3) & ~3) + 4; }

template <int P>
__device__ __forceinline__ void bin_tile_p(const SysDesc& d, int tile, int parity, long long* red) {
  constexpr int RF = rec_floats(P);
  constexpr int NW = RF - 8;                   // weight floats incl. padding
  const Geom& g = d.g;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int idx = tile * bin_tile_atoms(d) + threadIdx.x;
  const bool valid = (int)threadIdx.x < bin_tile_atoms(d) && idx < d.natom;
  const int nbins = d.nby * d.nbz;
  // walk the atoms in the previous evaluation's bin-sorted order when it is one for this count;
  // coordinates in host memory are read in index order (whole lines over the bus, not 16 bytes)
  const bool sorted = !d.xyzq_host && __ldcg(&d.bin_meta[kMetaPermNatom]) == d.natom;
  const int i = valid && sorted ? __ldcg(&d.perm[idx]) : idx;
  step_mark(d, 16);
  long long q2 = 0;
  unsigned int qbits = 0u;
  int b = -1, ix = 0, iy = 0, iz = 0;
  float ux = 0.0f, uy = 0.0f, uz = 0.0f, q = 0.0f;
  float w[NW];
#pragma unroll
  for (int k = 0; k < NW; k++) w[k] = 0.0f;
  if (valid) {
    const float4 a = __ldg(&d.xyzq[i]);
    frac_coords(g, a.x, a.y, a.z, ix, iy, iz, ux, uy, uz);
    bspline<P>(ux, w, nullptr);
#pragma unroll
    for (int k = 0; k < P; k++) w[k] = __fmul_rn(a.w, w[k]);
    bspline<P>(uy, w + P, nullptr);
    bspline<P>(uz, w + 2 * P, nullptr);
    q = a.w;
    b = iy / d.bry + d.nby * (iz / d.brz);
    q2 = q2_fixed(a.w);
    qbits = (unsigned int)__float_as_int(fabsf(a.w));
  }
  step_mark(d, 17);
  // slots: one counter update per group of lanes with the same bin
  const unsigned int grp = __match_any_sync(0xffffffffu, b);
  const int leader = __ffs(grp) - 1;
  int base = 0;
  if (valid && lane == leader) base = atomicAdd(&d.bin_count[parity * nbins + b], __popc(grp));
  base = __shfl_sync(0xffffffffu, base, leader);
  step_mark(d, 18);
  if (valid) {
    const int slot = base + __popc(grp & ((1u << lane) - 1u));
    float* rec;
    if (slot < d.bin_cap) {
      rec = d.bin_recs + ((size_t)b * d.bin_cap + slot) * RF;
    } else {
      const int o = atomicAdd(&d.bin_meta[kMetaOvf + parity], 1);
      rec = d.ovf_recs + (size_t)o * RF;
    }
    float4* r4 = (float4*)rec;
    __stcg(&r4[0], make_float4(__int_as_float(ix), __int_as_float(iy), __int_as_float(iz), __int_as_float(i)));
#pragma unroll
    for (int c = 0; c < NW / 4; c++)
      __stcg(&r4[1 + c], make_float4(w[4 * c], w[4 * c + 1], w[4 * c + 2], w[4 * c + 3]));
    __stcg(&r4[RF / 4 - 1], make_float4(ux, uy, uz, q));
  }
  step_mark(d, 19);
  // max |q| of the system (float bits of non-negative values order as integers) and sum q^2
  qbits = __reduce_max_sync(0xffffffffu, qbits);
  unsigned int* qs = (unsigned int*)(red + 16);
  if (lane == 0) qs[warp] = qbits;
  const long long sum = block_sum_ll(q2, red);
  if (threadIdx.x == 0) {
    unsigned int m = 0u;
#pragma unroll
    for (int k = 0; k < kThreads / 32; k++) m = max(m, qs[k]);
    if (m != 0u) atomicMax((unsigned int*)&d.bin_meta[kMetaQmax + parity], m);
    if (d.calc_self && sum != 0) atomicAdd((unsigned long long*)&d.acc[kAccQ2], (unsigned long long)sum);
  }
  step_mark(d, 20);
  __syncthreads();
  step_mark(d, 21);
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
// The work is split so that every lane does the same amount: a round takes up to spread_slots(P)
// candidates; step A tests each against the block and lists the ones that reach it (their
// weights) and one item per (atom, block row) it covers; step B gives each lane one item at a
// time, i.e. the P contributions of one stencil row.  The accumulator rows are P-1 points longer
// than the grid row, so a stencil row never wraps while spreading (the overhang is folded back
// when the rows are converted), and their stride is odd, so the rows of one atom fall in
// different banks.
// ---------------------------------------------------------------------------------------------
constexpr int kSpreadMaxBlock = 4;                  // row-block edge limit (bry, brz)
constexpr int kSpreadBookInts = 168;                // counters, candidate-bin offsets and bases
// candidates per round (listed-atom slots) and the items they can produce
__host__ __device__ constexpr int spread_slots(int order) { return order <= 4 ? 2 * kThreads : kThreads; }
__host__ __device__ constexpr int spread_item_cap(int order) {
  return spread_slots(order) * kSpreadMaxBlock * kSpreadMaxBlock;
}

__host__ __device__ inline int spread_row_stride(int nx, int order) { return (nx + order - 1) | 1; }
__host__ __device__ inline size_t align16(size_t b) { return (b + 15) & ~(size_t)15; }

// smem of the spread + x tile: 3 x 32-bit accumulators per point, twiddles, bookkeeping, then a
// work area that holds the listed atoms and items while spreading and the FFT buffers after.
__host__ __device__ inline size_t spread_x_smem_bytes(int nx, int rows, int order) {
  const size_t acc = align16((size_t)rows * spread_row_stride(nx, order) * 12);
  const size_t fft = (size_t)2 * nx * (rows + 1) * sizeof(float2);
  const size_t lists = (size_t)spread_slots(order) * 3 * order * 4 + (size_t)spread_item_cap(order) * sizeof(unsigned int);
  return acc + align16((size_t)nx * sizeof(float2)) + kSpreadBookInts * sizeof(int) + (fft > lists ? fft : lists);
}

// Exact int64 accumulation in shared memory with native 32-bit atomics, in one of three forms
// chosen per tile before its first contribution.  A point receives at most one contribution per
// candidate atom (the P stencil points of an axis are distinct), so with n candidates:
//  split2(k): v = lo + hi 2^k, lo = v mod 2^k in [0, 2^k), hi = v >> k (signed): two sums.  The
//    lo sum stays below n 2^k <= 2^32; the hi sum's magnitude below n (|v|max / 2^k + 1), where
//    |v| <= |q| 2^40 because every spline weight is at most 1.  k is the largest value with
//    n 2^k < 2^32, and the form is taken when the hi bound, from the system's max |q|, is below
//    2^31.
//  split3: v = p0 + p1 2^16 + p2 2^32 (p0, p1 in [0, 2^16), p2 = v >> 32): the p0 and p1 sums
//    cannot wrap for n <= 2^16; the p2 sum may wrap, harmlessly, since only its value modulo 2^32
//    enters the int64 result.
//  carry: lo (u32) + hi (s32), the wrap of lo detected from the returned old value (any n).
// Only the carry form waits for an atomic's result.  In every form the point's value is
// s0 + s1 2^16 + s2 2^sh (s2 sign-extended; sh = k for split2, 32 otherwise) modulo 2^64.
enum SpreadMode { kSplit2 = 0, kSplit3 = 1, kCarry = 2 };

template <int MODE>
__device__ __forceinline__ void add_fixed(unsigned int* s0, unsigned int* s1, int* s2, int idx, long long v,
                                          int k, unsigned int kmask) {
  if (MODE == kSplit2) {
    atomicAdd(&s0[idx], (unsigned int)(unsigned long long)v & kmask);
    atomicAdd(&s2[idx], (int)(v >> k));
  } else if (MODE == kSplit3) {
    const unsigned long long u = (unsigned long long)v;
    const unsigned int p0 = (unsigned int)(u & 0xffffull), p1 = (unsigned int)((u >> 16) & 0xffffull);
    const int p2 = (int)(v >> 32);
    atomicAdd(&s0[idx], p0);
    atomicAdd(&s1[idx], p1);
    if (p2 != 0) atomicAdd(&s2[idx], p2);
  } else {
    const unsigned int l = (unsigned int)(unsigned long long)v;
    const int h = (int)(v >> 32);
    const unsigned int old = atomicAdd(&s0[idx], l);
    const int carry = (old + l) < old ? 1 : 0;
    if (h + carry != 0) atomicAdd(&s2[idx], h + carry);
  }
}

// The listed atoms of a round: w[k][slot] over spread_slots(P) slots, k < 3P: q thx, thy, thz.
// An item is slot | b << 9 | c << 12 | (row * Lp + ix) << 15: stencil indices b (y) and c (z)
// and the accumulator offset of the stencil row's first point.
struct SpreadLists {
  float* w;
  unsigned int* items;
  int* counters;   // [0] listed atoms, [1] items
};

// Block rows [0, nr) covered by a stencil whose first row sits at r0 in [0, n) relative to the
// block (rows r0 .. r0+P-1, wrapped mod n), as a bitmask.
__device__ __forceinline__ unsigned int covered_rows(int r0, int P, int n, int nr) {
  unsigned int m = 0u;
  if (r0 < nr) {
    const int hi = min(nr, r0 + P);
    m = (1u << hi) - (1u << r0);
  }
  if (r0 + P > n) {
    const int hi = min(nr, r0 + P - n);
    m |= (1u << hi) - 1u;
  }
  return m;
}

// First candidate bin and number of candidate bins along one axis: the origin rows
// R0-P+1 .. R0+nr-1 (wrapped) cover the consecutive bins b0, b0+1, ..., own (mod nb), or every
// bin when the window spans the axis.  At most ceil((P-1)/br) + 2 <= 8 bins.
__device__ __forceinline__ void cand_axis(int P, int n, int br, int nb, int own, int R0, int nr, int& b0, int& cnt) {
  if (P - 1 + nr >= n) {
    b0 = 0;
    cnt = nb;
    return;
  }
  int r0 = (R0 - P + 1) % n;
  if (r0 < 0) r0 += n;
  b0 = r0 / br;
  cnt = own - b0;
  if (cnt < 0) cnt += nb;
  cnt += 1;
}

// Step A for PRE candidates per lane, their records already loaded (has[u] == false: none).
// The lane's listed atoms and items are reserved together: one warp scan and one pair of counter
// updates per warp.  Every lane of the warp calls it.
template <int P, int PRE>
__device__ __forceinline__ void spread_list_atoms(const SysDesc& d, const bool (&has)[PRE], const float4 (&head)[PRE],
                                                  const float4 (&w4)[PRE][(rec_floats(P) - 8) / 4], int Y0, int Z0,
                                                  int nry, int nrz, int Lp, const SpreadLists& sl) {
  constexpr int S = spread_slots(P);
  const Geom& g = d.g;
  const int lane = threadIdx.x & 31;
  unsigned int my[PRE], mz[PRE];
  int ry0[PRE], rz0[PRE], nrow[PRE];
  int v = 0;   // this lane's items (low 16 bits) and listed atoms (high bits)
#pragma unroll
  for (int u = 0; u < PRE; u++) {
    my[u] = mz[u] = 0u;
    ry0[u] = rz0[u] = 0;
    if (has[u]) {
      ry0[u] = __float_as_int(head[u].y) - Y0;
      if (ry0[u] < 0) ry0[u] += g.ny;
      rz0[u] = __float_as_int(head[u].z) - Z0;
      if (rz0[u] < 0) rz0[u] += g.nz;
      my[u] = covered_rows(ry0[u], P, g.ny, nry);
      mz[u] = covered_rows(rz0[u], P, g.nz, nrz);
    }
    nrow[u] = __popc(my[u]) * __popc(mz[u]);
    v += nrow[u] + (nrow[u] > 0 ? 1 << 16 : 0);
  }
  int incl = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int t = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += t;
  }
  const int wtot = __shfl_sync(0xffffffffu, incl, 31);
  if (wtot == 0) return;
  int sbase = 0, ibase = 0;
  if (lane == 0) {
    sbase = atomicAdd(&sl.counters[0], wtot >> 16);
    ibase = atomicAdd(&sl.counters[1], wtot & 0xffff);
  }
  sbase = __shfl_sync(0xffffffffu, sbase, 0);
  ibase = __shfl_sync(0xffffffffu, ibase, 0);
  const int excl = incl - v;
  unsigned int slot = (unsigned int)(sbase + (excl >> 16));
  unsigned int* it = sl.items + (ibase + (excl & 0xffff));
#pragma unroll
  for (int u = 0; u < PRE; u++) {
    if (nrow[u] == 0) continue;
    float* ws = sl.w + slot;
#pragma unroll
    for (int c = 0; c < 3 * P / 4; c++) {
      ws[(4 * c) * S] = w4[u][c].x;
      ws[(4 * c + 1) * S] = w4[u][c].y;
      ws[(4 * c + 2) * S] = w4[u][c].z;
      ws[(4 * c + 3) * S] = w4[u][c].w;
    }
    if ((3 * P) % 4 != 0) {   // P = 6: the last two weights
      ws[(3 * P - 2) * S] = w4[u][(3 * P) / 4].x;
      ws[(3 * P - 1) * S] = w4[u][(3 * P) / 4].y;
    }
    const unsigned int ix = (unsigned int)__float_as_int(head[u].x);
    unsigned int mzz = mz[u];
    while (mzz) {
      const int rz = __ffs(mzz) - 1;
      mzz &= mzz - 1;
      int c = rz - rz0[u];
      if (c < 0) c += g.nz;
      unsigned int myy = my[u];
      while (myy) {
        const int ry = __ffs(myy) - 1;
        myy &= myy - 1;
        int b = ry - ry0[u];
        if (b < 0) b += g.ny;
        *it++ = slot | (unsigned int)b << 9 | (unsigned int)c << 12 | ((unsigned int)(ry + nry * rz) * Lp + ix) << 15;
      }
    }
    slot++;
  }
}

// Step B: the P contributions of one (atom, stencil row) item per lane.
template <int P, int MODE>
__device__ __forceinline__ void spread_items(const SpreadLists& sl, int nitems, unsigned int* s0, unsigned int* s1,
                                             int* s2, int k2, unsigned int kmask) {
  constexpr int S = spread_slots(P);
  for (int j = threadIdx.x; j < nitems; j += kThreads) {
    const unsigned int it = sl.items[j];
    const float* ws = sl.w + (it & 511u);
    const float ty = ws[(P + ((it >> 9) & 7u)) * S];
    const float tz = ws[(2 * P + ((it >> 12) & 7u)) * S];
    const int base = (int)(it >> 15);
#pragma unroll
    for (int k = 0; k < P; k++)
      add_fixed<MODE>(s0, s1, s2, base + k, fixed_contrib(ws[k * S], ty, tz), k2, kmask);
  }
}

template <int P>
__device__ __forceinline__ void spread_x_tile(const SysDesc& d, int tile, int parity, char* smem_raw) {
  constexpr int RF = rec_floats(P);
  constexpr int NW4 = (RF - 8) / 4;          // float4s of spreading weights
  constexpr int S = spread_slots(P);
  constexpr int PRE = S / kThreads;            // candidates whose records a thread loads at once
  const Geom& g = d.g;
  const FftPlan1D& plan = d.px;
  const int L = g.nx, Lp = spread_row_stride(L, P);
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
  int* book = (int*)p;                         // [0..1] counters, [32..96] candidate-bin offsets,
  int* coff = book + 32;                       // [100..163] their first record (in records)
  int* cbase = book + 100;
  p += kSpreadBookInts * sizeof(int);
  SpreadLists sl;
  sl.w = (float*)p;
  sl.items = (unsigned int*)(sl.w + (size_t)3 * P * S);
  sl.counters = book;
  float2* b0 = (float2*)p;                     // FFT view of the work area (after spreading)
  float2* b1 = b0 + (size_t)L * ld;
  const int nbins = d.nby * d.nbz;
  step_mark(d, 0);
  // twiddles: loaded now, stored to smem once the spreading is done (L <= 2 kThreads)
  const float2 tw0 = tid < L ? __ldg(&d.tw[plan.tw_off + tid]) : make_float2(0.0f, 0.0f);
  const float2 tw1 = tid + kThreads < L ? __ldg(&d.tw[plan.tw_off + tid + kThreads]) : make_float2(0.0f, 0.0f);
  if (tid < 32) {
    // counts of the candidate bins (c = cy + ncy cz, at most 64), their exclusive prefix and the
    // index of their first record
    int b0y, ncy, b0z, ncz;
    cand_axis(P, g.ny, d.bry, d.nby, by, Y0, nry, b0y, ncy);
    cand_axis(P, g.nz, d.brz, d.nbz, bz, Z0, nrz, b0z, ncz);
    const int nc = ncy * ncz;
    int n01[2], inc[2];
#pragma unroll
    for (int h = 0; h < 2; h++) {
      const int c = tid + 32 * h;
      n01[h] = 0;
      if (c < nc) {
        int cby = b0y + c % ncy, cbz = b0z + c / ncy;
        if (cby >= d.nby) cby -= d.nby;
        if (cbz >= d.nbz) cbz -= d.nbz;
        const int b = cby + d.nby * cbz;
        n01[h] = min(__ldcg(&d.bin_count[parity * nbins + b]), d.bin_cap);
        cbase[c] = b * d.bin_cap;
      }
      inc[h] = n01[h];
    }
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
#pragma unroll
      for (int h = 0; h < 2; h++) {
        const int t = __shfl_up_sync(0xffffffffu, inc[h], o);
        if (tid >= o) inc[h] += t;
      }
    }
    const int tot0 = __shfl_sync(0xffffffffu, inc[0], 31);
    coff[tid] = inc[0] - n01[0];
    coff[tid + 32] = tot0 + inc[1] - n01[1];
    if (tid == 31) coff[64] = tot0 + inc[1];
    if (tid < 2) sl.counters[tid] = 0;
  }
  {
    // the three accumulator arrays are one 16-byte-aligned block of 3 rows*Lp words
    const int words = 3 * rows * Lp;
    uint4* z4 = (uint4*)s0;
    for (int i = tid; i < words / 4; i += kThreads) z4[i] = make_uint4(0u, 0u, 0u, 0u);
    for (int i = (words & ~3) + tid; i < words; i += kThreads) s0[i] = 0u;
  }
  const int novf = __ldcg(&d.bin_meta[kMetaOvf + parity]);
  const float qmax = __int_as_float(__ldcg(&d.bin_meta[kMetaQmax + parity]));
  __syncthreads();
  const int total = coff[64];
  step_mark(d, 1);
  const int ncand = total + novf;
  // accumulation form for this tile (see add_fixed)
  const int k2 = __clz(max(ncand, 1));          // largest k with ncand 2^k < 2^32
  const unsigned int kmask = (unsigned int)((1ull << k2) - 1ull);
  // hi-sum bound in FP32 (the 1.001 covers its rounding); NaN or inf qmax fails the test
  const float hib = (float)ncand * __fmaf_rn(qmax, ldexpf(1.001f, 40 - k2), 2.0f);
  const int mode = hib < 2147483648.0f ? kSplit2 : (ncand <= 65536 ? kSplit3 : kCarry);
  for (int base0 = 0; base0 < ncand; base0 += S) {
#pragma unroll 1
    for (int h0 = 0; h0 < S; h0 += PRE * kThreads) {
      bool has[PRE];
      float4 head[PRE];
      float4 w4[PRE][NW4];
#pragma unroll
      for (int u = 0; u < PRE; u++) {
        const int q = base0 + h0 + u * kThreads + tid;
        const float* rec = nullptr;
        if (q < total) {
          int c = 0;
          while (q >= coff[c + 1]) c++;
          rec = d.bin_recs + ((size_t)cbase[c] + (q - coff[c])) * RF;
        } else if (q < ncand) {
          rec = d.ovf_recs + (size_t)(q - total) * RF;
        }
        has[u] = rec != nullptr;
        if (has[u]) {
          const float4* r4 = (const float4*)rec;
          head[u] = __ldcg(r4);
#pragma unroll
          for (int c = 0; c < NW4; c++) w4[u][c] = __ldcg(r4 + 1 + c);
        } else {
          head[u] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
#pragma unroll
          for (int c = 0; c < NW4; c++) w4[u][c] = head[u];
        }
      }
      spread_list_atoms<P, PRE>(d, has, head, w4, Y0, Z0, nry, nrz, Lp, sl);
    }
    __syncthreads();
    if (base0 == 0) step_mark(d, 2);
    const int ni = sl.counters[1];
    if (mode == kSplit2) spread_items<P, kSplit2>(sl, ni, s0, s1, s2, k2, kmask);
    else if (mode == kSplit3) spread_items<P, kSplit3>(sl, ni, s0, s1, s2, k2, kmask);
    else spread_items<P, kCarry>(sl, ni, s0, s1, s2, k2, kmask);
    __syncthreads();
    if (tid < 2) sl.counters[tid] = 0;
    __syncthreads();
  }
  step_mark(d, 3);
  // the other parity's counters are cleared for the next launch by the system's first block
  if (tile == 0) {
    for (int j = tid; j < nbins; j += kThreads) d.bin_count[(1 - parity) * nbins + j] = 0;
    if (tid < 2) d.bin_meta[2 * tid + 1 - parity] = 0;   // overflow count, max |q|
  }
  const int sh = mode == kSplit2 ? k2 : 32;
  if (tid < L) tw[tid] = tw0;
  if (tid + kThreads < L) tw[tid + kThreads] = tw1;
  // rows: r = ry + nry*rz (r < nry*nrz valid); FFT line t = r.  Point e of a row also takes the
  // overhang at e + L (the stencil rows that ran past the row end).
  for (int idx = tid; idx < rows * L; idx += kThreads) {
    const int t = fdiv(idx, plan.n_div), e = idx - t * L;
    const int a = t * Lp + e;
    unsigned long long u = (unsigned long long)s0[a] + ((unsigned long long)s1[a] << 16) +
                           ((unsigned long long)(long long)s2[a] << sh);
    if (e < P - 1)
      u += (unsigned long long)s0[a + L] + ((unsigned long long)s1[a + L] << 16) +
           ((unsigned long long)(long long)s2[a + L] << sh);
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
// With a mirror (fused evaluations only: solve and self together) this evaluation's own record is
// also stored there, zeros for the terms not asked for.
__device__ __forceinline__ void finalize_system(const SysDesc& d, bool solve, bool self) {
  long long* acc = d.acc;
  double* ev = d.ev;
  double own[kEvCount];
  for (int c = 0; c < kEvCount; c++) own[c] = 0.0;
  if (solve && d.calc_ev) {
    double s[7];
    for (int c = 0; c < 7; c++) {
      s[c] = (double)acc[kAccE + c] / kEvScale;
      acc[kAccE + c] = 0;
    }
    const double h = 0.5 * kCcelec;
    own[kEvRecip] = h * s[0];
    double* vir = own + kEvVirial;
    vir[0] = -h * s[1]; vir[1] = -h * s[2]; vir[2] = -h * s[3];
    vir[3] = -h * s[2]; vir[4] = -h * s[4]; vir[5] = -h * s[5];
    vir[6] = -h * s[3]; vir[7] = -h * s[5]; vir[8] = -h * s[6];
    ev[kEvRecip] += own[kEvRecip];
    for (int c = 0; c < 9; c++) ev[kEvVirial + c] += vir[c];
  }
  if (self && d.calc_self) {
    const double q2 = (double)acc[kAccQ2] / kQ2Scale;
    acc[kAccQ2] = 0;
    own[kEvSelf] = d.self_coef * q2;
    ev[kEvSelf] += own[kEvSelf];
  }
  if (d.ev_mirror != nullptr && solve && self)
    for (int c = 0; c < kEvCount; c++) d.ev_mirror[c] = own[c];
}

// ---------------------------------------------------------------------------------------------
// Gather of one atom by LPA lanes (2, 4 or 8).  The P^2 stencil rows (b, c), r = b + P c, fall
// into 8 groups r mod 8; each group's rows are summed in order of r, then the 8 group sums are
// combined by the same pairwise tree whatever LPA is (groups g and g^4, then g^2, then g^1), the
// pairs on one lane added locally and the others by shuffles.  Every LPA therefore gives the same
// bits, so the staged and the fused gather agree however many lanes each gives an atom.
// F_d = q ccelec n_d r_d sum(...) (gradient convention, CudaPMERecip.cu:1234-1242).
template <int P>
struct GatherSplines {
  float thx[P], dthx[P], thy[P], dthy[P], thz[P], dthz[P];
  int xs[P];
};

// Where a gather reads the solved real grid: the global rgrid, or (GX) a window of rows in shared
// memory: row t = j + ry i holds grid row (y0 + j, z0 + i) wrapped, x fastest; every atom of the
// window's tile has its stencil origin in [y0, y0 + bry) x [z0, z0 + brz).
struct RowWin {
  const float* rows;
  int y0, z0, ry;
};

// Sum of the rows r = g, g+8, g+16, ... < P^2 (group g) for the three force components.
template <int P, bool GX = false>
__device__ __forceinline__ float3 gather_group(const SysDesc& d, const GatherSplines<P>& sp, int g, int iy, int iz,
                                               bool valid, const RowWin& w) {
  const Geom& gm = d.g;
  constexpr int RPG = (P * P + 7) / 8;
  float f1 = 0.0f, f2 = 0.0f, f3 = 0.0f;
#pragma unroll
  for (int rr = 0; rr < RPG; rr++) {
    const int r = g + 8 * rr;
    if (valid && r < P * P) {
      const int b = r % P, c = r / P;
      float wy = 0.0f, dwy = 0.0f, wz = 0.0f, dwz = 0.0f;
#pragma unroll
      for (int q = 0; q < P; q++) {
        if (q == b) { wy = sp.thy[q]; dwy = sp.dthy[q]; }
        if (q == c) { wz = sp.thz[q]; dwz = sp.dthz[q]; }
      }
      const float* row;
      if (GX) {
        row = w.rows + (size_t)gm.nx * ((iy - w.y0 + b) + w.ry * (iz - w.z0 + c));
      } else {
        const int y = wrap_add(iy, b, gm.ny), z = wrap_add(iz, c, gm.nz);
        row = d.rgrid + (size_t)gm.nx * (y + (size_t)gm.ny * z);
      }
      float s1 = 0.0f, s2 = 0.0f;
#pragma unroll
      for (int i = 0; i < P; i++) {
        const float v = row[sp.xs[i]];
        s1 = fmaf(sp.dthx[i], v, s1);
        s2 = fmaf(sp.thx[i], v, s2);
      }
      f1 = fmaf(s1, wy * wz, f1);
      f2 = fmaf(s2, dwy * wz, f2);
      f3 = fmaf(s2, wy * dwz, f3);
    }
  }
  return make_float3(f1, f2, f3);
}

__device__ __forceinline__ float3 add3(float3 a, float3 b) { return make_float3(a.x + b.x, a.y + b.y, a.z + b.z); }

template <int P, int KIND, int LPA, bool GX = false>
__device__ __forceinline__ void gather_core(const SysDesc& d, int atom, bool valid, int gl, int ix, int iy, int iz,
                                            float ux, float uy, float uz, float q,
                                            const RowWin& w = RowWin{nullptr, 0, 0, 0}) {
  static_assert(LPA == 2 || LPA == 4 || LPA == 8, "lanes per atom");
  const Geom& g = d.g;
  GatherSplines<P> sp;
  bspline<P>(ux, sp.thx, sp.dthx);
  bspline<P>(uy, sp.thy, sp.dthy);
  bspline<P>(uz, sp.thz, sp.dthz);
#pragma unroll
  for (int i = 0; i < P; i++) sp.xs[i] = wrap_add(ix, i, g.nx);
  // this lane's groups gl + LPA m, combined locally in the tree's order
  float3 f;
  if (LPA == 8) {
    f = gather_group<P, GX>(d, sp, gl, iy, iz, valid, w);
  } else if (LPA == 4) {
    f = add3(gather_group<P, GX>(d, sp, gl, iy, iz, valid, w), gather_group<P, GX>(d, sp, gl + 4, iy, iz, valid, w));
  } else {
    const float3 a = add3(gather_group<P, GX>(d, sp, gl, iy, iz, valid, w),
                          gather_group<P, GX>(d, sp, gl + 4, iy, iz, valid, w));
    const float3 b = add3(gather_group<P, GX>(d, sp, gl + 2, iy, iz, valid, w),
                          gather_group<P, GX>(d, sp, gl + 6, iy, iz, valid, w));
    f = add3(a, b);
  }
#pragma unroll
  for (int off = LPA / 2; off >= 1; off >>= 1) {
    f.x += __shfl_xor_sync(0xffffffffu, f.x, off);
    f.y += __shfl_xor_sync(0xffffffffu, f.y, off);
    f.z += __shfl_xor_sync(0xffffffffu, f.z, off);
  }
  if (valid && gl == 0) {
    const float qc = q * (float)kCcelec;
    float fx, fy, fz;
    if (!g.tric) {
      fx = qc * g.sx_hi * f.x;
      fy = qc * g.sy_hi * f.y;
      fz = qc * g.sz_hi * f.z;
    } else {   // F_j = q ccelec sum_d R[j][d] n_d f_d
      const float* S = g.shi;
      fx = __fmul_rn(qc, __fmaf_rn(S[2], f.z, __fmaf_rn(S[1], f.y, __fmul_rn(S[0], f.x))));
      fy = __fmul_rn(qc, __fmaf_rn(S[5], f.z, __fmaf_rn(S[4], f.y, __fmul_rn(S[3], f.x))));
      fz = __fmul_rn(qc, __fmaf_rn(S[8], f.z, __fmaf_rn(S[7], f.y, __fmul_rn(S[6], f.x))));
    }
    const size_t st = (size_t)d.stride;
    if (KIND == kForceF32Soa) {
      float* fo = (float*)d.force;
      fo[atom] = fx;
      fo[atom + st] = fy;
      fo[atom + 2 * st] = fz;
    } else if (KIND == kForceF32x3) {
      float* fo = (float*)d.force + 3 * (size_t)atom;
      fo[0] = fx; fo[1] = fy; fo[2] = fz;
    } else {
      unsigned long long* fo = (unsigned long long*)d.force;
      atomicAdd(&fo[atom], (unsigned long long)__float2ll_rn(__fmul_rn(fx, kFixedScale)));
      atomicAdd(&fo[atom + st], (unsigned long long)__float2ll_rn(__fmul_rn(fy, kFixedScale)));
      atomicAdd(&fo[atom + 2 * st], (unsigned long long)__float2ll_rn(__fmul_rn(fz, kFixedScale)));
    }
  }
}

// One atom's force from its coordinates (the staged gather).
template <int P, int KIND, int LPA>
__device__ __forceinline__ void gather_atom(const SysDesc& d, int atom, bool valid, int gl) {
  const Geom& g = d.g;
  const float4 a = valid ? __ldg(&d.xyzq[atom]) : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  int ix, iy, iz;
  float ux, uy, uz;
  frac_coords(g, a.x, a.y, a.z, ix, iy, iz, ux, uy, uz);
  gather_core<P, KIND, LPA>(d, atom, valid, gl, ix, iy, iz, ux, uy, uz, a.w);
}

template <int P, int KIND>
__device__ __forceinline__ void gather_tile(const SysDesc& d, int tile) {
  constexpr int LPA = gather_lanes(P), APP = kThreads / LPA;
  const int atom = tile * APP + threadIdx.x / LPA, gl = threadIdx.x % LPA;
  if (tile * APP + (threadIdx.x >> 5) * (32 / LPA) < d.natom)   // warp-uniform
    gather_atom<P, KIND, LPA>(d, atom, atom < d.natom, gl);
}

// Fused path: gather the atoms of one row-block bin (plus the overflow atoms whose origin lies in
// the block), kGatherAtoms at a time, so that the tile's stencil rows (about
// (4+P-1)^2 grid rows) stay in L1.  Atoms come from the bin's records (origin, fractional offsets
// and charge, so no coordinate reload), the next pass's records loading while the current ones are
// gathered.  The tile also writes its atoms into the system's bin-sorted atom order at the bin's
// offset; the next evaluation's binning walks the atoms in that order, so that the atoms of a warp
// share a few bins.  Overflow atoms follow all binned ones.
// Shared memory of a gather tile that runs its own inverse x pass: 64 bytes of reduction space,
// the x twiddles, and two FFT buffers of nx lines x (rows + 1, odd) for the (bry + P - 1) x
// (brz + P - 1) rows its atoms reach.
__host__ __device__ inline int gx_rows_count(int bry, int brz, int order) { return (bry + order - 1) * (brz + order - 1); }
__host__ __device__ inline int gx_ld(int rows) { return (rows + 1) | 1; }
__host__ __device__ inline size_t gx_smem_bytes(int nx, int bry, int brz, int order) {
  const int R = gx_rows_count(bry, brz, order);
  return 64 + (size_t)nx * 8 + 2 * (size_t)nx * gx_ld(R) * 8;
}

// The inverse x pass of the rows a gather tile reads (bin (y0 / bry, z0 / brz)): Hermitian
// rebuild, inverse FFT and real part of each row, the same lines with the same arithmetic as
// x_inv_tile (so the same bits), into real rows in shared memory (RowWin layout).  The rows of
// the halo are transformed again by the neighbouring bins' tiles: about (1 + (P-1)/bry)^2 times
// the x-inverse work, for one grid barrier and one pass over the real grid less.
template <int P>
__device__ __forceinline__ RowWin gx_rows(const SysDesc& d, int y0, int z0, char* smem_raw) {
  const Geom& g = d.g;
  const FftPlan1D& plan = d.px;
  const int L = g.nx, hx = g.hx, RY = d.bry + P - 1, R = gx_rows_count(d.bry, d.brz, P), ld = gx_ld(R);
  float2* tw = (float2*)(smem_raw + 64);
  float2* b0 = tw + L;
  float2* b1 = b0 + (size_t)L * ld;
  const int tid = threadIdx.x;
  for (int i = tid; i < L; i += kThreads) tw[i] = __ldg(&d.tw[plan.tw_off + i]);
  const FastDiv Rd = make_fastdiv(R), RYd = make_fastdiv(RY);
  for (int idx = tid; idx < hx * R; idx += kThreads) {
    const int k = fdiv(idx, Rd), t = idx - k * R;
    const int i = fdiv(t, RYd), j = t - i * RY;
    const int y = (y0 + j) % g.ny, z = (z0 + i) % g.nz;
    const float2 v = __ldcg(&d.cgrid[cidx(g, k, z, y)]);
    b0[k * ld + t] = v;
    if (k >= 1 && L - k >= hx) b0[(L - k) * ld + t] = make_float2(v.x, -v.y);
  }
  __syncthreads();
  TileLane ln(tid, kThreads, R);
  float2* res = fft_tile(b0, b1, plan, ld, 1, ln, tw, true);
  float* rows = (float*)(res == b0 ? b1 : b0);
  // the tile's own rows (its bin's row block) also go to the global solved grid, which therefore
  // holds the whole grid after the evaluation, as after the separate x-inverse phase
  const int ymax = min(d.bry, g.ny - y0), zmax = min(d.brz, g.nz - z0);
  for (int idx = tid; idx < L * R; idx += kThreads) {
    const int t = fdiv(idx, plan.n_div), e = idx - t * L;
    const float v = res[e * ld + t].x;
    rows[t * L + e] = v;
    const int i = fdiv(t, RYd), j = t - i * RY;
    if (j < ymax && i < zmax) __stcg(&d.rgrid[((size_t)(z0 + i) * g.ny + (y0 + j)) * L + e], v);
  }
  __syncthreads();
  return RowWin{rows, y0, z0, RY};
}

// Shared memory of the x-sorted order of a gather tile's atoms: 64 bytes of reduction space, a
// histogram of nx + 1 counts, the sorted slot indices of up to bin_cap atoms.
__host__ __device__ inline size_t gsort_smem_bytes(int nx, int bin_cap) {
  return 64 + sizeof(int) * ((size_t)nx + 1 + (size_t)bin_cap);
}

// Whether a system's gather tiles sort their atoms by x: only without the gather's own inverse x
// pass, where the sort's shared memory fits in what the launch takes (smem), and where bins are
// dense (at least 128 atoms per bin on average; measured: 216^3 with ~194 atoms per bin 2.6%
// faster per evaluation, 64^3 systems with ~94 atoms per bin 5-10% slower).  Only the throughput
// build of the fused kernel has the sorting gather; the latency build ignores the flag.
__host__ inline int gather_sorts(const SysDesc& d, size_t smem) {
  const int nb = d.nby * d.nbz;
  return (!d.gx && gsort_smem_bytes(d.g.nx, d.bin_cap) <= smem && nb > 0 && d.natom >= 128 * nb) ? 1 : 0;
}

// The slots 0..cnt-1 of a bin's records ordered by the atoms' stencil origin ix (counting sort in
// shared memory; equal origins in any order): the atoms that one warp gathers together then read
// the same few sectors of each grid row.  Returns the order array in shared memory.
template <int P>
__device__ __forceinline__ const int* gather_order_by_x(const SysDesc& d, const float* list, int cnt, char* smem_raw) {
  constexpr int RF = rec_floats(P);
  const int nx = d.g.nx, tid = threadIdx.x, lane = tid & 31;
  int* hist = (int*)(smem_raw + 64);
  int* order = hist + nx + 1;
  for (int i = tid; i <= nx; i += kThreads) hist[i] = 0;
  __syncthreads();
  for (int j = tid; j < cnt; j += kThreads) atomicAdd(&hist[__float_as_int(__ldcg(list + (size_t)j * RF)) + 1], 1);
  __syncthreads();
  if (tid < 32) {   // exclusive starts: hist[b] = atoms with origin < b
    const int per = (nx + 1 + 31) / 32, b0 = lane * per;
    int s = 0;
    for (int b = b0; b < min(b0 + per, nx + 1); b++) s += hist[b];
    int incl = s;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int t = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += t;
    }
    int run = incl - s;
    for (int b = b0; b < min(b0 + per, nx + 1); b++) {
      run += hist[b];
      hist[b] = run;
    }
  }
  __syncthreads();
  for (int j = tid; j < cnt; j += kThreads) {
    const int ix = __float_as_int(__ldcg(list + (size_t)j * RF));
    order[atomicAdd(&hist[ix], 1)] = j;
  }
  __syncthreads();
  return order;
}

template <int P, int KIND, int LPA, bool GX = false, bool SORT = false>
__device__ __forceinline__ void gather_bin_tile(const SysDesc& d, int tile, int parity, char* smem_raw) {
  constexpr int RF = rec_floats(P);
  const int nbins = d.nby * d.nbz;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  int* red = (int*)smem_raw;
  RowWin w{nullptr, 0, 0, 0};
  if (GX) w = gx_rows<P>(d, (tile % d.nby) * d.bry, (tile / d.nby) * d.brz, smem_raw);
  const int* counts = d.bin_count + parity * nbins;
  const int cnt = min(__ldcg(&counts[tile]), d.bin_cap);
  const float* list = d.bin_recs + (size_t)tile * d.bin_cap * RF;
  const int* order = SORT ? gather_order_by_x<P>(d, list, cnt, smem_raw) : nullptr;
  constexpr int APP = kThreads / LPA;         // atoms per pass
  const int gl = tid % LPA, slot = tid / LPA;
  step_mark(d, 24);
  // offset of this bin in the bin-sorted order, and the number of binned atoms
  int pre = 0, tot = 0;
  for (int b = tid; b < nbins; b += kThreads) {
    const int c = min(__ldcg(&counts[b]), d.bin_cap);
    tot += c;
    if (b < tile) pre += c;
  }
  float4 h = make_float4(0.0f, 0.0f, 0.0f, 0.0f), u = h;
  if (slot < cnt) {
    const int r = SORT ? order[slot] : slot;
    h = __ldcg((const float4*)(list + (size_t)r * RF));
    u = __ldcg((const float4*)(list + (size_t)r * RF + RF - 4));
  }
#pragma unroll
  for (int off = 16; off >= 1; off >>= 1) {
    pre += __shfl_xor_sync(0xffffffffu, pre, off);
    tot += __shfl_xor_sync(0xffffffffu, tot, off);
  }
  if (lane == 0) {
    red[warp] = pre;
    red[8 + warp] = tot;
  }
  __syncthreads();
  pre = 0;
  tot = 0;
#pragma unroll
  for (int w = 0; w < kThreads / 32; w++) {
    pre += red[w];
    tot += red[8 + w];
  }
  for (int j0 = 0; j0 < cnt; j0 += APP) {
    const int j = j0 + slot;
    const bool valid = j < cnt;
    // order 4: the next pass's records load while this one is gathered; orders 6 and 8 load them
    // at the top of their pass (the registers the prefetch holds cost the 80-register build more
    // spills than the latency hides: 216^3 order 6 1.253 against 1.275 ms)
    constexpr bool kPrefetch = P <= 4;
    float4 hn = make_float4(0.0f, 0.0f, 0.0f, 0.0f), un = hn;
    if (kPrefetch && j + APP < cnt) {
      const int r = SORT ? order[j + APP] : j + APP;
      hn = __ldcg((const float4*)(list + (size_t)r * RF));
      un = __ldcg((const float4*)(list + (size_t)r * RF + RF - 4));
    }
    if (!kPrefetch && j0 > 0) {
      h = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
      u = h;
      if (valid) {
        const int r = SORT ? order[j] : j;
        h = __ldcg((const float4*)(list + (size_t)r * RF));
        u = __ldcg((const float4*)(list + (size_t)r * RF + RF - 4));
      }
    }
    const int atom = __float_as_int(h.w);
    // warps whose atoms all lie beyond the bin's count skip the pass (the test is warp-uniform)
    if (j0 + (warp * 32) / LPA < cnt)
      gather_core<P, KIND, LPA, GX>(d, atom, valid, gl, __float_as_int(h.x), __float_as_int(h.y), __float_as_int(h.z),
                                    u.x, u.y, u.z, u.w, w);
    if (valid && gl == 0) d.perm[pre + j] = atom;
    if (kPrefetch) {
      h = hn;
      u = un;
    }
    if (j0 == 0) step_mark(d, 25);
  }
  step_mark(d, 26);
  const int novf = __ldcg(&d.bin_meta[kMetaOvf + parity]);
  for (int j0 = 0; j0 < novf; j0 += APP) {
    const int j = j0 + slot;
    bool mine = false;
    float4 hh = make_float4(0.0f, 0.0f, 0.0f, 0.0f), uu = hh;
    if (j < novf) {
      hh = __ldcg((const float4*)(d.ovf_recs + (size_t)j * RF));
      uu = __ldcg((const float4*)(d.ovf_recs + (size_t)j * RF + RF - 4));
      mine = (__float_as_int(hh.y) / d.bry + d.nby * (__float_as_int(hh.z) / d.brz)) == tile;
      if (tile == 0 && gl == 0) d.perm[tot + j] = __float_as_int(hh.w);
    }
    if (j0 + (warp * 32) / LPA < novf)
      gather_core<P, KIND, LPA, GX>(d, __float_as_int(hh.w), mine, gl, __float_as_int(hh.x), __float_as_int(hh.y),
                                    __float_as_int(hh.z), uu.x, uu.y, uu.z, uu.w, w);
  }
  // binned + overflow atoms are all natom atoms: the order is a permutation for this atom count
  if (tile == 0 && tid == 0) d.bin_meta[kMetaPermNatom] = d.natom;
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

template <int P, bool GX, bool SORT>
__device__ __forceinline__ void gather_bin_any(const SysDesc& d, int tile, int parity, char* smem) {
  switch (d.force_kind) {
    case kForceF32Soa: gather_bin_tile<P, kForceF32Soa, gather_lanes(P), GX, SORT>(d, tile, parity, smem); break;
    case kForceF32x3: gather_bin_tile<P, kForceF32x3, gather_lanes(P), GX, SORT>(d, tile, parity, smem); break;
    default: gather_bin_tile<P, kForceI64SoaAccum, gather_lanes(P), GX, SORT>(d, tile, parity, smem); break;
  }
}

template <bool GX, bool SORT = false>
__device__ __forceinline__ void gather_bin_order(const SysDesc& d, int tile, int parity, char* smem) {
  switch (d.order) {
    case 4: gather_bin_any<4, GX, SORT>(d, tile, parity, smem); break;
    case 6: gather_bin_any<6, GX, SORT>(d, tile, parity, smem); break;
    default: gather_bin_any<8, GX, SORT>(d, tile, parity, smem); break;
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

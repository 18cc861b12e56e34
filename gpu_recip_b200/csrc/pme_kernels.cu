// pme_kernels.cu -- sm_100a kernels of the smooth-PME reciprocal path.
//
// Stages (reference CudaPMERecip.cu):
//   spread ......... int64 fixed-point charge spreading (:479-580, :44-66)
//   x_r2c .......... fixed->float conversion fused into the x-direction real-to-complex FFT
//                    (replaces reduce_force :1908-1921 + the x part of cufftExecR2C :2421)
//   c2c (y, z) ..... complex line FFTs; the z pass can fuse forward FFT + influence-function
//                    solve with energy/virial + inverse FFT (:594-901)
//   x_c2r .......... x-direction complex-to-real FFT (x part of cufftExecC2R :2464)
//   gather ......... force interpolation (:1031-1245)
//   self_energy .... -kappa ccelec/sqrt(pi) sum q^2 (:1252-1275)
// Every energy/virial reduction is deterministic: per-CTA partials in FP64 summed in a fixed
// order by the last CTA to finish.
#include <cuda_runtime.h>
#include <stdint.h>

#include "pme_common.cuh"
#include "pme_fft.cuh"
#include "pme_internal.h"

namespace pme {

// ---------------------------------------------------------------------------------------------
// Deterministic grid-wide reduction of K doubles.  Returns true in thread 0 of the last CTA,
// with the grid total in `total`.
// ---------------------------------------------------------------------------------------------
template <int K>
__device__ __forceinline__ void warp_sum(double (&v)[K]) {
#pragma unroll
  for (int off = 16; off >= 1; off >>= 1)
#pragma unroll
    for (int c = 0; c < K; c++) v[c] += __shfl_down_sync(0xffffffffu, v[c], off);
}

template <int K>
__device__ bool grid_reduce(double (&v)[K], const ReduceScratch& rs, int site, double (&total)[K]) {
  __shared__ double red[32][K];
  __shared__ bool am_last;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  warp_sum<K>(v);
  if (lane == 0)
#pragma unroll
    for (int c = 0; c < K; c++) red[warp][c] = v[c];
  __syncthreads();
  if (warp == 0) {
    double x[K];
#pragma unroll
    for (int c = 0; c < K; c++) x[c] = lane < nw ? red[lane][c] : 0.0;
    warp_sum<K>(x);
    if (lane == 0) {
#pragma unroll
      for (int c = 0; c < K; c++) rs.partials[(size_t)blockIdx.x * 8 + c] = x[c];
      __threadfence();
      unsigned int t = atomicAdd(&rs.ticket[site], 1u);
      am_last = (t == gridDim.x - 1);
    }
  }
  __syncthreads();
  if (!am_last) return false;
  __threadfence();
  double s[K];
#pragma unroll
  for (int c = 0; c < K; c++) s[c] = 0.0;
  for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x)
#pragma unroll
    for (int c = 0; c < K; c++) s[c] += __ldcg(&rs.partials[(size_t)b * 8 + c]);
  warp_sum<K>(s);
  if (lane == 0)
#pragma unroll
    for (int c = 0; c < K; c++) red[warp][c] = s[c];
  __syncthreads();
  if (warp == 0) {
#pragma unroll
    for (int c = 0; c < K; c++) s[c] = lane < nw ? red[lane][c] : 0.0;
    warp_sum<K>(s);
    if (lane == 0) {
#pragma unroll
      for (int c = 0; c < K; c++) total[c] = s[c];
      rs.ticket[site] = 0u;
    }
  }
  return threadIdx.x == 0;
}

// ---------------------------------------------------------------------------------------------
// Spread: a warp takes 32 atoms; each lane evaluates one atom's fractional coordinate and
// weights (q folded into the x weights), then the warp walks the atoms and covers each atom's
// P^3 stencil points with its 32 lanes, adding fixed-point contributions with 64-bit integer
// reductions (order independent, hence an exact, deterministic grid).
// ---------------------------------------------------------------------------------------------
template <int P>
struct SplineAtom {
  int ix, iy, iz;
  float tx[P], ty[P], tz[P];
};

template <int P>
__global__ void __launch_bounds__(128) spread_kernel(const float4* __restrict__ xyzq, int n, Geom g,
                                                     unsigned long long* __restrict__ accum) {
  __shared__ SplineAtom<P> sh[4][32];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int base = (blockIdx.x * 4 + warp) * 32;
  if (base >= n) return;
  const int cnt = min(32, n - base);
  if (lane < cnt) {
    const float4 a = xyzq[base + lane];
    SplineAtom<P>& s = sh[warp][lane];
    float ux, uy, uz, th[P];
    frac_coord(a.x, g.rx, g.nx, s.ix, ux);
    frac_coord(a.y, g.ry, g.ny, s.iy, uy);
    frac_coord(a.z, g.rz, g.nz, s.iz, uz);
    bspline<P>(ux, th, nullptr);
#pragma unroll
    for (int i = 0; i < P; i++) s.tx[i] = __fmul_rn(a.w, th[i]);
    bspline<P>(uy, th, nullptr);
#pragma unroll
    for (int i = 0; i < P; i++) s.ty[i] = th[i];
    bspline<P>(uz, th, nullptr);
#pragma unroll
    for (int i = 0; i < P; i++) s.tz[i] = th[i];
  }
  __syncwarp();
  constexpr int P3 = P * P * P;
  for (int i = 0; i < cnt; i++) {
    const SplineAtom<P>& s = sh[warp][i];
    for (int q = lane; q < P3; q += 32) {
      const int a = q % P, b = (q / P) % P, c = q / (P * P);
      const int x = wrap_add(s.ix, a, g.nx);
      const int y = wrap_add(s.iy, b, g.ny);
      const int z = wrap_add(s.iz, c, g.nz);
      const long long v = fixed_contrib(s.tx[a], s.ty[b], s.tz[c]);
      atomicAdd(&accum[x + (size_t)g.nx * (y + (size_t)g.ny * z)], (unsigned long long)v);
    }
  }
}

// ---------------------------------------------------------------------------------------------
// x pass, forward: TX consecutive grid rows (row = y + ny z) per CTA; int64 -> FP32 on load;
// complex FFT of length nx with zero imaginary part; the nx/2+1 non-redundant outputs are
// written to the half-complex grid [z][y][kx].
// ---------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(256) x_r2c_kernel(const long long* __restrict__ accum,
                                                    float2* __restrict__ cgrid, Geom g,
                                                    FftPlan1D plan, const float2* __restrict__ twg,
                                                    int tx) {
  extern __shared__ float2 smem[];
  const int L = g.nx, ld = tx + 1;
  float2* tw = smem;
  float2* b0 = tw + L;
  float2* b1 = b0 + L * ld;
  const int nth = blockDim.x, tid = threadIdx.x;
  const int nrows = g.ny * g.nz, row0 = blockIdx.x * tx;
  for (int i = tid; i < L; i += nth) tw[i] = twg[plan.tw_off + i];
  for (int idx = tid; idx < L * tx; idx += nth) {
    const int t = idx / L, e = idx - t * L, row = row0 + t;
    float v = 0.0f;
    if (row < nrows) v = fixed_to_float(accum[(size_t)row * L + e]);
    b0[e * ld + t] = make_float2(v, 0.0f);
  }
  __syncthreads();
  TileLane ln(tid, nth, tx);
  float2* res = fft_tile(b0, b1, plan, ld, ln, tw, false);
  const int hx = g.hx;
  for (int idx = tid; idx < hx * tx; idx += nth) {
    const int t = idx / hx, k = idx - t * hx, row = row0 + t;
    if (row < nrows) cgrid[(size_t)row * hx + k] = res[k * ld + t];
  }
}

// ---------------------------------------------------------------------------------------------
// x pass, inverse: rebuild each row's full spectrum by Hermitian symmetry X[n-k] = conj X[k],
// inverse FFT, keep the real part (imaginary parts of X[0] and of the Nyquist term drop out, as
// in a library C2R).
// ---------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(256) x_c2r_kernel(const float2* __restrict__ cgrid,
                                                    float* __restrict__ rgrid, Geom g,
                                                    FftPlan1D plan, const float2* __restrict__ twg,
                                                    int tx) {
  extern __shared__ float2 smem[];
  const int L = g.nx, ld = tx + 1, hx = g.hx;
  float2* tw = smem;
  float2* b0 = tw + L;
  float2* b1 = b0 + L * ld;
  const int nth = blockDim.x, tid = threadIdx.x;
  const int nrows = g.ny * g.nz, row0 = blockIdx.x * tx;
  for (int i = tid; i < L; i += nth) tw[i] = twg[plan.tw_off + i];
  for (int idx = tid; idx < hx * tx; idx += nth) {
    const int t = idx / hx, k = idx - t * hx, row = row0 + t;
    float2 v = make_float2(0.0f, 0.0f);
    if (row < nrows) v = cgrid[(size_t)row * hx + k];
    b0[k * ld + t] = v;
    if (k >= 1 && L - k >= hx) b0[(L - k) * ld + t] = make_float2(v.x, -v.y);
  }
  __syncthreads();
  TileLane ln(tid, nth, tx);
  float2* res = fft_tile(b0, b1, plan, ld, ln, tw, true);
  for (int idx = tid; idx < L * tx; idx += nth) {
    const int t = idx / L, e = idx - t * L, row = row0 + t;
    if (row < nrows) rgrid[(size_t)row * L + e] = res[e * ld + t].x;
  }
}

// ---------------------------------------------------------------------------------------------
// Influence function on one element (CudaPMERecip.cu:671-691): m_d = k_d or k_d - n_d,
// mhat = r m, eterm = exp(-fac |mhat|^2) piv_inv b_x b_y b_z / |mhat|^2 (FP32).
// ---------------------------------------------------------------------------------------------
struct KTerm {
  float eterm, m1, m2, m3, msq;
};

__device__ __forceinline__ KTerm kterm(int kx, int ky, int kz, const Geom& g, const SolveParams& sp) {
  const int nfx = (g.nx >> 1) + (g.nx & 1), nfy = (g.ny >> 1) + (g.ny & 1),
            nfz = (g.nz >> 1) + (g.nz & 1);
  KTerm o;
  const int mx = kx < nfx ? kx : kx - g.nx;
  const int my = ky < nfy ? ky : ky - g.ny;
  const int mz = kz < nfz ? kz : kz - g.nz;
  o.m1 = g.rx * (float)mx;
  o.m2 = g.ry * (float)my;
  o.m3 = g.rz * (float)mz;
  o.msq = o.m1 * o.m1 + o.m2 * o.m2 + o.m3 * o.m3;
  o.eterm = expf(-sp.fac * o.msq) * sp.piv_inv * sp.bmx[kx] * sp.bmy[ky] * sp.bmz[kz] / o.msq;
  return o;
}

// Energy and virial terms of one k (CudaPMERecip.cu:694-742), accumulated in FP64:
// acc = [sum t, sum t (v mx mx - 1), t v mx my, t v mx mz, t (v my my - 1), t v my mz,
//        t (v mz mz - 1)], t = eterm |Q|^2, v = 2 (fac + 1/m^2).
__device__ __forceinline__ void ev_accum(double* acc, const KTerm& k, double q2, double fac) {
  const double t1 = (double)k.eterm * q2;
  const double vt = 2.0 * (fac + 1.0 / (double)k.msq);
  const double m1 = k.m1, m2 = k.m2, m3 = k.m3;
  acc[0] += t1;
  acc[1] += t1 * (vt * m1 * m1 - 1.0);
  acc[2] += t1 * vt * m1 * m2;
  acc[3] += t1 * vt * m1 * m3;
  acc[4] += t1 * (vt * m2 * m2 - 1.0);
  acc[5] += t1 * vt * m2 * m3;
  acc[6] += t1 * (vt * m3 * m3 - 1.0);
}

// Solve on a z-line tile (lines = consecutive kx at fixed ky, elements = kz).  Elements are
// assigned to threads in the same way as the tile loads, so that the staged solve kernel and
// the fused z kernel add the same terms in the same order.
__device__ __forceinline__ void solve_tile(float2* buf, int ld, int tx, int kx0, int ky,
                                           const Geom& g, const SolveParams& sp, double* acc) {
  const int L = g.nz, nth = blockDim.x;
  const double facd = (double)sp.fac;
  for (int idx = threadIdx.x; idx < L * tx; idx += nth) {
    const int e = idx / tx, t = idx - e * tx, kx = kx0 + t, kz = e;
    if (kx >= g.hx) continue;
    float2 q = buf[e * ld + t];
    if (kx == 0 && ky == 0 && kz == 0) {
      buf[e * ld + t] = make_float2(0.0f, 0.0f);
      continue;
    }
    const KTerm k = kterm(kx, ky, kz, g, sp);
    if (sp.calc_ev) {
      const double q2 = (double)q.x * (double)q.x + (double)q.y * (double)q.y;
      ev_accum(acc, k, q2, facd);
      if (kx >= 1) {
        const int kxs = g.nx - kx, kys = (g.ny - ky) % g.ny, kzs = (g.nz - kz) % g.nz;
        const KTerm ks = kterm(kxs, kys, kzs, g, sp);
        ev_accum(acc, ks, q2, facd);
      }
    }
    q.x *= k.eterm;
    q.y *= k.eterm;
    buf[e * ld + t] = q;
  }
}

// ---------------------------------------------------------------------------------------------
// Complex pass along y (axis 1) or z (axis 2).  A CTA takes TX consecutive kx at one outer index
// (z for the y pass, y for the z pass): each element row of the tile is TX contiguous complex
// values, so loads and stores are coalesced.  MODE 0 forward, 1 inverse, 2 forward + solve +
// inverse, 3 solve only.
// ---------------------------------------------------------------------------------------------
template <int MODE>
__global__ void __launch_bounds__(256) c2c_kernel(float2* __restrict__ cgrid, Geom g, int axis,
                                                  FftPlan1D plan, const float2* __restrict__ twg,
                                                  int tx, SolveParams sp, ReduceScratch rs,
                                                  int site) {
  extern __shared__ float2 smem[];
  const int L = (axis == 1) ? g.ny : g.nz, ld = tx + 1;
  float2* tw = smem;
  float2* b0 = tw + L;
  float2* b1 = b0 + L * ld;
  const int nth = blockDim.x, tid = threadIdx.x;
  const int tiles_x = (g.hx + tx - 1) / tx;
  const int tile_x = blockIdx.x % tiles_x, outer = blockIdx.x / tiles_x;
  const int kx0 = tile_x * tx;
  size_t estride, obase;
  if (axis == 1) {
    estride = (size_t)g.hx;
    obase = (size_t)outer * g.hx * g.ny;
  } else {
    estride = (size_t)g.hx * g.ny;
    obase = (size_t)outer * g.hx;
  }
  if (MODE != 3)
    for (int i = tid; i < L; i += nth) tw[i] = twg[plan.tw_off + i];
  for (int idx = tid; idx < L * tx; idx += nth) {
    const int e = idx / tx, t = idx - e * tx, kx = kx0 + t;
    float2 v = make_float2(0.0f, 0.0f);
    if (kx < g.hx) v = cgrid[obase + e * estride + kx];
    b0[e * ld + t] = v;
  }
  __syncthreads();
  TileLane ln(tid, nth, tx);
  float2* res = b0;
  if (MODE == 0 || MODE == 2) res = fft_tile(b0, b1, plan, ld, ln, tw, false);
  if (MODE == 1) res = fft_tile(b0, b1, plan, ld, ln, tw, true);
  if (MODE == 2 || MODE == 3) {
    double acc[7] = {0, 0, 0, 0, 0, 0, 0};
    solve_tile(res, ld, tx, kx0, outer, g, sp, acc);
    __syncthreads();
    if (sp.calc_ev) {
      double tot[7];
      if (grid_reduce<7>(acc, rs, site, tot)) {
        const double h = 0.5 * kCcelec;
        double* ev = sp.ev;
        ev[kEvRecip] += h * tot[0];
        double* vir = ev + kEvVirial;
        vir[0] -= h * tot[1]; vir[1] -= h * tot[2]; vir[2] -= h * tot[3];
        vir[3] -= h * tot[2]; vir[4] -= h * tot[4]; vir[5] -= h * tot[5];
        vir[6] -= h * tot[3]; vir[7] -= h * tot[5]; vir[8] -= h * tot[6];
      }
    }
    if (MODE == 2) {
      float2* other = (res == b0) ? b1 : b0;
      res = fft_tile(res, other, plan, ld, ln, tw, true);
    }
  }
  for (int idx = tid; idx < L * tx; idx += nth) {
    const int e = idx / tx, t = idx - e * tx, kx = kx0 + t;
    if (kx < g.hx) cgrid[obase + e * estride + kx] = res[e * ld + t];
  }
}

// ---------------------------------------------------------------------------------------------
// Gather: 8 lanes per atom; lane l takes stencil rows (b, c) = l, l+8, ... of the P^2 rows and
// sums the P points of each row; the 8 partial sums are combined with shuffles.  Output
// F_d = q ccelec r_d n_d sum(...) (gradient convention of CudaPMERecip.cu:1234-1242).
// ---------------------------------------------------------------------------------------------
template <int P, int KIND>
__global__ void __launch_bounds__(256) gather_kernel(const float4* __restrict__ xyzq, int n, Geom g,
                                                     const float* __restrict__ rgrid, int stride,
                                                     void* __restrict__ force) {
  const int gid = blockIdx.x * blockDim.x + threadIdx.x;
  const int atom = gid >> 3, gl = threadIdx.x & 7;
  const bool valid = atom < n;
  const float4 a = valid ? xyzq[atom] : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  int ix, iy, iz;
  float ux, uy, uz;
  frac_coord(a.x, g.rx, g.nx, ix, ux);
  frac_coord(a.y, g.ry, g.ny, iy, uy);
  frac_coord(a.z, g.rz, g.nz, iz, uz);
  float thx[P], dthx[P], thy[P], dthy[P], thz[P], dthz[P];
  bspline<P>(ux, thx, dthx);
  bspline<P>(uy, thy, dthy);
  bspline<P>(uz, thz, dthz);
  int xs[P];
#pragma unroll
  for (int i = 0; i < P; i++) xs[i] = wrap_add(ix, i, g.nx);
  float f1 = 0.0f, f2 = 0.0f, f3 = 0.0f;
  constexpr int RPL = (P * P + 7) / 8;
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
      const float* row = rgrid + (size_t)g.nx * (y + (size_t)g.ny * z);
      float s1 = 0.0f, s2 = 0.0f;
#pragma unroll
      for (int i = 0; i < P; i++) {
        const float v = __ldg(row + xs[i]);
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
    const float fx = qc * g.rx * f1 * (float)g.nx;
    const float fy = qc * g.ry * f2 * (float)g.ny;
    const float fz = qc * g.rz * f3 * (float)g.nz;
    if (KIND == kForceF32Soa) {
      float* f = (float*)force;
      f[atom] = fx;
      f[atom + (size_t)stride] = fy;
      f[atom + 2 * (size_t)stride] = fz;
    } else if (KIND == kForceF32x3) {
      float* f = (float*)force + 3 * (size_t)atom;
      f[0] = fx; f[1] = fy; f[2] = fz;
    } else {
      unsigned long long* f = (unsigned long long*)force;
      atomicAdd(&f[atom], (unsigned long long)__float2ll_rn(__fmul_rn(fx, kFixedScale)));
      atomicAdd(&f[atom + (size_t)stride], (unsigned long long)__float2ll_rn(__fmul_rn(fy, kFixedScale)));
      atomicAdd(&f[atom + 2 * (size_t)stride], (unsigned long long)__float2ll_rn(__fmul_rn(fz, kFixedScale)));
    }
  }
}

// ---------------------------------------------------------------------------------------------
// Self energy: sum q^2 in FP64, deterministic grid reduction, ev[self] += coef * sum.
// ---------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(256) self_energy_kernel(const float4* __restrict__ xyzq, int n,
                                                          double coef, double* ev,
                                                          ReduceScratch rs, int site) {
  double acc[1] = {0.0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double q = (double)xyzq[i].w;
    acc[0] += q * q;
  }
  double tot[1];
  if (grid_reduce<1>(acc, rs, site, tot)) ev[kEvSelf] += coef * tot[0];
}

__global__ void fixed_to_float_kernel(const long long* __restrict__ in, float* __restrict__ out,
                                      size_t count) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < count;
       i += (size_t)gridDim.x * blockDim.x)
    out[i] = fixed_to_float(in[i]);
}

// ---------------------------------------------------------------------------------------------
// Launchers
// ---------------------------------------------------------------------------------------------
static int num_threads_for(int L, int tx) {
  // about one radix-4 butterfly per thread and stage, in whole warps, 64..256 threads
  int want = (L / 4) * tx;
  int th = ((want + 31) / 32) * 32;
  return th < 64 ? 64 : (th > 256 ? 256 : th);
}

static size_t tile_smem(int L, int tx) {
  return sizeof(float2) * ((size_t)L + 2 * (size_t)L * (tx + 1));
}

size_t c2c_smem_bytes(int L, const PassTiling& t) { return tile_smem(L, t.tx); }

int c2c_num_blocks(const Geom& g, int axis, const PassTiling& t) {
  const int tiles_x = (g.hx + t.tx - 1) / t.tx;
  return tiles_x * (axis == 1 ? g.nz : g.ny);
}

cudaError_t launch_spread(const float4* xyzq, int n, const Geom& g, int order,
                          unsigned long long* accum, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  const int blocks = (n + 127) / 128;
  switch (order) {
    case 4: spread_kernel<4><<<blocks, 128, 0, s>>>(xyzq, n, g, accum); break;
    case 6: spread_kernel<6><<<blocks, 128, 0, s>>>(xyzq, n, g, accum); break;
    case 8: spread_kernel<8><<<blocks, 128, 0, s>>>(xyzq, n, g, accum); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

cudaError_t launch_x_r2c(const long long* accum, float2* cgrid, const Geom& g,
                         const FftPlan1D& px, const float2* tw, const PassTiling& t,
                         cudaStream_t s) {
  const int nrows = g.ny * g.nz;
  const int blocks = (nrows + t.tx - 1) / t.tx;
  const size_t smem = tile_smem(g.nx, t.tx);
  x_r2c_kernel<<<blocks, num_threads_for(g.nx, t.tx), smem, s>>>(accum, cgrid, g, px, tw, t.tx);
  return cudaGetLastError();
}

cudaError_t launch_x_c2r(const float2* cgrid, float* rgrid, const Geom& g, const FftPlan1D& px,
                         const float2* tw, const PassTiling& t, cudaStream_t s) {
  const int nrows = g.ny * g.nz;
  const int blocks = (nrows + t.tx - 1) / t.tx;
  const size_t smem = tile_smem(g.nx, t.tx);
  x_c2r_kernel<<<blocks, num_threads_for(g.nx, t.tx), smem, s>>>(cgrid, rgrid, g, px, tw, t.tx);
  return cudaGetLastError();
}

cudaError_t launch_c2c(float2* cgrid, const Geom& g, int axis, int mode, const FftPlan1D& plan,
                       const float2* tw, const PassTiling& t, const SolveParams* sp,
                       const ReduceScratch& rs, int rs_site, cudaStream_t s) {
  const int L = axis == 1 ? g.ny : g.nz;
  const int blocks = c2c_num_blocks(g, axis, t);
  const size_t smem = tile_smem(L, t.tx);
  const int th = num_threads_for(L, t.tx);
  SolveParams spv = {};
  if (sp) spv = *sp;
  if ((mode == 2 || mode == 3) && (axis != 2 || sp == nullptr)) return cudaErrorInvalidValue;
  if ((mode == 2 || mode == 3) && spv.calc_ev && blocks > rs.max_blocks) return cudaErrorInvalidValue;
  switch (mode) {
    case 0: c2c_kernel<0><<<blocks, th, smem, s>>>(cgrid, g, axis, plan, tw, t.tx, spv, rs, rs_site); break;
    case 1: c2c_kernel<1><<<blocks, th, smem, s>>>(cgrid, g, axis, plan, tw, t.tx, spv, rs, rs_site); break;
    case 2: c2c_kernel<2><<<blocks, th, smem, s>>>(cgrid, g, axis, plan, tw, t.tx, spv, rs, rs_site); break;
    case 3: c2c_kernel<3><<<blocks, th, smem, s>>>(cgrid, g, axis, plan, tw, t.tx, spv, rs, rs_site); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

template <int P>
static void launch_gather_p(const float4* xyzq, int n, const Geom& g, const float* rgrid, int kind,
                            int stride, void* force, cudaStream_t s) {
  const int blocks = (n + 31) / 32;
  switch (kind) {
    case kForceF32Soa: gather_kernel<P, kForceF32Soa><<<blocks, 256, 0, s>>>(xyzq, n, g, rgrid, stride, force); break;
    case kForceF32x3: gather_kernel<P, kForceF32x3><<<blocks, 256, 0, s>>>(xyzq, n, g, rgrid, stride, force); break;
    default: gather_kernel<P, kForceI64SoaAccum><<<blocks, 256, 0, s>>>(xyzq, n, g, rgrid, stride, force); break;
  }
}

cudaError_t launch_gather(const float4* xyzq, int n, const Geom& g, int order, const float* rgrid,
                          int kind, int stride, void* force, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  switch (order) {
    case 4: launch_gather_p<4>(xyzq, n, g, rgrid, kind, stride, force, s); break;
    case 6: launch_gather_p<6>(xyzq, n, g, rgrid, kind, stride, force, s); break;
    case 8: launch_gather_p<8>(xyzq, n, g, rgrid, kind, stride, force, s); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

cudaError_t launch_self_energy(const float4* xyzq, int n, double kappa, double* ev,
                               const ReduceScratch& rs, int rs_site, cudaStream_t s) {
  int blocks = (n + 255) / 256;
  if (blocks < 1) blocks = 1;
  if (blocks > rs.max_blocks) blocks = rs.max_blocks;
  const double coef = -kappa * kCcelec / sqrt(kPi);
  self_energy_kernel<<<blocks, 256, 0, s>>>(xyzq, n, coef, ev, rs, rs_site);
  return cudaGetLastError();
}

cudaError_t launch_fixed_to_float(const long long* accum, float* out, size_t count,
                                  cudaStream_t s) {
  int blocks = (int)((count + 255) / 256);
  if (blocks > 4096) blocks = 4096;
  if (blocks < 1) blocks = 1;
  fixed_to_float_kernel<<<blocks, 256, 0, s>>>(accum, out, count);
  return cudaGetLastError();
}

// Opt every dynamic-shared-memory kernel in to the full per-CTA budget once per device.
cudaError_t configure_kernels() {
  const int maxsm = 227 * 1024;
  cudaError_t e = cudaSuccess;
  e = cudaFuncSetAttribute(x_r2c_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, maxsm);
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(x_c2r_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, maxsm);
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(c2c_kernel<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, maxsm);
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(c2c_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, maxsm);
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(c2c_kernel<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, maxsm);
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(c2c_kernel<3>, cudaFuncAttributeMaxDynamicSharedMemorySize, maxsm);
  return e;
}

}  // namespace pme

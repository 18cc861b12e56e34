// pme_oracle.cpp -- TEST INFRASTRUCTURE ONLY. CPU oracle for the smooth-PME reciprocal path.
//
// This file is the checker, never the product: only tests/, __graft_entry__.smoke() and the
// cpu_baseline / --impl reference legs of bench.py load it.  The CUDA library in
// gpu_recip_b200/ never links or calls it.
//
// It restates, in double precision and from the mathematics, the algorithm of the reference
// operator CudaPMERecip (ap-hynninen/gpu_recip, CudaPMERecip.cu):
//   * fractional coordinates / stencil origin ......... CudaPMERecip.cu:502-529 (spread),
//                                                         :1056-1086 (gather)
//   * cardinal B-spline weights and derivatives ....... CudaPMERecip.cu:120-208, :2507-2537
//   * charge spreading, stencil i0..i0+p-1 mod n ...... CudaPMERecip.cu:479-580
//   * B-spline moduli (dftmod) ......................... CudaPMERecip.cu:2481-2505, :2543-2579
//   * forward R2C / inverse C2R 3-D DFT, unnormalised .. CudaPMERecip.cu:2421-2423, :2464-2466
//   * influence function, energy and virial ........... CudaPMERecip.cu:594-901, :1960-2040
//   * force gather (gradient, CHARMM sign) ............. CudaPMERecip.cu:1031-1245
//   * self energy ...................................... CudaPMERecip.cu:1252-1275, :2052-2061
//   * triclinic boxes (*_tric): an extension beyond the reference, which accepts only
//     orthorhombic recip (CudaPMERecip.cu:2042-2045); same algorithm with full-matrix maps
//
// Two spreading modes:
//   * orc_spread_f64:   FP64 weights, FP64 grid (the tolerance reference);
//   * orc_spread_fixed: the FP32 operation sequence of the GPU kernel (explicit fmaf, no
//     contraction: this file is compiled with -ffp-contract=off) rounded to int64 at 2^40,
//     so that the fixed-point charge grid can be compared bit for bit.
//
// The FFT is an independent recursive mixed-radix (any n; radix 2/3/5 fast, other primes by
// direct DFT) double-precision transform.  All entry points are extern "C", return 0 on
// success and a negative value on bad arguments.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#include <complex>
#include <thread>
#include <algorithm>
#include <atomic>

typedef std::complex<double> cplx;

static const double kPi = 3.14159265358979323846;
static const double kCcelec = 332.0716;   // CudaPMERecip.h:27 (CHARMM value)

static int hw_threads(int requested) {
  if (requested > 0) return requested;
  unsigned h = std::thread::hardware_concurrency();
  return h == 0 ? 1 : (int)h;
}

template <class F>
static void parallel_for(int nthreads, int count, F f) {
  nthreads = std::max(1, std::min(nthreads, count));
  if (nthreads == 1) { for (int i = 0; i < count; i++) f(i); return; }
  std::vector<std::thread> pool;
  for (int t = 0; t < nthreads; t++) {
    pool.emplace_back([=, &f]() {
      int lo = (int)((long long)count * t / nthreads);
      int hi = (int)((long long)count * (t + 1) / nthreads);
      for (int i = lo; i < hi; i++) f(i);
    });
  }
  for (auto& th : pool) th.join();
}

// ---------------------------------------------------------------------------------------------
// B-spline weights (CudaPMERecip.cu:2507-2537 fill_bspline_host; recursion of :181-208)
// theta[k], k = 0..p-1, are the weights of grid points i0+k; dtheta is d theta / du, built from
// the order p-1 weights before the last recursion step.
// ---------------------------------------------------------------------------------------------
static void bspline_f64(int p, double u, double* th, double* dth) {
  for (int i = 0; i < p; i++) th[i] = 0.0;
  th[0] = 1.0 - u;
  th[1] = u;
  for (int k = 3; k <= p; k++) {
    if (k == p && dth) {
      dth[0] = -th[0];
      for (int j = 1; j < p; j++) dth[j] = th[j - 1] - th[j];
    }
    double d = 1.0 / (double)(k - 1);
    th[k - 1] = d * u * th[k - 2];
    for (int j = 1; j <= k - 2; j++)
      th[k - j - 1] = d * ((u + j) * th[k - j - 2] + ((k - j) - u) * th[k - j - 1]);
    th[0] = d * (1.0 - u) * th[0];
  }
  if (p == 2 && dth) { dth[0] = -1.0; dth[1] = 1.0; }
}

extern "C" int orc_bspline(int p, double u, double* th, double* dth) {
  if (p < 2 || p > 16) return -1;
  bspline_f64(p, u, th, dth);
  return 0;
}

// FP32 mirror of the GPU spline evaluation: identical operation order, explicit fmaf.
static void bspline_f32(int p, float u, float* th) {
  for (int i = 0; i < p; i++) th[i] = 0.0f;
  th[0] = 1.0f - u;
  th[1] = u;
  for (int k = 3; k <= p; k++) {
    const float d = 1.0f / (float)(k - 1);
    th[k - 1] = (d * u) * th[k - 2];
    for (int j = 1; j <= k - 2; j++) {
      float a = u + (float)j;
      float b = (float)(k - j) - u;
      float hi = b * th[k - j - 1];
      th[k - j - 1] = d * std::fmaf(a, th[k - j - 2], hi);
    }
    th[0] = (d * (1.0f - u)) * th[0];
  }
}

// Fractional coordinate in grid units, FP32 mirror of the kernel: fr = n * frac(x*r + 1/2)
// (the function of CudaPMERecip.cu:510-529), evaluated as p + e with p = fl(x s_hi) and the
// product's rounding error recovered by fmaf, s_hi + s_lo = n r as a float-float pair.
// Non-finite or huge inputs map to i0 = 0, u = 0.
static inline void frac_f32(float x, float s_hi, float s_lo, int n, int* i0, float* u) {
  float p = x * s_hi;
  float e = std::fmaf(x, s_lo, std::fmaf(x, s_hi, -p));
  if (!(std::fabs(p) < 16777216.0f)) { p = 0.0f; e = 0.0f; }
  const float fl = std::floor(p);
  float f = p - fl;
  int i = (int)fl + (n >> 1);
  if (n & 1) f = f + 0.5f;
  float v = f + e;
  if (v >= 1.0f) { v = v - 1.0f; i += 1; }
  if (v < 0.0f) { v = v + 1.0f; i -= 1; }
  i %= n;
  if (i < 0) i += n;
  *i0 = i;
  *u = v;
}

static inline void split_scale(double r, int n, float* hi, float* lo) {
  const double s = r * (double)n;
  *hi = (float)s;
  *lo = (float)(s - (double)*hi);
}

static inline void frac_f64(double x, double r, int n, int* i0, double* u) {
  double w = x * r + 2.0;
  double fr = (double)n * (w - (std::floor(w + 0.5) - 0.5));
  if (!(fr >= 0.0 && fr < (double)n)) fr = 0.0;
  int i = (int)fr;
  if (i >= n) i = n - 1;
  *i0 = i;
  *u = fr - (double)i;
}

// ---------------------------------------------------------------------------------------------
// Triclinic boxes -- an extension: the reference accepts only orthorhombic recip
// (CudaPMERecip.cu:2042-2045).  recip9[3 j + d] = R[j][d] is the inverse of the matrix whose rows
// are the box vectors: fractional coordinate s_d = sum_j x_j R[j][d], k vector of Miller indices m
// k_j = sum_d R[j][d] m_d, cell volume V = 1 / |det R|.  Everything else is the orthorhombic
// algorithm with these two maps.
// ---------------------------------------------------------------------------------------------
static inline void frac_f64_tric(const double* x, const double* R, int d, int n, int* i0, double* u) {
  const double sd = x[0] * R[d] + x[1] * R[3 + d] + x[2] * R[6 + d];
  frac_f64(sd, 1.0, n, i0, u);
}

// FP32 mirror of the kernel's triclinic coordinate: float-float sum of the three products (each
// split exactly with fmaf, leading parts summed by two Knuth two-sums), then the tail of frac_f32.
static inline void frac_f32_tric(const float* x, const float* shi, const float* slo, int d, int n,
                                 int* i0, float* u) {
  const float p0 = x[0] * shi[d], p1 = x[1] * shi[3 + d], p2 = x[2] * shi[6 + d];
  const float e0 = std::fmaf(x[0], slo[d], std::fmaf(x[0], shi[d], -p0));
  const float e1 = std::fmaf(x[1], slo[3 + d], std::fmaf(x[1], shi[3 + d], -p1));
  const float e2 = std::fmaf(x[2], slo[6 + d], std::fmaf(x[2], shi[6 + d], -p2));
  const float s01 = p0 + p1;
  const float b01 = s01 - p0;
  const float t01 = (p0 - (s01 - b01)) + (p1 - b01);
  float p = s01 + p2;
  const float b2 = p - s01;
  const float t2 = (s01 - (p - b2)) + (p2 - b2);
  float e = ((e0 + e1) + e2) + (t01 + t2);
  if (!(std::fabs(p) < 16777216.0f)) { p = 0.0f; e = 0.0f; }
  const float fl = std::floor(p);
  float f = p - fl;
  int i = (int)fl + (n >> 1);
  if (n & 1) f = f + 0.5f;
  float v = f + e;
  if (v >= 1.0f) { v = v - 1.0f; i += 1; }
  if (v < 0.0f) { v = v + 1.0f; i -= 1; }
  i %= n;
  if (i < 0) i += n;
  *i0 = i;
  *u = v;
}

static inline double det3(const double* m) {
  return m[0] * (m[4] * m[8] - m[5] * m[7]) - m[1] * (m[3] * m[8] - m[5] * m[6]) +
         m[2] * (m[3] * m[7] - m[4] * m[6]);
}

// ---------------------------------------------------------------------------------------------
// Spreading (CudaPMERecip.cu:479-580).  Q[i0x+a, i0y+b, i0z+c] += q thx[a] thy[b] thz[c],
// indices mod n, grid layout x + nx*(y + ny*z).  Threads own z-planes so that each grid point
// is summed by one thread in atom order (deterministic for any thread count).
// ---------------------------------------------------------------------------------------------
// frac(i, ix, iy, iz, ux, uy, uz): stencil origins and offsets of atom i.
template <class Frac>
static int spread_f64_impl(const double* xyzq, int natom, int nx, int ny, int nz, int p, double* grid,
                           int nthreads, Frac frac) {
  if (natom < 0 || nx < p || ny < p || nz < p || p < 2 || p > 16) return -1;
  const size_t G = (size_t)nx * ny * nz;
  std::fill(grid, grid + G, 0.0);
  std::vector<int> iz0(natom);
  for (int i = 0; i < natom; i++) {
    int ix, iy;
    double ux, uy, uz;
    frac(i, &ix, &iy, &iz0[i], &ux, &uy, &uz);
  }
  parallel_for(hw_threads(nthreads), nz, [&](int z) {
    double thx[16], thy[16], thz[16];
    for (int i = 0; i < natom; i++) {
      int c = z - iz0[i];
      if (c < 0) c += nz;
      if (c >= p) continue;
      int ix, iy, izz;
      double ux, uy, uz;
      frac(i, &ix, &iy, &izz, &ux, &uy, &uz);
      bspline_f64(p, ux, thx, nullptr);
      bspline_f64(p, uy, thy, nullptr);
      bspline_f64(p, uz, thz, nullptr);
      const double q = xyzq[4 * i + 3];
      for (int b = 0; b < p; b++) {
        int y = iy + b; if (y >= ny) y -= ny;
        double qyz = q * thy[b] * thz[c];
        double* row = grid + (size_t)nx * (y + (size_t)ny * z);
        for (int a = 0; a < p; a++) {
          int x = ix + a; if (x >= nx) x -= nx;
          row[x] += qyz * thx[a];
        }
      }
    }
  });
  return 0;
}

extern "C" int orc_spread_f64(const double* xyzq, int natom, const double* recip3,
                              int nx, int ny, int nz, int p, double* grid, int nthreads) {
  return spread_f64_impl(xyzq, natom, nx, ny, nz, p, grid, nthreads,
                         [&](int i, int* ix, int* iy, int* iz, double* ux, double* uy, double* uz) {
                           frac_f64(xyzq[4 * i + 0], recip3[0], nx, ix, ux);
                           frac_f64(xyzq[4 * i + 1], recip3[1], ny, iy, uy);
                           frac_f64(xyzq[4 * i + 2], recip3[2], nz, iz, uz);
                         });
}

extern "C" int orc_spread_f64_tric(const double* xyzq, int natom, const double* recip9,
                                   int nx, int ny, int nz, int p, double* grid, int nthreads) {
  return spread_f64_impl(xyzq, natom, nx, ny, nz, p, grid, nthreads,
                         [&](int i, int* ix, int* iy, int* iz, double* ux, double* uy, double* uz) {
                           const double* x = xyzq + 4 * i;
                           frac_f64_tric(x, recip9, 0, nx, ix, ux);
                           frac_f64_tric(x, recip9, 1, ny, iy, uy);
                           frac_f64_tric(x, recip9, 2, nz, iz, uz);
                         });
}

// Fixed-point spreading, FP32 mirror: each contribution is ((q*thx[a])*thy[b])*thz[c] in FP32,
// scaled by 2^40 and rounded to nearest-even int64 (CudaPMERecip.cu:44-66 write_grid<long long>).
template <class Frac>
static int spread_fixed_impl(const float* xyzq, int natom, int nx, int ny, int nz, int p, int64_t* grid,
                             int nthreads, Frac frac) {
  if (natom < 0 || nx < p || ny < p || nz < p || p < 2 || p > 16) return -1;
  const size_t G = (size_t)nx * ny * nz;
  std::fill(grid, grid + G, (int64_t)0);
  std::vector<int> iz0(natom);
  for (int i = 0; i < natom; i++) {
    int ix, iy;
    float ux, uy, uz;
    frac(i, &ix, &iy, &iz0[i], &ux, &uy, &uz);
  }
  parallel_for(hw_threads(nthreads), nz, [&](int z) {
    float thx[16], thy[16], thz[16];
    for (int i = 0; i < natom; i++) {
      int c = z - iz0[i];
      if (c < 0) c += nz;
      if (c >= p) continue;
      int ix, iy, izz;
      float ux, uy, uz;
      frac(i, &ix, &iy, &izz, &ux, &uy, &uz);
      bspline_f32(p, ux, thx);
      bspline_f32(p, uy, thy);
      bspline_f32(p, uz, thz);
      const float q = xyzq[4 * i + 3];
      for (int b = 0; b < p; b++) {
        int y = iy + b; if (y >= ny) y -= ny;
        int64_t* row = grid + (size_t)nx * (y + (size_t)ny * z);
        for (int a = 0; a < p; a++) {
          int x = ix + a; if (x >= nx) x -= nx;
          float qx = q * thx[a];
          float v = (qx * thy[b]) * thz[c];
          row[x] += (int64_t)std::llrintf(v * 0x1p40f);
        }
      }
    }
  });
  return 0;
}

extern "C" int orc_spread_fixed(const float* xyzq, int natom, const double* recip3,
                                int nx, int ny, int nz, int p, int64_t* grid, int nthreads) {
  float shi[3], slo[3];
  split_scale(recip3[0], nx, &shi[0], &slo[0]);
  split_scale(recip3[1], ny, &shi[1], &slo[1]);
  split_scale(recip3[2], nz, &shi[2], &slo[2]);
  return spread_fixed_impl(xyzq, natom, nx, ny, nz, p, grid, nthreads,
                           [&](int i, int* ix, int* iy, int* iz, float* ux, float* uy, float* uz) {
                             frac_f32(xyzq[4 * i + 0], shi[0], slo[0], nx, ix, ux);
                             frac_f32(xyzq[4 * i + 1], shi[1], slo[1], ny, iy, uy);
                             frac_f32(xyzq[4 * i + 2], shi[2], slo[2], nz, iz, uz);
                           });
}

// Triclinic, FP32 mirror: S[j][d] = n_d R[j][d] split into float-float pairs.
extern "C" int orc_spread_fixed_tric(const float* xyzq, int natom, const double* recip9,
                                     int nx, int ny, int nz, int p, int64_t* grid, int nthreads) {
  const int n3[3] = {nx, ny, nz};
  float shi[9], slo[9];
  for (int j = 0; j < 3; j++)
    for (int d = 0; d < 3; d++) split_scale(recip9[3 * j + d], n3[d], &shi[3 * j + d], &slo[3 * j + d]);
  return spread_fixed_impl(xyzq, natom, nx, ny, nz, p, grid, nthreads,
                           [&](int i, int* ix, int* iy, int* iz, float* ux, float* uy, float* uz) {
                             const float* x = xyzq + 4 * i;
                             frac_f32_tric(x, shi, slo, 0, nx, ix, ux);
                             frac_f32_tric(x, shi, slo, 1, ny, iy, uy);
                             frac_f32_tric(x, shi, slo, 2, nz, iz, uz);
                           });
}

// int64 fixed point -> FP32 grid value: the integer rounded once to float (round to nearest),
// then scaled by 2^-40 (exact), i.e. one rounding of the exact quotient.
extern "C" int orc_fixed_to_float(const int64_t* in, size_t n, float* out) {
  for (size_t i = 0; i < n; i++) out[i] = (float)in[i] * 0x1p-40f;
  return 0;
}

// ---------------------------------------------------------------------------------------------
// FFT: recursive mixed radix, double precision, sign -1 forward / +1 inverse, unnormalised.
// ---------------------------------------------------------------------------------------------
struct Plan1D {
  int n;
  std::vector<cplx> w;   // w[k] = exp(-2 pi i k / n)
  explicit Plan1D(int n_) : n(n_), w(n_) {
    for (int k = 0; k < n; k++) {
      double a = -2.0 * kPi * (double)k / (double)n;
      w[k] = cplx(std::cos(a), std::sin(a));
    }
  }
};

static int smallest_factor(int n) {
  for (int f : {2, 3, 5}) if (n % f == 0) return f;
  for (int f = 7; f * f <= n; f += 2) if (n % f == 0) return f;
  return n;
}

// out[0..n) = DFT of in[0], in[s], in[2s], ...; tmp has n entries; tw_step maps to plan.w.
static void fft_rec(const cplx* in, cplx* out, int n, int s, int sign, const Plan1D& P,
                    int tw_step, cplx* tmp) {
  if (n == 1) { out[0] = in[0]; return; }
  const int f = smallest_factor(n);
  const int m = n / f;
  for (int q = 0; q < f; q++) fft_rec(in + (size_t)q * s, out + (size_t)q * m, m, s * f, sign, P,
                                      tw_step * f, tmp);
  // combine: X[k + j m] = sum_q W_n^{q (k + j m)} Y_q[k]
  for (int k = 0; k < m; k++) {
    for (int j = 0; j < f; j++) {
      cplx acc(0.0, 0.0);
      for (int q = 0; q < f; q++) {
        long long e = ((long long)q * (k + (long long)j * m)) % n;
        cplx tw = P.w[(size_t)(e * tw_step) % P.n];
        if (sign > 0) tw = std::conj(tw);
        acc += tw * out[(size_t)q * m + k];
      }
      tmp[k + (size_t)j * m] = acc;
    }
  }
  for (int i = 0; i < n; i++) out[i] = tmp[i];
}

static void fft_line(cplx* data, int n, int stride, int sign, const Plan1D& P) {
  std::vector<cplx> in(n), out(n), tmp(n);
  for (int i = 0; i < n; i++) in[i] = data[(size_t)i * stride];
  fft_rec(in.data(), out.data(), n, 1, sign, P, 1, tmp.data());
  for (int i = 0; i < n; i++) data[(size_t)i * stride] = out[i];
}

extern "C" int orc_fft1d(double* inout, int n, int sign) {
  if (n < 1) return -1;
  Plan1D P(n);
  fft_line(reinterpret_cast<cplx*>(inout), n, 1, sign, P);
  return 0;
}

// Naive O(n^2) DFT for testing.
extern "C" int orc_dft1d(const double* in, double* out, int n, int sign) {
  const cplx* a = reinterpret_cast<const cplx*>(in);
  cplx* b = reinterpret_cast<cplx*>(out);
  for (int k = 0; k < n; k++) {
    cplx acc(0, 0);
    for (int j = 0; j < n; j++) {
      double ang = sign * 2.0 * kPi * (double)(((long long)j * k) % n) / (double)n;
      acc += a[j] * cplx(std::cos(ang), std::sin(ang));
    }
    b[k] = acc;
  }
  return 0;
}

// Full complex 3-D transform in place on a [z][y][x] grid.
static void fft3d_c2c(cplx* g, int nx, int ny, int nz, int sign, int nthreads) {
  Plan1D Px(nx), Py(ny), Pz(nz);
  int T = hw_threads(nthreads);
  parallel_for(T, ny * nz, [&](int r) { fft_line(g + (size_t)r * nx, nx, 1, sign, Px); });
  parallel_for(T, nx * nz, [&](int r) {
    int x = r % nx, z = r / nx;
    fft_line(g + x + (size_t)nx * ny * z, ny, nx, sign, Py);
  });
  parallel_for(T, nx * ny, [&](int r) { fft_line(g + r, nz, nx * ny, sign, Pz); });
}

// Forward R2C: real [z][y][x] -> half complex [z][y][kx], kx = 0..nx/2 (interleaved re,im).
extern "C" int orc_fft3d_r2c(const double* in, int nx, int ny, int nz, double* out, int nthreads) {
  const size_t G = (size_t)nx * ny * nz;
  std::vector<cplx> g(G);
  for (size_t i = 0; i < G; i++) g[i] = cplx(in[i], 0.0);
  fft3d_c2c(g.data(), nx, ny, nz, -1, nthreads);
  const int hx = nx / 2 + 1;
  cplx* o = reinterpret_cast<cplx*>(out);
  for (size_t r = 0; r < (size_t)ny * nz; r++)
    for (int k = 0; k < hx; k++) o[r * hx + k] = g[r * nx + k];
  return 0;
}

// Inverse C2R: half complex [z][y][kx] -> real [z][y][x], unnormalised.  The full spectrum is
// rebuilt by Hermitian symmetry X[n-k] = conj(X[k]); imaginary parts that a real signal cannot
// have (kx = 0 and the Nyquist plane) drop out with the real part, as for a library C2R.
extern "C" int orc_fft3d_c2r(const double* in, int nx, int ny, int nz, double* out, int nthreads) {
  const size_t G = (size_t)nx * ny * nz;
  const int hx = nx / 2 + 1;
  const cplx* h = reinterpret_cast<const cplx*>(in);
  std::vector<cplx> g(G);
  for (int z = 0; z < nz; z++)
    for (int y = 0; y < ny; y++)
      for (int x = 0; x < nx; x++) {
        cplx v;
        if (x < hx) {
          v = h[((size_t)z * ny + y) * hx + x];
        } else {
          int xs = nx - x, ys = (ny - y) % ny, zs = (nz - z) % nz;
          v = std::conj(h[((size_t)zs * ny + ys) * hx + xs]);
        }
        g[((size_t)z * ny + y) * nx + x] = v;
      }
  fft3d_c2c(g.data(), nx, ny, nz, +1, nthreads);
  for (size_t i = 0; i < G; i++) out[i] = g[i].real();
  return 0;
}

// ---------------------------------------------------------------------------------------------
// B-spline moduli (CudaPMERecip.cu:2481-2505 dftmod, :2543-2579 calc_prefac).
// bmod[k] = 1 / |sum_{j=0}^{n-2} M[j] e^{2 pi i k j / n}|^2 with M[0] = 0, M[1..p] = theta(u=0),
// values below 1e-10 replaced by the mean of their neighbours before inversion.
// ---------------------------------------------------------------------------------------------
extern "C" int orc_bspline_moduli(int p, int n, double* bmod) {
  if (p < 2 || p > 16 || n < 2) return -1;
  std::vector<double> arr(std::max(n, p + 2), 0.0), th(p), dth(p);
  bspline_f64(p, 0.0, th.data(), dth.data());
  for (int i = 1; i <= p; i++) arr[i] = th[i - 1];
  std::vector<double> mod(n);
  for (int k = 0; k < n; k++) {
    double s1 = 0.0, s2 = 0.0;
    for (int j = 0; j < n - 1; j++) {
      double arg = 2.0 * kPi * (double)k * (double)j / (double)n;
      s1 += arr[j] * std::cos(arg);
      s2 += arr[j] * std::sin(arg);
    }
    mod[k] = s1 * s1 + s2 * s2;
  }
  for (int k = 0; k < n; k++)
    if (mod[k] < 1.0e-10) {
      double lo = mod[(k - 1 + n) % n], hi = mod[(k + 1) % n];
      mod[k] = 0.5 * (lo + hi);
    }
  for (int k = 0; k < n; k++) bmod[k] = 1.0 / mod[k];
  return 0;
}

// ---------------------------------------------------------------------------------------------
// Scalar sum (CudaPMERecip.cu:594-901, host :1928-2047), FP64.  Operates in place on the half
// complex grid.  Energy/virial: every stored k contributes eterm |Q|^2, and every stored k with
// kx >= 1 contributes again through its mirror -k (the reference's x-mirror doubling, which also
// doubles the Nyquist plane of an even nx).  energy = 1/2 ccelec sum, virial_ij =
// -1/2 ccelec sum eterm |Q|^2 (2 (pi^2/kappa^2 + 1/m^2) m_i m_j - delta_ij).
// ---------------------------------------------------------------------------------------------
// kvec(mx, my, mz, mh): k vector of the Miller indices; piv_inv = 1 / (pi V).
template <class KVec>
static int scalar_sum_impl(double* cgrid, int nx, int ny, int nz, int p, double piv_inv, double kappa,
                           int calc_ev, double* energy, double* vir9, int nthreads, KVec kvec) {
  if (nx < 2 || ny < 2 || nz < 2 || kappa <= 0.0) return -1;
  std::vector<double> bx(nx), by(ny), bz(nz);
  if (orc_bspline_moduli(p, nx, bx.data()) || orc_bspline_moduli(p, ny, by.data()) ||
      orc_bspline_moduli(p, nz, bz.data()))
    return -1;
  const int hx = nx / 2 + 1;
  const int nfx = nx / 2 + nx % 2, nfy = ny / 2 + ny % 2, nfz = nz / 2 + nz % 2;
  const double fac = kPi * kPi / (kappa * kappa);
  cplx* g = reinterpret_cast<cplx*>(cgrid);
  int T = hw_threads(nthreads);
  std::vector<double> part((size_t)nz * 7, 0.0);
  auto eterm_of = [&](int kx, int ky, int kz, double* mh) {
    int mx = kx < nfx ? kx : kx - nx;
    int my = ky < nfy ? ky : ky - ny;
    int mz = kz < nfz ? kz : kz - nz;
    kvec(mx, my, mz, mh);
    double msq = mh[0] * mh[0] + mh[1] * mh[1] + mh[2] * mh[2];
    return std::exp(-fac * msq) * piv_inv * bx[kx] * by[ky] * bz[kz] / msq;
  };
  auto accum = [&](double* acc, double eterm, double q2, const double* mh) {
    double msq = mh[0] * mh[0] + mh[1] * mh[1] + mh[2] * mh[2];
    double t1 = eterm * q2;
    double vt = 2.0 * (fac + 1.0 / msq);
    acc[0] += t1;
    acc[1] += t1 * (vt * mh[0] * mh[0] - 1.0);
    acc[2] += t1 * vt * mh[0] * mh[1];
    acc[3] += t1 * vt * mh[0] * mh[2];
    acc[4] += t1 * (vt * mh[1] * mh[1] - 1.0);
    acc[5] += t1 * vt * mh[1] * mh[2];
    acc[6] += t1 * (vt * mh[2] * mh[2] - 1.0);
  };
  parallel_for(T, nz, [&](int kz) {
    double* acc = &part[(size_t)kz * 7];
    for (int ky = 0; ky < ny; ky++)
      for (int kx = 0; kx < hx; kx++) {
        cplx& q = g[((size_t)kz * ny + ky) * hx + kx];
        if (kx == 0 && ky == 0 && kz == 0) { q = 0.0; continue; }
        double mh[3];
        double e = eterm_of(kx, ky, kz, mh);
        if (calc_ev) {
          double q2 = std::norm(q);
          accum(acc, e, q2, mh);
          if (kx >= 1) {
            int kxs = nx - kx, kys = (ny - ky) % ny, kzs = (nz - kz) % nz;
            double mhs[3];
            double es = eterm_of(kxs, kys, kzs, mhs);
            accum(acc, es, q2, mhs);
          }
        }
        q *= e;
      }
  });
  if (calc_ev) {
    double s[7] = {0, 0, 0, 0, 0, 0, 0};
    for (int kz = 0; kz < nz; kz++)
      for (int c = 0; c < 7; c++) s[c] += part[(size_t)kz * 7 + c];
    const double h = 0.5 * kCcelec;
    if (energy) *energy = h * s[0];
    if (vir9) {
      vir9[0] = -h * s[1]; vir9[1] = -h * s[2]; vir9[2] = -h * s[3];
      vir9[3] = -h * s[2]; vir9[4] = -h * s[4]; vir9[5] = -h * s[5];
      vir9[6] = -h * s[3]; vir9[7] = -h * s[5]; vir9[8] = -h * s[6];
    }
  }
  return 0;
}

extern "C" int orc_scalar_sum(double* cgrid, int nx, int ny, int nz, int p, const double* recip3,
                              double kappa, int calc_ev, double* energy, double* vir9,
                              int nthreads) {
  const double piv_inv = recip3[0] * recip3[1] * recip3[2] / kPi;
  return scalar_sum_impl(cgrid, nx, ny, nz, p, piv_inv, kappa, calc_ev, energy, vir9, nthreads,
                         [&](int mx, int my, int mz, double* mh) {
                           mh[0] = recip3[0] * mx; mh[1] = recip3[1] * my; mh[2] = recip3[2] * mz;
                         });
}

// Triclinic: k_j = sum_d R[j][d] m_d; the x-mirror is the grid element (nx-kx, ny-ky, nz-kz) with
// its own Miller indices, as in the orthorhombic sum.
extern "C" int orc_scalar_sum_tric(double* cgrid, int nx, int ny, int nz, int p, const double* recip9,
                                   double kappa, int calc_ev, double* energy, double* vir9,
                                   int nthreads) {
  const double piv_inv = std::fabs(det3(recip9)) / kPi;
  const double* R = recip9;
  return scalar_sum_impl(cgrid, nx, ny, nz, p, piv_inv, kappa, calc_ev, energy, vir9, nthreads,
                         [&](int mx, int my, int mz, double* mh) {
                           for (int j = 0; j < 3; j++) mh[j] = R[3 * j] * mx + R[3 * j + 1] * my + R[3 * j + 2] * mz;
                         });
}

// ---------------------------------------------------------------------------------------------
// Gather (CudaPMERecip.cu:1031-1245).  F_d = q ccelec r_d n_d sum (dtheta_d theta theta) Phi,
// i.e. +dE/dx (gradient; CHARMM convention).  Output AoS force[3*i + d].
// ---------------------------------------------------------------------------------------------
// frac(i, ...) as for spreading; out(i, qc, f1, f2, f3) writes atom i's force from the three
// grid-unit gradient sums.
template <class Frac, class Out>
static int gather_impl(const double* xyzq, int natom, const double* grid, int nx, int ny, int nz, int p,
                       int nthreads, Frac frac, Out out) {
  if (natom < 0 || p < 2 || p > 16) return -1;
  parallel_for(hw_threads(nthreads), natom, [&](int i) {
    double thx[16], thy[16], thz[16], dx[16], dy[16], dz[16];
    int ix, iy, iz;
    double ux, uy, uz;
    frac(i, &ix, &iy, &iz, &ux, &uy, &uz);
    bspline_f64(p, ux, thx, dx);
    bspline_f64(p, uy, thy, dy);
    bspline_f64(p, uz, thz, dz);
    double f1 = 0, f2 = 0, f3 = 0;
    for (int c = 0; c < p; c++) {
      int z = iz + c; if (z >= nz) z -= nz;
      for (int b = 0; b < p; b++) {
        int y = iy + b; if (y >= ny) y -= ny;
        const double* row = grid + (size_t)nx * (y + (size_t)ny * z);
        for (int a = 0; a < p; a++) {
          int x = ix + a; if (x >= nx) x -= nx;
          double v = row[x];
          f1 += dx[a] * thy[b] * thz[c] * v;
          f2 += thx[a] * dy[b] * thz[c] * v;
          f3 += thx[a] * thy[b] * dz[c] * v;
        }
      }
    }
    out(i, xyzq[4 * i + 3] * kCcelec, f1, f2, f3);
  });
  return 0;
}

extern "C" int orc_gather(const double* xyzq, int natom, const double* grid, const double* recip3,
                          int nx, int ny, int nz, int p, double* force, int nthreads) {
  return gather_impl(
      xyzq, natom, grid, nx, ny, nz, p, nthreads,
      [&](int i, int* ix, int* iy, int* iz, double* ux, double* uy, double* uz) {
        frac_f64(xyzq[4 * i + 0], recip3[0], nx, ix, ux);
        frac_f64(xyzq[4 * i + 1], recip3[1], ny, iy, uy);
        frac_f64(xyzq[4 * i + 2], recip3[2], nz, iz, uz);
      },
      [&](int i, double qc, double f1, double f2, double f3) {
        force[3 * i + 0] = qc * recip3[0] * nx * f1;
        force[3 * i + 1] = qc * recip3[1] * ny * f2;
        force[3 * i + 2] = qc * recip3[2] * nz * f3;
      });
}

// Triclinic: F_j = q ccelec sum_d R[j][d] n_d f_d (the chain rule through s_d = sum_j x_j R[j][d]).
extern "C" int orc_gather_tric(const double* xyzq, int natom, const double* grid, const double* recip9,
                               int nx, int ny, int nz, int p, double* force, int nthreads) {
  const double* R = recip9;
  return gather_impl(
      xyzq, natom, grid, nx, ny, nz, p, nthreads,
      [&](int i, int* ix, int* iy, int* iz, double* ux, double* uy, double* uz) {
        const double* x = xyzq + 4 * i;
        frac_f64_tric(x, R, 0, nx, ix, ux);
        frac_f64_tric(x, R, 1, ny, iy, uy);
        frac_f64_tric(x, R, 2, nz, iz, uz);
      },
      [&](int i, double qc, double f1, double f2, double f3) {
        const double g0 = nx * f1, g1 = ny * f2, g2 = nz * f3;
        for (int j = 0; j < 3; j++)
          force[3 * i + j] = qc * (R[3 * j] * g0 + R[3 * j + 1] * g1 + R[3 * j + 2] * g2);
      });
}

// Self energy (CudaPMERecip.cu:1252-1275): -kappa ccelec / sqrt(pi) * sum q^2.
extern "C" double orc_self_energy(const double* xyzq, int natom, double kappa) {
  double s = 0.0;
  for (int i = 0; i < natom; i++) s += xyzq[4 * i + 3] * xyzq[4 * i + 3];
  return -s * kappa * kCcelec / std::sqrt(kPi);
}

// ---------------------------------------------------------------------------------------------
// Whole evaluation in FP64: spread -> R2C -> scalar sum (energy, virial) -> C2R -> gather, plus
// self energy.  force is AoS (3*natom).  Work buffers are allocated per call.
// ---------------------------------------------------------------------------------------------
extern "C" int orc_eval(const double* xyzq, int natom, const double* recip3, int nx, int ny,
                        int nz, int p, double kappa, double* force, double* e_recip,
                        double* e_self, double* vir9, int nthreads) {
  const size_t G = (size_t)nx * ny * nz;
  const size_t H = (size_t)(nx / 2 + 1) * ny * nz;
  std::vector<double> grid(G), cg(2 * H);
  int rc = orc_spread_f64(xyzq, natom, recip3, nx, ny, nz, p, grid.data(), nthreads);
  if (rc) return rc;
  orc_fft3d_r2c(grid.data(), nx, ny, nz, cg.data(), nthreads);
  double e = 0.0, v[9] = {0};
  rc = orc_scalar_sum(cg.data(), nx, ny, nz, p, recip3, kappa, 1, &e, v, nthreads);
  if (rc) return rc;
  orc_fft3d_c2r(cg.data(), nx, ny, nz, grid.data(), nthreads);
  rc = orc_gather(xyzq, natom, grid.data(), recip3, nx, ny, nz, p, force, nthreads);
  if (rc) return rc;
  if (e_recip) *e_recip = e;
  if (vir9) for (int i = 0; i < 9; i++) vir9[i] = v[i];
  if (e_self) *e_self = orc_self_energy(xyzq, natom, kappa);
  return 0;
}

// Whole triclinic evaluation in FP64 (recip9 as for orc_spread_f64_tric).
extern "C" int orc_eval_tric(const double* xyzq, int natom, const double* recip9, int nx, int ny,
                             int nz, int p, double kappa, double* force, double* e_recip,
                             double* e_self, double* vir9, int nthreads) {
  const size_t G = (size_t)nx * ny * nz;
  const size_t H = (size_t)(nx / 2 + 1) * ny * nz;
  std::vector<double> grid(G), cg(2 * H);
  int rc = orc_spread_f64_tric(xyzq, natom, recip9, nx, ny, nz, p, grid.data(), nthreads);
  if (rc) return rc;
  orc_fft3d_r2c(grid.data(), nx, ny, nz, cg.data(), nthreads);
  double e = 0.0, v[9] = {0};
  rc = orc_scalar_sum_tric(cg.data(), nx, ny, nz, p, recip9, kappa, 1, &e, v, nthreads);
  if (rc) return rc;
  orc_fft3d_c2r(cg.data(), nx, ny, nz, grid.data(), nthreads);
  rc = orc_gather_tric(xyzq, natom, grid.data(), recip9, nx, ny, nz, p, force, nthreads);
  if (rc) return rc;
  if (e_recip) *e_recip = e;
  if (vir9) for (int i = 0; i < 9; i++) vir9[i] = v[i];
  if (e_self) *e_self = orc_self_energy(xyzq, natom, kappa);
  return 0;
}

// ---------------------------------------------------------------------------------------------
// Direct-space nonbonded terms (CudaPMEDirectForce, CudaDirectForceKernels.cu), FP64, for the
// models the reference's test runs: VDW_VSH (shifted Lennard-Jones, :175-195) and EWALD real-space
// electrostatics (:353-391).  Per pair, with r the minimum-image distance:
//   U_vdw  = c12/12 (r^-12 + 2 r^6 roff^-18 - 3 roff^-12) - c6/6 (r^-6 + r^6 roff^-12 - 2 roff^-6)
//   r dU_vdw/dr as the reference writes it: c6 (r^-6 - r^6 roff^-12) - c12 (r^-12 + r^6 roff^-18)
//     (the sign of its roff^-18 term differs from the derivative of U_vdw; kept, it changes forces
//     by ~1e-6 kcal/mol/A at roff = 9 A)
//   U_elec = qq (erfc(kappa r) + s - 1) / r,  r dU_elec/dr = -qq 2/sqrt(pi) kappa exp(-kappa^2 r^2)
//     - U_elec, qq = ccelec q_i q_j, s = 1 for ordinary pairs, e14fac for 1-4 pairs, 0 for excluded
//     pairs (the Ewald exclusion correction -qq erf(kappa r)/r)
//   gradient on i: (r dU/dr) / r^2 * (x_i - x_j); virial_ab -= (r dU/dr) / r^2 dx_a dx_b (the sign
//     of the reference's virial tensor, gpu_direct.cu:67-70, as for the reciprocal virial).
// c6/c12 of types (a, b): 6 vdwparam[2 k] and 12 vdwparam[2 k + 1], k = A (A + 1) / 2 + B,
// A = max, B = min (CudaDirectForce_util.h:265-278; the factors 6 and 12 are applied to the
// caller's table when it is set, CudaPMEDirectForce.cu:381-387).
// ---------------------------------------------------------------------------------------------
struct DirectPair {
  double f_over_r2, u_vdw, u_elec;
};

static DirectPair direct_pair(double r2, double qq, double c6, double c12, double kappa, double roff,
                              double s_elec, bool vdw) {
  const double r = std::sqrt(r2), rinv = 1.0 / r, rinv2 = rinv * rinv;
  DirectPair p{0.0, 0.0, 0.0};
  double fr = 0.0;
  if (vdw) {
    const double r6 = r2 * r2 * r2, rinv6 = rinv2 * rinv2 * rinv2, rinv12 = rinv6 * rinv6;
    const double ro6 = std::pow(roff, -6.0), ro12 = ro6 * ro6, ro18 = ro12 * ro6;
    p.u_vdw = c12 / 12.0 * (rinv12 + 2.0 * r6 * ro18 - 3.0 * ro12) - c6 / 6.0 * (rinv6 + r6 * ro12 - 2.0 * ro6);
    fr += c6 * (rinv6 - r6 * ro12) - c12 * (rinv12 + r6 * ro18);
  }
  const double e = qq * (std::erfc(kappa * r) + s_elec - 1.0) * rinv;
  p.u_elec = e;
  fr += -qq * 2.0 / std::sqrt(kPi) * kappa * std::exp(-kappa * kappa * r2) - e;
  p.f_over_r2 = fr * rinv2;
  return p;
}

static inline void vdw_c6c12(const double* vdwparam, const int* vdwtype, int i, int j, double* c6, double* c12) {
  const int a = std::max(vdwtype[i], vdwtype[j]), b = std::min(vdwtype[i], vdwtype[j]);
  const long k = (long)a * (a + 1) / 2 + b;
  *c6 = 6.0 * vdwparam[2 * k];
  *c12 = 12.0 * vdwparam[2 * k + 1];
}

// All pairs within roff (minimum image in the orthorhombic box box3; roff <= min(box)/2), less the
// excluded pairs excl_idx[excl_ptr[i] .. excl_ptr[i+1]) (0-based, symmetric).  force: AoS
// (3*natom), overwritten with the gradient; energies and the virial of the pair sum.
extern "C" int orc_direct_force(const double* xyzq, int natom, const double* box3, double kappa, double roff,
                                const double* vdwparam, const int* vdwtype, const int* excl_ptr,
                                const int* excl_idx, double* force, double* e_vdw, double* e_elec,
                                double* vir9, int nthreads) {
  if (natom < 0 || !(roff > 0.0) || 2.0 * roff > std::min(box3[0], std::min(box3[1], box3[2]))) return -1;
  int nc[3];
  for (int d = 0; d < 3; d++) nc[d] = std::max(1, (int)std::floor(box3[d] / roff));
  const int ncell = nc[0] * nc[1] * nc[2];
  std::vector<int> head(ncell, -1), next(natom, -1), cell(natom);
  auto wrap = [](double x, double L) { return x - L * std::floor(x / L); };
  for (int i = natom - 1; i >= 0; i--) {
    int c3[3];
    for (int d = 0; d < 3; d++) {
      c3[d] = (int)(wrap(xyzq[4 * i + d], box3[d]) / box3[d] * nc[d]);
      c3[d] = std::min(std::max(c3[d], 0), nc[d] - 1);
    }
    cell[i] = (c3[2] * nc[1] + c3[1]) * nc[0] + c3[0];
    next[i] = head[cell[i]];
    head[cell[i]] = i;
  }
  const double roff2 = roff * roff;
  const int T = hw_threads(nthreads);
  std::vector<double> part((size_t)T * 11, 0.0);
  std::atomic<int> nexti(0);
  std::vector<std::thread> th;
  for (int t = 0; t < T; t++) th.emplace_back([&, t]() {
    double* acc = &part[(size_t)t * 11];
    std::vector<char> mark(natom, 0);
    for (int i = nexti++; i < natom; i = nexti++) {
      for (int k = excl_ptr[i]; k < excl_ptr[i + 1]; k++) mark[excl_idx[k]] = 1;
      const int ci = cell[i];
      const int c3[3] = {ci % nc[0], (ci / nc[0]) % nc[1], ci / (nc[0] * nc[1])};
      int lo[3], cnt[3];
      for (int d = 0; d < 3; d++) {
        if (nc[d] >= 3) { lo[d] = -1; cnt[d] = 3; } else { lo[d] = 0; cnt[d] = nc[d]; }
      }
      double fx = 0, fy = 0, fz = 0;
      for (int oz = 0; oz < cnt[2]; oz++)
        for (int oy = 0; oy < cnt[1]; oy++)
          for (int ox = 0; ox < cnt[0]; ox++) {
            const int z = nc[2] >= 3 ? (c3[2] + lo[2] + oz + nc[2]) % nc[2] : oz;
            const int y = nc[1] >= 3 ? (c3[1] + lo[1] + oy + nc[1]) % nc[1] : oy;
            const int x = nc[0] >= 3 ? (c3[0] + lo[0] + ox + nc[0]) % nc[0] : ox;
            for (int j = head[(z * nc[1] + y) * nc[0] + x]; j >= 0; j = next[j]) {
              if (j == i || mark[j]) continue;
              double dx[3];
              for (int d = 0; d < 3; d++) {
                dx[d] = xyzq[4 * i + d] - xyzq[4 * j + d];
                dx[d] -= box3[d] * std::nearbyint(dx[d] / box3[d]);
              }
              const double r2 = dx[0] * dx[0] + dx[1] * dx[1] + dx[2] * dx[2];
              if (!(r2 < roff2)) continue;
              double c6, c12;
              vdw_c6c12(vdwparam, vdwtype, i, j, &c6, &c12);
              const DirectPair p = direct_pair(r2, kCcelec * xyzq[4 * i + 3] * xyzq[4 * j + 3], c6, c12, kappa,
                                               roff, 1.0, true);
              fx += p.f_over_r2 * dx[0];
              fy += p.f_over_r2 * dx[1];
              fz += p.f_over_r2 * dx[2];
              acc[0] += 0.5 * p.u_vdw;
              acc[1] += 0.5 * p.u_elec;
              for (int a = 0; a < 3; a++)
                for (int b = 0; b < 3; b++) acc[2 + 3 * a + b] -= 0.5 * p.f_over_r2 * dx[a] * dx[b];
            }
          }
      force[3 * i + 0] = fx;
      force[3 * i + 1] = fy;
      force[3 * i + 2] = fz;
      for (int k = excl_ptr[i]; k < excl_ptr[i + 1]; k++) mark[excl_idx[k]] = 0;
    }
  });
  for (auto& x : th) x.join();
  double s[11] = {0};
  for (int t = 0; t < T; t++)
    for (int c = 0; c < 11; c++) s[c] += part[(size_t)t * 11 + c];
  if (e_vdw) *e_vdw = s[0];
  if (e_elec) *e_elec = s[1];
  if (vir9) for (int c = 0; c < 9; c++) vir9[c] = s[2 + c];
  return 0;
}

// The 1-4 lists (CudaDirectForceKernels.cu:504-640): in14 (i, j, ishift) triples get the 1-4 vdW
// parameters and electrostatics scaled as erfc + e14fac - 1; ex14 triples the exclusion correction
// (e14fac 0); no cutoff test, the VSH shift uses roff.  ishift encodes the periodic image of j: shift_d = (digit_d - 1) box_d with
// ishift = dx + 3 dy + 9 dz digits (gpu_utils.h:312-320).  force (AoS) is ADDED to.
extern "C" int orc_direct_14(const double* xyzq, const double* box3, double kappa, double roff, double e14fac,
                             const double* vdwparam14, const int* vdwtype, const int* in14, int nin14,
                             const int* ex14, int nex14, double* force, double* e_vdw, double* e_elec,
                             double* e_excl, double* vir9) {
  double ev = 0, ee = 0, ex = 0, w[9] = {0};
  for (int pass = 0; pass < 2; pass++) {
    const int* L = pass == 0 ? in14 : ex14;
    const int n = pass == 0 ? nin14 : nex14;
    for (int k = 0; k < n; k++) {
      const int i = L[3 * k], j = L[3 * k + 1];
      int ish = L[3 * k + 2];
      const double sh[3] = {(double)(ish % 3 - 1) * box3[0], (double)((ish / 3) % 3 - 1) * box3[1],
                            (double)(ish / 9 - 1) * box3[2]};
      double dx[3];
      for (int d = 0; d < 3; d++) dx[d] = xyzq[4 * i + d] - xyzq[4 * j + d] + sh[d];
      const double r2 = dx[0] * dx[0] + dx[1] * dx[1] + dx[2] * dx[2];
      const double qq = kCcelec * xyzq[4 * i + 3] * xyzq[4 * j + 3];
      double c6 = 0, c12 = 0;
      if (pass == 0) vdw_c6c12(vdwparam14, vdwtype, i, j, &c6, &c12);
      // no cutoff test for listed pairs; the VSH shift terms use roff as for the main pairs
      const DirectPair p = direct_pair(r2, qq, c6, c12, kappa, roff, pass == 0 ? e14fac : 0.0, pass == 0);
      for (int d = 0; d < 3; d++) {
        force[3 * i + d] += p.f_over_r2 * dx[d];
        force[3 * j + d] -= p.f_over_r2 * dx[d];
      }
      if (pass == 0) { ev += p.u_vdw; ee += p.u_elec; } else { ex += p.u_elec; }
      for (int a = 0; a < 3; a++)
        for (int b = 0; b < 3; b++) w[3 * a + b] -= p.f_over_r2 * dx[a] * dx[b];
    }
  }
  if (e_vdw) *e_vdw = ev;
  if (e_elec) *e_elec = ee;
  if (e_excl) *e_excl = ex;
  if (vir9) for (int c = 0; c < 9; c++) vir9[c] = w[c];
  return 0;
}

extern "C" int orc_hardware_threads(void) { return hw_threads(0); }

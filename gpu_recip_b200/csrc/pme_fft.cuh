// pme_fft.cuh -- shared-memory mixed-radix FFT engine for the 3-D PME transforms (sm_100a).
//
// A CTA owns a tile of TX lines of length L, held in shared memory with element e of line t at
// buf[e * ld + t] (ld >= TX; consecutive threads work on consecutive lines, so shared-memory
// accesses are conflict free).  The transform is a Stockham autosort FFT: stage s with radix R
// reads butterfly j's inputs at j + r*L/R, twiddles them by W_{Ns R}^{r k} (k = j mod Ns), does an
// R-point DFT in registers and writes the outputs at (j div Ns) Ns R + k + u Ns, ping-ponging
// between two buffers.  Radices 8, 4, 2, 3, 5 (largest power of two first) cover every
// 2/3/5-smooth length.  Twiddles W_L^i = exp(-2 pi i i/L) are read from a per-length table
// computed in FP64 on the host and rounded to FP32.  sign = -1 forward, +1 inverse; transforms are unnormalised.
#pragma once

#include <cuda_runtime.h>

namespace pme {

constexpr int kMaxStages = 12;
constexpr int kMaxFftLen = 512;

// Division by a small constant d (1 <= d <= 2^16) as one multiply-high: x / d == umulhi(x, m)
// with m = ceil(2^32 / d), exact for 0 <= x < 2^32 / d (all index ranges here are < 2^16).
struct FastDiv {
  unsigned int m;
  int d;
};

__host__ __device__ inline FastDiv make_fastdiv(int d) {
  FastDiv f;
  f.d = d;
  f.m = d <= 1 ? 0u : (unsigned int)((0x100000000ull + (unsigned long long)d - 1ull) / (unsigned long long)d);
  return f;
}

__device__ __forceinline__ int fdiv(int x, const FastDiv& f) {
  return f.d <= 1 ? x : (int)__umulhi((unsigned int)x, f.m);
}

struct FftPlan1D {
  int n;                    // transform length
  int code;                 // > 0: a length with a compile-time stage sequence (fft_tile)
  int nstages;
  int radix[kMaxStages];
  FastDiv ns_div[kMaxStages];   // division by the stage's sub-transform length Ns
  FastDiv n_div;                // division by n
  int tw_off;               // offset of this length's table in the twiddle array
};

__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(__fmaf_rn(a.x, b.x, -__fmul_rn(a.y, b.y)), __fmaf_rn(a.x, b.y, __fmul_rn(a.y, b.x)));
}
__device__ __forceinline__ float2 cadd(float2 a, float2 b) {
  return make_float2(__fadd_rn(a.x, b.x), __fadd_rn(a.y, b.y));
}
__device__ __forceinline__ float2 csub(float2 a, float2 b) {
  return make_float2(__fsub_rn(a.x, b.x), __fsub_rn(a.y, b.y));
}
// a + s b with one rounding per component (explicit FMA)
__device__ __forceinline__ float2 cfma(float s, float2 b, float2 a) {
  return make_float2(__fmaf_rn(s, b.x, a.x), __fmaf_rn(s, b.y, a.y));
}
// s * i * a for s = +1 / -1:  i (x + i y) = -y + i x
__device__ __forceinline__ float2 cmul_si(float2 a, bool inv) {
  return inv ? make_float2(-a.y, a.x) : make_float2(a.y, -a.x);
}

// R-point DFTs in registers.  Forward uses W_R = exp(-2 pi i / R); inverse its conjugate.
template <int R> __device__ __forceinline__ void dft_small(float2* v, bool inv);

template <> __device__ __forceinline__ void dft_small<2>(float2* v, bool) {
  float2 a = cadd(v[0], v[1]), b = csub(v[0], v[1]);
  v[0] = a; v[1] = b;
}

template <> __device__ __forceinline__ void dft_small<4>(float2* v, bool inv) {
  float2 a0 = cadd(v[0], v[2]), a1 = csub(v[0], v[2]);
  float2 b0 = cadd(v[1], v[3]), b1 = csub(v[1], v[3]);
  float2 jb1 = cmul_si(b1, inv);          // forward: -i b1, inverse: +i b1
  v[0] = cadd(a0, b0);
  v[2] = csub(a0, b0);
  v[1] = cadd(a1, jb1);
  v[3] = csub(a1, jb1);
}

template <> __device__ __forceinline__ void dft_small<3>(float2* v, bool inv) {
  const float h = 0.866025403784438646763723f;   // sin(2 pi/3)
  float2 s = cadd(v[1], v[2]), d = csub(v[1], v[2]);
  float2 m = cfma(-0.5f, s, v[0]);
  float2 jd = cmul_si(d, inv);                    // forward: -i d
  v[0] = cadd(v[0], s);
  v[1] = cfma(h, jd, m);
  v[2] = cfma(-h, jd, m);
}

template <> __device__ __forceinline__ void dft_small<5>(float2* v, bool inv) {
  const float c1 = 0.309016994374947424102293f;   // cos(2 pi/5)
  const float c2 = -0.809016994374947424102293f;  // cos(4 pi/5)
  const float s1 = 0.951056516295153572116439f;   // sin(2 pi/5)
  const float s2 = 0.587785252292473129168706f;   // sin(4 pi/5)
  float2 a1 = cadd(v[1], v[4]), b1 = csub(v[1], v[4]);
  float2 a2 = cadd(v[2], v[3]), b2 = csub(v[2], v[3]);
  float2 x0 = v[0];
  float2 r1 = cfma(c2, a2, cfma(c1, a1, x0));
  float2 r2 = cfma(c1, a2, cfma(c2, a1, x0));
  float2 t1 = cfma(s2, b2, make_float2(__fmul_rn(s1, b1.x), __fmul_rn(s1, b1.y)));
  float2 t2 = cfma(-s1, b2, make_float2(__fmul_rn(s2, b1.x), __fmul_rn(s2, b1.y)));
  float2 j1 = cmul_si(t1, inv), j2 = cmul_si(t2, inv);   // forward: -i t
  v[0] = cadd(cadd(x0, a1), a2);
  v[1] = cadd(r1, j1);
  v[4] = csub(r1, j1);
  v[2] = cadd(r2, j2);
  v[3] = csub(r2, j2);
}

// 8-point DFT as two 4-point DFTs of the even and odd inputs, joined by the twiddles W_8^k:
// forward W_8 = (1 - i)/sqrt(2), W_8^2 = -i, W_8^3 = -(1 + i)/sqrt(2); inverse the conjugates.
template <> __device__ __forceinline__ void dft_small<8>(float2* v, bool inv) {
  const float r = 0.707106781186547524400844f;   // 1/sqrt(2)
  float2 e[4] = {v[0], v[2], v[4], v[6]};
  float2 o[4] = {v[1], v[3], v[5], v[7]};
  dft_small<4>(e, inv);
  dft_small<4>(o, inv);
  // o[1] *= W_8, o[2] *= W_8^2, o[3] *= W_8^3
  const float2 a = o[1], c = o[3];
  if (!inv) {
    o[1] = make_float2(__fmul_rn(__fadd_rn(a.x, a.y), r), __fmul_rn(__fsub_rn(a.y, a.x), r));
    o[3] = make_float2(__fmul_rn(__fsub_rn(c.y, c.x), r), -__fmul_rn(__fadd_rn(c.x, c.y), r));
  } else {
    o[1] = make_float2(__fmul_rn(__fsub_rn(a.x, a.y), r), __fmul_rn(__fadd_rn(a.x, a.y), r));
    o[3] = make_float2(-__fmul_rn(__fadd_rn(c.x, c.y), r), __fmul_rn(__fsub_rn(c.x, c.y), r));
  }
  o[2] = cmul_si(o[2], inv);
#pragma unroll
  for (int k = 0; k < 4; k++) {
    v[k] = cadd(e[k], o[k]);
    v[k + 4] = csub(e[k], o[k]);
  }
}

// Thread placement inside a tile: line t = tid mod nlines, butterfly lane y = tid div nlines
// (lanes 0..ny-1; threads beyond nlines*ny idle during stages).
struct TileLane {
  int t, y, ny;
  __device__ __forceinline__ TileLane(int tid, int nthreads, int nlines) {
    t = tid % nlines;
    y = tid / nlines;
    ny = nthreads / nlines;
  }
  __device__ __forceinline__ bool active() const { return y < ny; }
};

// One Stockham stage over all lines of the tile; element e of line t lives at e*es + t*ls.
template <int R>
__device__ __forceinline__ void fft_stage(const float2* __restrict__ in, float2* __restrict__ out,
                                          int L, int Ns, const FastDiv& nsd, int es, int ls,
                                          const TileLane& ln, const float2* tw, bool inv) {
  const int nb = L / R;
  const int tstride = L / (Ns * R);
  const int lo = ln.t * ls;
  if (!ln.active()) return;
  for (int j = ln.y; j < nb; j += ln.ny) {
    const int blk = fdiv(j, nsd);
    const int k = j - blk * Ns;
    float2 v[R];
#pragma unroll
    for (int r = 0; r < R; r++) v[r] = in[(j + r * nb) * es + lo];
#pragma unroll
    for (int r = 1; r < R; r++) {
      float2 w = tw[r * k * tstride];
      if (inv) w.y = -w.y;
      v[r] = cmul(v[r], w);
    }
    dft_small<R>(v, inv);
    const int base = blk * Ns * R + k;
#pragma unroll
    for (int u = 0; u < R; u++) out[(base + u * Ns) * es + lo] = v[u];
  }
}

// One Stockham stage with the radix, the sub-transform length NS and the line length L known at
// compile time: the same butterflies and the same roundings as fft_stage, with constant index
// arithmetic.
template <int R, int NS, int L>
__device__ __forceinline__ void fft_stage_ct(const float2* __restrict__ in, float2* __restrict__ out, int es, int ls,
                                             const TileLane& ln, const float2* tw, bool inv) {
  constexpr int nb = L / R;
  constexpr int tstride = L / (NS * R);
  const int lo = ln.t * ls;
  if (!ln.active()) return;
  for (int j = ln.y; j < nb; j += ln.ny) {
    const int blk = j / NS;
    const int k = j - blk * NS;
    float2 v[R];
#pragma unroll
    for (int r = 0; r < R; r++) v[r] = in[(j + r * nb) * es + lo];
#pragma unroll
    for (int r = 1; r < R; r++) {
      float2 w = tw[r * k * tstride];
      if (inv) w.y = -w.y;
      v[r] = cmul(v[r], w);
    }
    dft_small<R>(v, inv);
    const int base = blk * NS * R + k;
#pragma unroll
    for (int u = 0; u < R; u++) out[(base + u * NS) * es + lo] = v[u];
  }
}

// The stages R, Rest... of a length-L transform from sub-transform length NS on, unrolled at
// compile time; returns the buffer holding the result.
template <int L, int NS, int R, int... Rest>
__device__ __forceinline__ float2* fft_seq_ct(float2* src, float2* dst, int es, int ls, const TileLane& ln,
                                              const float2* tw, bool inv) {
  fft_stage_ct<R, NS, L>(src, dst, es, ls, ln, tw, inv);
  __syncthreads();
  if constexpr (sizeof...(Rest) == 0) {
    return dst;
  } else {
    return fft_seq_ct<L, NS * R, Rest...>(dst, src, es, ls, ln, tw, inv);
  }
}

// Lengths with a compile-time stage sequence (FftPlan1D::code): a generic stage loop with a
// runtime radix costs about three times the cycles of the same stages unrolled (measured on a
// 16 x 64 tile: 2,390 against 730 cycles per transform).
// The lengths are those of the benchmarked grids: 32, 64, 216 and the 24-60 of the batch.
enum {
  kFftGeneric = 0, kFft64, kFft32, kFft216, kFft24, kFft25, kFft27, kFft30, kFft36, kFft40, kFft45, kFft48,
  kFft50, kFft54, kFft60
};
__host__ __device__ inline int fft_code(int n) {
  switch (n) {
    case 64: return kFft64;
    case 32: return kFft32;
    case 216: return kFft216;
    case 24: return kFft24;
    case 25: return kFft25;
    case 27: return kFft27;
    case 30: return kFft30;
    case 36: return kFft36;
    case 40: return kFft40;
    case 45: return kFft45;
    case 48: return kFft48;
    case 50: return kFft50;
    case 54: return kFft54;
    case 60: return kFft60;
    default: return kFftGeneric;
  }
}

// The batch lengths (24-60), in a function of their own that fft_tile calls: fft_tile's dispatch
// for 64, 32 and 216 stays a short compare chain (one switch over all fourteen lengths cost the
// 32^3 evaluation 2 us).
static __device__ __noinline__ float2* fft_tile_batch(float2* buf0, float2* buf1, int code, int es, int ls,
                                                      const TileLane ln, const float2* tw, bool inv) {
  switch (code) {
    case kFft24: return fft_seq_ct<24, 1, 8, 3>(buf0, buf1, es, ls, ln, tw, inv);
    case kFft25: return fft_seq_ct<25, 1, 5, 5>(buf0, buf1, es, ls, ln, tw, inv);
    case kFft27: return fft_seq_ct<27, 1, 3, 3, 3>(buf0, buf1, es, ls, ln, tw, inv);
    case kFft30: return fft_seq_ct<30, 1, 2, 3, 5>(buf0, buf1, es, ls, ln, tw, inv);
    case kFft36: return fft_seq_ct<36, 1, 4, 3, 3>(buf0, buf1, es, ls, ln, tw, inv);
    case kFft40: return fft_seq_ct<40, 1, 8, 5>(buf0, buf1, es, ls, ln, tw, inv);
    case kFft45: return fft_seq_ct<45, 1, 3, 3, 5>(buf0, buf1, es, ls, ln, tw, inv);
    case kFft48: return fft_seq_ct<48, 1, 8, 2, 3>(buf0, buf1, es, ls, ln, tw, inv);
    case kFft50: return fft_seq_ct<50, 1, 2, 5, 5>(buf0, buf1, es, ls, ln, tw, inv);
    case kFft54: return fft_seq_ct<54, 1, 2, 3, 3, 3>(buf0, buf1, es, ls, ln, tw, inv);
    default: return fft_seq_ct<60, 1, 4, 3, 5>(buf0, buf1, es, ls, ln, tw, inv);
  }
}

// Full transform of every line of the tile held in buf0 (element stride es, line stride ls);
// returns the buffer that holds the result (buf0 or buf1).  Every thread of the CTA must call
// it; it synchronises between stages and before returning.  Not inlined: the fused evaluation
// runs it in five phases, and one shared copy of its stages is what those phases fetch (with L2
// cold, per-phase inlined copies cost ~15 us of instruction fetch per evaluation).
static __device__ __noinline__ float2* fft_tile(float2* buf0, float2* buf1, const FftPlan1D& plan,
                                         int es, int ls, const TileLane ln, const float2* tw,
                                         bool inv) {
  switch (plan.code) {   // factorize() orders the radices 8, 4, 2, 3, 5
    case kFft64: return fft_seq_ct<64, 1, 8, 8>(buf0, buf1, es, ls, ln, tw, inv);
    case kFft32: return fft_seq_ct<32, 1, 8, 4>(buf0, buf1, es, ls, ln, tw, inv);
    case kFft216: return fft_seq_ct<216, 1, 8, 3, 3, 3>(buf0, buf1, es, ls, ln, tw, inv);
    default: break;
  }
  if (plan.code >= kFft24) return fft_tile_batch(buf0, buf1, plan.code, es, ls, ln, tw, inv);
  float2* src = buf0;
  float2* dst = buf1;
  int Ns = 1;
  const int L = plan.n;
  for (int s = 0; s < plan.nstages; s++) {
    const int R = plan.radix[s];
    const FastDiv nsd = plan.ns_div[s];
    switch (R) {
      case 8: fft_stage<8>(src, dst, L, Ns, nsd, es, ls, ln, tw, inv); break;
      case 4: fft_stage<4>(src, dst, L, Ns, nsd, es, ls, ln, tw, inv); break;
      case 2: fft_stage<2>(src, dst, L, Ns, nsd, es, ls, ln, tw, inv); break;
      case 3: fft_stage<3>(src, dst, L, Ns, nsd, es, ls, ln, tw, inv); break;
      case 5: fft_stage<5>(src, dst, L, Ns, nsd, es, ls, ln, tw, inv); break;
      default: break;
    }
    __syncthreads();
    float2* tmp = src; src = dst; dst = tmp;
    Ns *= R;
  }
  return src;
}

}  // namespace pme

// pme_direct.cu -- direct-space (real-space) PME nonbonded terms on sm_100a (include/pme_direct.h).
//
// The role of CudaPMEDirectForce<long long, float> with its topological exclusions, for the
// models of the reference's direct test: shifted Lennard-Jones (VDW_VSH,
// CudaDirectForceKernels.cu:175-195) and Ewald real-space electrostatics (EWALD, :353-391).
//
// One calc_force is five launches on the handle's stream:
//   k_direct_cell   atom -> cell (cells >= roff along x, >= roff/2 along y and z), counts;
//   k_direct_scan   cell starts (one CTA);
//   k_direct_fill   atoms into their cells (unordered);
//   k_direct_order  one warp per cell: order the cell's atoms by index (so every run sums in the
//                   same order) and gather coordinates, type, global index and exclusion window;
//   k_direct_pairs  one warp per 32 atoms of a cell (lane = atom i) and z slice of its 3 x 5 x 5
//                   neighbouring cells: a cheap distance/exclusion pass compacts the pairs within
//                   roff, whose terms then run on full lanes.
// Each pair is evaluated from both sides (no third-law scatter): each pair's force is rounded once
// to 2^-40 and every sum after that is exact int64, so results are run-to-run identical and the
// only FP32 error is that of the pair terms themselves.  Energies are rounded to 2^-32 per pair and summed in int64; both sides
// give the same pair distance (dx = (x_i - x_j) - shift is antisymmetric), so the doubled sums
// halve exactly (1-4 terms are added twice to match).
// Exclusions: a 128-bit window per atom over global indices g_j - g_i in [-64, 64) (bit 64: the
// atom itself), plus an explicit list for partners beyond the window.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "../../include/pme_direct.h"
#include "pme_state.h"

namespace pme {
namespace direct {

constexpr int kWarps = 8;             // warps per CTA of the pair kernel (256 threads)
constexpr int kMaxTypes = 200;        // vdW types (packed pairs held in shared memory)
constexpr float kEnergyScale = 4294967296.0f;     // 2^32
constexpr float kForceScaleF = 1099511627776.0f;  // 2^40
constexpr float kTwoSqrtPi = 1.1283791670955126f; // 2/sqrt(pi)
constexpr int kTabN = 4096;          // Ewald table intervals
constexpr double kTabR0 = 1.5;       // Ewald table from r = 1.5 A (closer pairs use erfc and exp)

struct Params {
  float box[3], inv_box[3];
  float kappa, kappa2, roff2, ro6, ro12, ro18;   // roff^-6, roff^-12, roff^-18
  float e14fac;
  int vdw, elec;
  int nc[3];          // cells per axis
  int lo[3], cnt[3];  // neighbour cell offsets per axis: lo .. lo + cnt - 1
  int npair;          // vdW type pairs
  double kappad, ro6d, ro12d, ro18d;   // FP64 copies for the main-list pair terms
  double boxd[3];
  // Ewald real-space table (Hermite cubic in s = r^2 on [tab_s0, roff^2], tab_n intervals):
  // per node (E, h dE/ds, F, h dF/ds) with E = erfc(kappa r)/r and F = (r dE/dr) / r^2
  const double4* tab;
  double tab_s0, tab_invh;
  int tab_n;
};

enum Acc { kAccVdw = 0, kAccElec = 1, kAccExcl = 2, kAccVir = 3, kAccN = 9 };   // vir: xx xy xz yy yz zz

// r dU/dr / r^2 and the energies of one pair at squared distance r2.  a_elec is the factor of
// qq / r in U_elec: erfc(kappa r) for ordinary pairs, e14fac - erf(kappa r) for 1-4 pairs,
// -erf(kappa r) for excluded pairs (formed with erff, not as erfc + s - 1, which cancels in FP32).
// c6 / c12 carry the reference's factors 6 and 12.
__device__ __forceinline__ float pair_terms(float r2, float qq, float c6, float c12, const Params& p, int kind,
                                            bool vdw, float& u_vdw, float& u_elec) {
  const float r = sqrtf(r2);        // IEEE square root and reciprocal, as the reference computes them
  const float rinv = 1.0f / r;
  const float rinv2 = rinv * rinv;
  float fr = 0.0f;
  u_vdw = 0.0f;
  if (vdw) {
    const float rinv6 = rinv2 * rinv2 * rinv2, rinv12 = rinv6 * rinv6, r6 = r2 * r2 * r2;
    fr = c6 * (rinv6 - r6 * p.ro12) - c12 * (rinv12 + r6 * p.ro18);
    u_vdw = c12 * (1.0f / 12.0f) * (rinv12 + 2.0f * r6 * p.ro18 - 3.0f * p.ro12) -
            c6 * (1.0f / 6.0f) * (rinv6 + r6 * p.ro12 - 2.0f * p.ro6);
  }
  u_elec = 0.0f;
  if (p.elec == PME_ELEC_NONE) return fr * rinv2;
  const float kr = p.kappa * r;
  const float a = kind == 0 ? erfcf(kr) : (kind == 1 ? p.e14fac - erff(kr) : -erff(kr));
  const float e = qq * a * rinv;
  u_elec = e;
  fr += -qq * kTwoSqrtPi * p.kappa * expf(-p.kappa2 * r2) - e;
  return fr * rinv2;
}

// The same terms in FP64 from the FP32 pair geometry, for the main pair list: the atoms' net
// forces are small differences of large pair forces (close contacts of ~1e3 kcal/mol/A), where
// the few-ulp error of an FP32 evaluation shows.
__device__ __forceinline__ double pair_terms_f64(double r2, double qq, double c6, double c12, const Params& p,
                                                 bool vdw, double& u_vdw, double& u_elec) {
  const double rinv = rsqrt(r2);
  const double r = r2 * rinv;
  const double rinv2 = rinv * rinv;
  double fr = 0.0;
  u_vdw = 0.0;
  if (vdw) {
    const double rinv6 = rinv2 * rinv2 * rinv2, rinv12 = rinv6 * rinv6, r6 = r2 * r2 * r2;
    fr = c6 * (rinv6 - r6 * p.ro12d) - c12 * (rinv12 + r6 * p.ro18d);
    u_vdw = c12 * (1.0 / 12.0) * (rinv12 + 2.0 * r6 * p.ro18d - 3.0 * p.ro12d) -
            c6 * (1.0 / 6.0) * (rinv6 + r6 * p.ro12d - 2.0 * p.ro6d);
  }
  u_elec = 0.0;
  if (p.elec == PME_ELEC_NONE) return fr * rinv2;
  if (p.tab != nullptr && r2 >= p.tab_s0) {
    const double u = (r2 - p.tab_s0) * p.tab_invh;
    const int i = min((int)u, p.tab_n - 1);
    const double t = u - (double)i;
    const double2* q = reinterpret_cast<const double2*>(p.tab + i);
    const double2 a0 = __ldg(q), a1 = __ldg(q + 1), b0 = __ldg(q + 2), b1 = __ldg(q + 3);
    const double t2 = t * t;
    const double h01 = t2 * (3.0 - 2.0 * t), h00 = 1.0 - h01;
    const double h10 = t * (1.0 - t) * (1.0 - t), h11 = t2 * (t - 1.0);
    u_elec = qq * (h00 * a0.x + h10 * a0.y + h01 * b0.x + h11 * b0.y);
    return fr * rinv2 + qq * (h00 * a1.x + h10 * a1.y + h01 * b1.x + h11 * b1.y);
  }
  const double e = qq * erfc(p.kappad * r) * rinv;
  u_elec = e;
  fr += -qq * 1.1283791670955126 * p.kappad * exp(-p.kappad * p.kappad * r2) - e;
  return fr * rinv2;
}

__device__ __forceinline__ float2 vdw_c6c12(const float2* tab, int ta, int tb) {
  const int a = max(ta, tb), b = min(ta, tb);
  return tab[a * (a + 1) / 2 + b];
}

__device__ __forceinline__ long long warp_sum_ll(long long v) {
#pragma unroll
  for (int off = 16; off >= 1; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
  return v;
}

// ---------------------------------------------------------------------------------------------
// Binning
// ---------------------------------------------------------------------------------------------
// Coordinate wrapped into the box: x - L floor(x / L), which FP32 rounding can leave a hair below
// 0 or equal to L; non-finite inputs become 0.  The cell comes from this same value, so an atom's
// cell and its stored position always agree (the cells are wider than their reach by a margin).
__device__ __forceinline__ float wrap_coord(float x, float box, float inv_box) {
  const float w = x - box * floorf(x * inv_box);
  return (w >= -box && w <= 2.0f * box) ? w : 0.0f;
}

__device__ __forceinline__ int cell_of_wrapped(float w, float inv_box, int n) {
  return max(0, min((int)(w * inv_box * (float)n), n - 1));
}

__global__ void k_direct_cell(const float4* __restrict__ xyzq, int n, const Params p, int* __restrict__ cell_of,
                              int* __restrict__ count) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float4 a = xyzq[i];
  const int cx = cell_of_wrapped(wrap_coord(a.x, p.box[0], p.inv_box[0]), p.inv_box[0], p.nc[0]);
  const int cy = cell_of_wrapped(wrap_coord(a.y, p.box[1], p.inv_box[1]), p.inv_box[1], p.nc[1]);
  const int cz = cell_of_wrapped(wrap_coord(a.z, p.box[2], p.inv_box[2]), p.inv_box[2], p.nc[2]);
  const int c = (cz * p.nc[1] + cy) * p.nc[0] + cx;
  cell_of[i] = c;
  atomicAdd(&count[c], 1);
}

// Exclusive scans of count[0..ncell) into start[0..ncell] (atoms) and of ceil(count / 32) into
// chunk[0..ncell] (32-atom chunks, chunk[ncell] the total); one CTA of 1024 threads, each owning a
// contiguous run of cells.
__global__ void __launch_bounds__(1024) k_direct_scan(const int* __restrict__ count, int ncell, int* __restrict__ start,
                                                      int* __restrict__ chunk) {
  __shared__ int part[1024], partc[1024];
  const int t = threadIdx.x;
  const int per = (ncell + 1023) / 1024;
  const int b = min(t * per, ncell), e = min(b + per, ncell);
  int s = 0, sc = 0;
  for (int c = b; c < e; c++) {
    s += count[c];
    sc += (count[c] + 31) >> 5;
  }
  part[t] = s;
  partc[t] = sc;
  __syncthreads();
  for (int off = 1; off < 1024; off <<= 1) {   // inclusive Hillis-Steele scans of the run sums
    const int v = t >= off ? part[t - off] : 0;
    const int vc = t >= off ? partc[t - off] : 0;
    __syncthreads();
    part[t] += v;
    partc[t] += vc;
    __syncthreads();
  }
  int run = part[t] - s, runc = partc[t] - sc;
  for (int c = b; c < e; c++) {
    start[c] = run;
    chunk[c] = runc;
    run += count[c];
    runc += (count[c] + 31) >> 5;
  }
  if (t == 1023) {
    start[ncell] = part[1023];
    chunk[ncell] = partc[1023];
  }
}

__global__ void k_direct_fill(const int* __restrict__ cell_of, int n, const int* __restrict__ start,
                              int* __restrict__ fill, int* __restrict__ tmp) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int c = cell_of[i];
  tmp[start[c] + atomicAdd(&fill[c], 1)] = i;
}

// One warp per cell: rank each of the cell's atoms by index and gather its data to that slot.
__global__ void k_direct_order(const int* __restrict__ start, int ncell, const int* __restrict__ tmp,
                               const float4* __restrict__ xyzq, const int* __restrict__ vdwtype,
                               const int* __restrict__ glob, const ulonglong2* __restrict__ win,
                               const int* __restrict__ far_ptr, float box_x, float box_y, float box_z, float inv_x,
                               float inv_y, float inv_z, float4* __restrict__ pos, int4* __restrict__ info,
                               ulonglong2* __restrict__ mask) {
  const int lane = threadIdx.x & 31;
  for (int c = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; c < ncell; c += (gridDim.x * blockDim.x) >> 5) {
    const int s = start[c], e = start[c + 1];
    for (int k = s + lane; k < e; k += 32) {
      const int a = tmp[k];
      int rank = 0;
      for (int m = s; m < e; m++) rank += tmp[m] < a ? 1 : 0;
      const int d = s + rank;
      float4 q = xyzq[a];   // wrapped: neighbour cells then need only their periodic shift
      q.x = wrap_coord(q.x, box_x, inv_x);
      q.y = wrap_coord(q.y, box_y, inv_y);
      q.z = wrap_coord(q.z, box_z, inv_z);
      pos[d] = q;
      info[d] = make_int4(vdwtype[a], glob[a], a, far_ptr[a + 1] > far_ptr[a] ? 1 : 0);
      mask[d] = win[a];
    }
  }
}

// ---------------------------------------------------------------------------------------------
// Pairs
// ---------------------------------------------------------------------------------------------
__device__ __forceinline__ bool far_excluded(const int* __restrict__ far_ptr, const int* __restrict__ far_idx,
                                             int i, int gj) {
  for (int k = far_ptr[i]; k < far_ptr[i + 1]; k++)
    if (far_idx[k] == gj) return true;
  return false;
}

// One warp per (cell, 32-atom chunk of it, z slice of its neighbour cells): lane = atom i.  For
// each batch of 32 j atoms staged in shared memory, a cheap pass tests the 32 x 32 pairs (distance
// with the neighbour cell's periodic shift, or the minimum image when an axis has too few cells,
// then the exclusion window) and compacts the hits into a per-warp list; the pair terms then run
// in FP64 (from the FP32 positions, exactly) on full lanes, 32 hits at a time (the list is ordered
// by i, so a segmented warp scan folds each i's run into one add to its shared-memory
// accumulator).  Every pair force is rounded once to 2^-40 and summed in
// int64 from there on (exact: no accumulation error, and no dependence on the order of the adds
// or of the slices).  FP64 because an atom's net force is a small difference of large pair forces,
// where the few-ulp error of FP32 pair terms reaches ~1e-5 kcal/mol/A.
template <bool MINIMG>
__global__ void __launch_bounds__(kWarps * 32, 3) k_direct_pairs(
    const Params p, const int* __restrict__ start, const int* __restrict__ chunkp, const float4* __restrict__ pos,
    const int4* __restrict__ info,
    const ulonglong2* __restrict__ mask, const int* __restrict__ far_ptr, const int* __restrict__ far_idx,
    const float2* __restrict__ vdwp, int calc_energy, int calc_virial, int stride, long long* __restrict__ force,
    long long* __restrict__ acc, int* __restrict__ next_task) {
  extern __shared__ float2 sh_vdw[];
  __shared__ float4 sh_jpos[kWarps][32];
  __shared__ int2 sh_jtg[kWarps][32];
  __shared__ float4 sh_ipos[kWarps][32];
  __shared__ int sh_itype[kWarps][32];
  __shared__ long long sh_f[kWarps][3][32];   // force sums at 2^40 (exact)
  __shared__ unsigned short sh_items[kWarps][1024];
  for (int k = threadIdx.x; k < p.npair; k += blockDim.x) sh_vdw[k] = vdwp[k];
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int ncell = p.nc[0] * p.nc[1] * p.nc[2];
  const int nslice = p.cnt[2];
  const bool vdw_on = p.vdw != PME_VDW_NONE;
  long long ev = 0, ee = 0;
  long long wv[6] = {0, 0, 0, 0, 0, 0};   // virial at 2^32: each task's FP64 partials folded in (exact)
  const int nchunk = chunkp[ncell];
  const int ntask = nchunk * nslice;
  // tasks differ in cost (cell populations): warps take them one at a time from a counter
  for (;;) {
    int task = 0;
    if (lane == 0) task = atomicAdd(next_task, 1);
    task = __shfl_sync(0xffffffffu, task, 0);
    if (task >= ntask) break;
    const int sl = task % nslice;
    const int g = task / nslice;
    int clo = 0, chi = ncell - 1;   // the cell holding chunk g: last c with chunkp[c] <= g
    while (clo < chi) {
      const int mid = (clo + chi + 1) >> 1;
      if (chunkp[mid] <= g) clo = mid; else chi = mid - 1;
    }
    const int c = clo;
    const int ce = start[c + 1];
    const int cx = c % p.nc[0], cy = (c / p.nc[0]) % p.nc[1], cz = c / (p.nc[0] * p.nc[1]);
    double w0 = 0.0, w1 = 0.0, w2 = 0.0, w3 = 0.0, w4 = 0.0, w5 = 0.0;   // this task's, in a fixed order
    {
      const int chunk = start[c] + (g - chunkp[c]) * 32;
      const int i = chunk + lane;
      const bool act = i < ce;
      const float4 pi = act ? pos[i] : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
      const int4 ii = act ? info[i] : make_int4(0, 0, 0, 0);
      const ulonglong2 mi = act ? mask[i] : make_ulonglong2(0ull, 0ull);
      sh_ipos[warp][lane] = pi;
      sh_itype[warp][lane] = ii.x;
      sh_f[warp][0][lane] = 0;
      sh_f[warp][1][lane] = 0;
      sh_f[warp][2][lane] = 0;
      // this task's z slice of the neighbour cells, with its periodic shift
      int z = MINIMG && p.cnt[2] == p.nc[2] ? sl : cz + p.lo[2] + sl;
      float shz = 0.0f;
      if (!MINIMG) {
        if (z < 0) { z += p.nc[2]; shz = -p.box[2]; } else if (z >= p.nc[2]) { z -= p.nc[2]; shz = p.box[2]; }
      } else if (p.cnt[2] != p.nc[2]) {
        z = (z + p.nc[2]) % p.nc[2];
      }
      __syncwarp();
      for (int oy = 0; oy < p.cnt[1]; oy++) {
        int y = MINIMG && p.cnt[1] == p.nc[1] ? oy : cy + p.lo[1] + oy;
        float shy = 0.0f;
        if (!MINIMG) {
          if (y < 0) { y += p.nc[1]; shy = -p.box[1]; } else if (y >= p.nc[1]) { y -= p.nc[1]; shy = p.box[1]; }
        } else if (p.cnt[1] != p.nc[1]) {
          y = (y + p.nc[1]) % p.nc[1];
        }
        for (int ox = 0; ox < p.cnt[0]; ox++) {
          int x = MINIMG && p.cnt[0] == p.nc[0] ? ox : cx + p.lo[0] + ox;
          float shx = 0.0f;
          if (!MINIMG) {
            if (x < 0) { x += p.nc[0]; shx = -p.box[0]; } else if (x >= p.nc[0]) { x -= p.nc[0]; shx = p.box[0]; }
          } else if (p.cnt[0] != p.nc[0]) {
            x = (x + p.nc[0]) % p.nc[0];
          }
          const int cn = (z * p.nc[1] + y) * p.nc[0] + x;
          const int js = start[cn], je = start[cn + 1];
          for (int b = js; b < je; b += 32) {
            if (b + lane < je) {
              sh_jpos[warp][lane] = pos[b + lane];
              const int4 jt = info[b + lane];
              sh_jtg[warp][lane] = make_int2(jt.x, jt.y);
            }
            __syncwarp();
            const int nb = min(32, je - b);
            // cheap pass: which of the batch's j are partners of this lane's i
            unsigned hits = 0u;
            if (act) {
              for (int t = 0; t < nb; t++) {
                const float4 pj = sh_jpos[warp][t];
                float dx = pi.x - pj.x, dy = pi.y - pj.y, dz = pi.z - pj.z;
                if (MINIMG) {
                  dx -= p.box[0] * rintf(dx * p.inv_box[0]);
                  dy -= p.box[1] * rintf(dy * p.inv_box[1]);
                  dz -= p.box[2] * rintf(dz * p.inv_box[2]);
                } else {
                  dx -= shx; dy -= shy; dz -= shz;
                }
                const float r2 = dx * dx + dy * dy + dz * dz;
                if (r2 < p.roff2) {
                  const unsigned k = (unsigned)(sh_jtg[warp][t].y - ii.y + 64);
                  bool excl;
                  if (k < 128u) {
                    const unsigned long long wb = k < 64u ? mi.x : mi.y;
                    excl = ((wb >> (k & 63u)) & 1ull) != 0ull;
                  } else {
                    excl = ii.w != 0 && far_excluded(far_ptr, far_idx, ii.z, sh_jtg[warp][t].y);
                  }
                  if (!excl) hits |= 1u << t;
                }
              }
            }
            // compact the hits, ordered by lane (i) then j
            const int cnt = __popc(hits);
            int off = cnt;
#pragma unroll
            for (int d = 1; d < 32; d <<= 1) {
              const int v = __shfl_up_sync(0xffffffffu, off, d);
              if (lane >= d) off += v;
            }
            const int total = __shfl_sync(0xffffffffu, off, 31);
            off -= cnt;
            for (unsigned m = hits; m; m &= m - 1u) sh_items[warp][off++] = (unsigned short)((lane << 5) | (__ffs(m) - 1));
            __syncwarp();
            // pair terms on full lanes
            for (int base = 0; base < total; base += 32) {
              const bool valid = base + lane < total;
              const int item = valid ? sh_items[warp][base + lane] : 0;
              const int il = valid ? item >> 5 : 32 + lane;   // invalid lanes get keys of their own
              long long gx = 0, gy = 0, gz = 0;
              if (valid) {
                const int t = item & 31;
                const float4 a = sh_ipos[warp][il];
                const float4 pj = sh_jpos[warp][t];
                // the pair vector in FP64 from the FP32 positions (exact), image by the FP64 box
                double ddx = (double)a.x - (double)pj.x, ddy = (double)a.y - (double)pj.y,
                       ddz = (double)a.z - (double)pj.z;
                if (MINIMG) {
                  ddx -= p.boxd[0] * rint(ddx / p.boxd[0]);
                  ddy -= p.boxd[1] * rint(ddy / p.boxd[1]);
                  ddz -= p.boxd[2] * rint(ddz / p.boxd[2]);
                } else {
                  ddx -= shx == 0.0f ? 0.0 : (shx > 0.0f ? p.boxd[0] : -p.boxd[0]);
                  ddy -= shy == 0.0f ? 0.0 : (shy > 0.0f ? p.boxd[1] : -p.boxd[1]);
                  ddz -= shz == 0.0f ? 0.0 : (shz > 0.0f ? p.boxd[2] : -p.boxd[2]);
                }
                const double r2 = ddx * ddx + ddy * ddy + ddz * ddz;
                float2 cc = make_float2(0.0f, 0.0f);
                if (vdw_on) cc = vdw_c6c12(sh_vdw, sh_itype[warp][il], sh_jtg[warp][t].x);
                double u_vdw, u_elec;
                const double g = pair_terms_f64(r2, kCcelec * (double)a.w * (double)pj.w, cc.x, cc.y, p, vdw_on,
                                                u_vdw, u_elec);
                const double fxd = g * ddx, fyd = g * ddy, fzd = g * ddz;
                gx = __double2ll_rn(fxd * 1099511627776.0);
                gy = __double2ll_rn(fyd * 1099511627776.0);
                gz = __double2ll_rn(fzd * 1099511627776.0);
                if (calc_energy) {
                  ev += __double2ll_rn(u_vdw * 4294967296.0);
                  ee += __double2ll_rn(u_elec * 4294967296.0);
                }
                if (calc_virial) {
                  w0 -= fxd * ddx; w1 -= fxd * ddy; w2 -= fxd * ddz;
                  w3 -= fyd * ddy; w4 -= fyd * ddz; w5 -= fzd * ddz;
                }
              }
              // segmented inclusive scan over runs of equal il (int64: exact), then one add per run
#pragma unroll
              for (int d = 1; d < 32; d <<= 1) {
                const int ku = __shfl_up_sync(0xffffffffu, il, d);
                const long long ux = __shfl_up_sync(0xffffffffu, gx, d);
                const long long uy = __shfl_up_sync(0xffffffffu, gy, d);
                const long long uz = __shfl_up_sync(0xffffffffu, gz, d);
                if (lane >= d && ku == il) { gx += ux; gy += uy; gz += uz; }
              }
              const int kn = __shfl_down_sync(0xffffffffu, il, 1);
              if (valid && (lane == 31 || kn != il)) {
                sh_f[warp][0][il] += gx;
                sh_f[warp][1][il] += gy;
                sh_f[warp][2][il] += gz;
              }
              __syncwarp();
            }
          }
        }
      }
      if (act) {
        const int a = ii.z;
        atomicAdd((unsigned long long*)&force[a], (unsigned long long)sh_f[warp][0][lane]);
        atomicAdd((unsigned long long*)&force[a + stride], (unsigned long long)sh_f[warp][1][lane]);
        atomicAdd((unsigned long long*)&force[a + 2 * (size_t)stride], (unsigned long long)sh_f[warp][2][lane]);
      }
      __syncwarp();
    }
    if (calc_virial) {
      wv[0] += __double2ll_rn(w0 * 4294967296.0); wv[1] += __double2ll_rn(w1 * 4294967296.0);
      wv[2] += __double2ll_rn(w2 * 4294967296.0); wv[3] += __double2ll_rn(w3 * 4294967296.0);
      wv[4] += __double2ll_rn(w4 * 4294967296.0); wv[5] += __double2ll_rn(w5 * 4294967296.0);
    }
  }
  if (calc_energy) {
    ev = warp_sum_ll(ev);
    ee = warp_sum_ll(ee);
    if (lane == 0) {
      atomicAdd((unsigned long long*)&acc[kAccVdw], (unsigned long long)ev);
      atomicAdd((unsigned long long*)&acc[kAccElec], (unsigned long long)ee);
    }
  }
  if (calc_virial) {
#pragma unroll
    for (int q = 0; q < 6; q++) {
      const long long sv = warp_sum_ll(wv[q]);
      if (lane == 0) atomicAdd((unsigned long long*)&acc[kAccVir + q], (unsigned long long)sv);
    }
  }
}

// 1-4 lists: one thread per (i, j, ishift, kind) entry, kind 1 = inclusion, 2 = exclusion.  Both
// atoms' forces by int64 atomics; energies and virial added twice (the doubled-sum convention).
__global__ void k_direct_14(const Params p, const int4* __restrict__ list, int nlist, const float4* __restrict__ xyzq,
                            const int* __restrict__ vdwtype, const float2* __restrict__ vdwp14, int calc_energy,
                            int calc_virial, int stride, long long* __restrict__ force, long long* __restrict__ acc) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  long long e[3] = {0, 0, 0};
  float w[6] = {0, 0, 0, 0, 0, 0};
  if (k < nlist) {
    const int4 L = list[k];
    const int i = L.x, j = L.y;
    const int ish = L.z;
    const float4 a = xyzq[i], b = xyzq[j];
    const float sx = (float)(ish % 3 - 1) * p.box[0];
    const float sy = (float)((ish / 3) % 3 - 1) * p.box[1];
    const float sz = (float)(ish / 9 - 1) * p.box[2];
    const float dx = a.x - b.x + sx, dy = a.y - b.y + sy, dz = a.z - b.z + sz;
    const float r2 = dx * dx + dy * dy + dz * dz;
    const bool in14 = L.w == 1;
    const bool vdw = in14 && p.vdw != PME_VDW_NONE;
    float2 cc = make_float2(0.0f, 0.0f);
    if (vdw) cc = vdw_c6c12(vdwp14, vdwtype[i], vdwtype[j]);
    float u_vdw, u_elec;
    const float g = pair_terms(r2, (float)kCcelec * a.w * b.w, cc.x, cc.y, p, in14 ? 1 : 2, vdw, u_vdw, u_elec);
    const long long fxi = __float2ll_rn(g * dx * kForceScaleF);
    const long long fyi = __float2ll_rn(g * dy * kForceScaleF);
    const long long fzi = __float2ll_rn(g * dz * kForceScaleF);
    atomicAdd((unsigned long long*)&force[i], (unsigned long long)fxi);
    atomicAdd((unsigned long long*)&force[i + stride], (unsigned long long)fyi);
    atomicAdd((unsigned long long*)&force[i + 2 * (size_t)stride], (unsigned long long)fzi);
    atomicAdd((unsigned long long*)&force[j], (unsigned long long)(-fxi));
    atomicAdd((unsigned long long*)&force[j + stride], (unsigned long long)(-fyi));
    atomicAdd((unsigned long long*)&force[j + 2 * (size_t)stride], (unsigned long long)(-fzi));
    if (calc_energy) {
      if (in14) {
        e[0] = 2 * __float2ll_rn(u_vdw * kEnergyScale);
        e[1] = 2 * __float2ll_rn(u_elec * kEnergyScale);
      } else {
        e[2] = 2 * __float2ll_rn(u_elec * kEnergyScale);
      }
    }
    if (calc_virial) {
      w[0] = -g * dx * dx; w[1] = -g * dx * dy; w[2] = -g * dx * dz;
      w[3] = -g * dy * dy; w[4] = -g * dy * dz; w[5] = -g * dz * dz;
    }
  }
  const int lane = threadIdx.x & 31;
  if (calc_energy) {
#pragma unroll
    for (int q = 0; q < 3; q++) {
      const long long s = warp_sum_ll(e[q]);
      if (lane == 0 && s != 0) atomicAdd((unsigned long long*)&acc[kAccVdw + q], (unsigned long long)s);
    }
  }
  if (calc_virial) {
#pragma unroll
    for (int q = 0; q < 6; q++) {
      const long long s = warp_sum_ll(2 * __float2ll_rn(w[q] * kEnergyScale));
      if (lane == 0 && s != 0) atomicAdd((unsigned long long*)&acc[kAccVir + q], (unsigned long long)s);
    }
  }
}

}  // namespace direct
}  // namespace pme

using namespace pme;
using namespace pme::direct;

struct pme_direct {
  int device = 0;
  cudaStream_t stream = nullptr;
  bool configured = false;
  double box[3] = {0, 0, 0};
  double kappa = 0, roff = 0, ron = 0, e14fac = 1.0;
  int vdw_model = PME_VDW_VSH, elec_model = PME_ELEC_EWALD;
  // tables
  int ntype = 0, ntype14 = 0, npair = 0, npair14 = 0;
  float2* d_vdw = nullptr;
  float2* d_vdw14 = nullptr;
  int n_types = 0;           // atoms of the vdW type table, and its largest type
  int max_type = -1;
  int n_excl = 0;            // atoms of the exclusion tables
  int* d_vdwtype = nullptr;
  int* d_glob = nullptr;     // global (original) index of every coordinate
  ulonglong2* d_win = nullptr;
  int* d_far_ptr = nullptr;
  int* d_far_idx = nullptr;
  bool excl_set = false;
  double4* d_tab = nullptr;  // Ewald real-space table for the current kappa and roff
  double tab_kappa = -1.0, tab_roff = -1.0;
  int4* d_list14 = nullptr;
  int n14 = 0;
  int max14 = -1;            // largest atom index in the 1-4 lists
  // per-call work space
  int cap_atoms = 0, cap_cells = 0;
  int* d_cell_of = nullptr;
  int* d_tmp = nullptr;
  int* d_count = nullptr;     // [cap_cells] counts, [cap_cells] fill counters, the pair-task counter
  int* d_start = nullptr;     // [cap_cells + 1]
  float4* d_pos = nullptr;
  int4* d_info = nullptr;
  ulonglong2* d_mask = nullptr;
  long long* d_acc = nullptr;  // kAccN
};

namespace {

int check_handle(const pme_direct* h) { return h ? PME_OK : fail(PME_EINVAL, "direct handle is NULL"); }

template <class T>
cudaError_t upload(T** dst, const T* src, size_t n, cudaStream_t s) {
  cudaError_t e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return e;
  if (*dst) cudaFree(*dst);
  *dst = nullptr;
  if (n == 0) return cudaSuccess;
  e = cudaMalloc(dst, n * sizeof(T));
  if (e == cudaSuccess) e = cudaMemcpy(*dst, src, n * sizeof(T), cudaMemcpyHostToDevice);
  return e;
}

Params make_params(const pme_direct* h) {
  Params p;
  std::memset(&p, 0, sizeof(p));
  for (int d = 0; d < 3; d++) {
    p.box[d] = (float)h->box[d];
    p.inv_box[d] = (float)(1.0 / h->box[d]);
  }
  p.kappa = (float)h->kappa;
  p.kappa2 = (float)(h->kappa * h->kappa);
  p.roff2 = (float)(h->roff * h->roff);
  p.ro6 = (float)std::pow(h->roff, -6.0);
  p.ro12 = (float)std::pow(h->roff, -12.0);
  p.ro18 = (float)std::pow(h->roff, -18.0);
  p.e14fac = (float)h->e14fac;
  p.vdw = h->vdw_model;
  p.elec = h->elec_model;
  // cells >= roff along x (offsets -1..1) and >= roff / 2 along y and z (offsets -2..2); an axis
  // with too few cells for distinct offsets visits each of its cells once
  const double size[3] = {h->roff * (1.0 + 1e-5), 0.5 * h->roff * (1.0 + 1e-5), 0.5 * h->roff * (1.0 + 1e-5)};
  const int reach[3] = {1, 2, 2};
  for (int d = 0; d < 3; d++) {
    p.nc[d] = std::max(1, (int)std::floor(h->box[d] / size[d]));
    if (p.nc[d] >= 2 * reach[d] + 1) {
      p.lo[d] = -reach[d];
      p.cnt[d] = 2 * reach[d] + 1;
    } else {
      p.lo[d] = 0;
      p.cnt[d] = p.nc[d];
    }
  }
  p.npair = h->npair;
  p.kappad = h->kappa;
  for (int d = 0; d < 3; d++) p.boxd[d] = h->box[d];
  p.tab = h->d_tab;
  p.tab_s0 = kTabR0 * kTabR0;
  p.tab_invh = kTabN / (h->roff * h->roff - p.tab_s0);
  p.tab_n = kTabN;
  p.ro6d = std::pow(h->roff, -6.0);
  p.ro12d = std::pow(h->roff, -12.0);
  p.ro18d = std::pow(h->roff, -18.0);
  return p;
}

// Hermite table of E(s) = erfc(kappa sqrt s) / sqrt s and F(s) = (r dE/dr) / r^2 (with r dE/dr =
// -2/sqrt(pi) kappa r exp(-kappa^2 s) - E... written per qq: the pair's r dU_elec/dr / r^2), values
// and h-scaled s-derivatives at kTabN + 1 nodes, built in FP64 on the host.  Cubic Hermite
// interpolation of these smooth functions at this spacing is within ~1e-9 relative.
int ensure_table(pme_direct* h) {
  if (h->elec_model == PME_ELEC_NONE) return PME_OK;
  if (h->d_tab && h->tab_kappa == h->kappa && h->tab_roff == h->roff) return PME_OK;
  cudaFree(h->d_tab);
  h->d_tab = nullptr;
  const double s0 = kTabR0 * kTabR0, s1 = h->roff * h->roff;
  if (!(s1 > s0)) return PME_OK;
  const double k = h->kappa, c1 = 2.0 / std::sqrt(kPi) * k, hs = (s1 - s0) / kTabN;
  std::vector<double4> t((size_t)kTabN + 1);
  for (int i = 0; i <= kTabN; i++) {
    const double sv = s0 + hs * i, r = std::sqrt(sv), ex = std::exp(-k * k * sv);
    const double E = std::erfc(k * r) / r;
    const double dEdr = (-c1 * ex * r - std::erfc(k * r)) / (r * r);
    const double dEds = dEdr / (2.0 * r);
    const double A = -c1 * ex - E;            // r dE/dr
    const double F = A / sv;
    const double dAds = c1 * k * k * ex - dEds;
    const double dFds = (dAds * sv - A) / (sv * sv);
    t[i] = make_double4(E, hs * dEds, F, hs * dFds);
  }
  cudaError_t e = upload(&h->d_tab, t.data(), t.size(), h->stream);
  if (e != cudaSuccess) return cuda_fail(e, "direct: Ewald table");
  h->tab_kappa = h->kappa;
  h->tab_roff = h->roff;
  return PME_OK;
}

int ensure_work(pme_direct* h, int n, int ncell) {
  if (n > h->cap_atoms) {
    cudaFree(h->d_cell_of); cudaFree(h->d_tmp); cudaFree(h->d_pos); cudaFree(h->d_info); cudaFree(h->d_mask);
    h->d_cell_of = h->d_tmp = nullptr; h->d_pos = nullptr; h->d_info = nullptr; h->d_mask = nullptr;
    h->cap_atoms = 0;
    const size_t m = (size_t)std::max(n, 1);
    if (cudaMalloc(&h->d_cell_of, m * sizeof(int)) != cudaSuccess || cudaMalloc(&h->d_tmp, m * sizeof(int)) != cudaSuccess ||
        cudaMalloc(&h->d_pos, m * sizeof(float4)) != cudaSuccess || cudaMalloc(&h->d_info, m * sizeof(int4)) != cudaSuccess ||
        cudaMalloc(&h->d_mask, m * sizeof(ulonglong2)) != cudaSuccess) {
      cudaGetLastError();
      return fail(PME_ENOMEM, "direct: atom work space");
    }
    h->cap_atoms = n;
  }
  if (ncell > h->cap_cells) {
    cudaFree(h->d_count); cudaFree(h->d_start);
    h->d_count = h->d_start = nullptr;
    h->cap_cells = 0;
    if (cudaMalloc(&h->d_count, (2 * (size_t)ncell + 1) * sizeof(int)) != cudaSuccess ||
        cudaMalloc(&h->d_start, 2 * ((size_t)ncell + 1) * sizeof(int)) != cudaSuccess) {
      cudaGetLastError();
      return fail(PME_ENOMEM, "direct: cell work space");
    }
    h->cap_cells = ncell;
  }
  return PME_OK;
}

// Exclusion windows of n atoms with no exclusions but themselves.
int self_exclusions(pme_direct* h, int n) {
  std::vector<ulonglong2> win((size_t)n, make_ulonglong2(0ull, 1ull));   // bit 64: offset 0
  std::vector<int> glob((size_t)n), ptr((size_t)n + 1, 0);
  for (int i = 0; i < n; i++) glob[i] = i;
  cudaError_t e = upload(&h->d_win, win.data(), win.size(), h->stream);
  if (e == cudaSuccess) e = upload(&h->d_glob, glob.data(), glob.size(), h->stream);
  if (e == cudaSuccess) e = upload(&h->d_far_ptr, ptr.data(), ptr.size(), h->stream);
  if (e == cudaSuccess) e = upload(&h->d_far_idx, (const int*)nullptr, 0, h->stream);
  return e == cudaSuccess ? PME_OK : cuda_fail(e, "direct: exclusions");
}

int upload_vdw(pme_direct* h, int nvdwparam, const float* hp, bool in14) {
  if (int rc = check_handle(h)) return rc;
  if (nvdwparam < 2 || (nvdwparam & 1) || !hp) return fail(PME_EINVAL, "vdwparam: need (c6, c12) pairs");
  const int npair = nvdwparam / 2;
  int ntype = 0;
  while ((ntype + 1) * (ntype + 2) / 2 <= npair) ntype++;
  if (ntype * (ntype + 1) / 2 != npair) return fail(PME_EINVAL, "vdwparam: not a packed lower triangle of types");
  if (ntype > kMaxTypes) return fail(PME_EUNSUPPORTED, "vdwparam: more than 200 vdW types");
  std::vector<float2> t((size_t)npair);
  for (int k = 0; k < npair; k++) t[k] = make_float2(6.0f * hp[2 * k], 12.0f * hp[2 * k + 1]);
  DeviceGuard dg(h->device);
  cudaError_t e = upload(in14 ? &h->d_vdw14 : &h->d_vdw, t.data(), t.size(), h->stream);
  if (e != cudaSuccess) return cuda_fail(e, "vdwparam: upload");
  if (in14) { h->npair14 = npair; h->ntype14 = ntype; }
  else { h->npair = npair; h->ntype = ntype; }
  return PME_OK;
}

}  // namespace

extern "C" {

int pme_direct_create(void* stream, pme_direct** out) {
  if (!out) return fail(PME_EINVAL, "out is NULL");
  *out = nullptr;
  pme_direct* h = new (std::nothrow) pme_direct();
  if (!h) return fail(PME_ENOMEM, "host allocation failed");
  cudaError_t e = cudaGetDevice(&h->device);
  h->stream = (cudaStream_t)stream;
  if (e == cudaSuccess && cudaMalloc(&h->d_acc, kAccN * sizeof(long long)) != cudaSuccess) e = cudaErrorMemoryAllocation;
  if (e == cudaSuccess) e = cudaMemset(h->d_acc, 0, kAccN * sizeof(long long));
  if (e != cudaSuccess) {
    cudaGetLastError();
    cudaFree(h->d_acc);
    delete h;
    return cuda_fail(e, "direct: create");
  }
  *out = h;
  return PME_OK;
}

int pme_direct_destroy(pme_direct* h) {
  if (!h) return PME_OK;
  DeviceGuard dg(h->device);
  cudaStreamSynchronize(h->stream);
  for (void* p : {(void*)h->d_vdw, (void*)h->d_vdw14, (void*)h->d_vdwtype, (void*)h->d_glob, (void*)h->d_win,
                  (void*)h->d_far_ptr, (void*)h->d_far_idx, (void*)h->d_list14, (void*)h->d_tab, (void*)h->d_cell_of, (void*)h->d_tmp,
                  (void*)h->d_count, (void*)h->d_start, (void*)h->d_pos, (void*)h->d_info, (void*)h->d_mask,
                  (void*)h->d_acc})
    if (p) cudaFree(p);
  delete h;
  return PME_OK;
}

int pme_direct_set_stream(pme_direct* h, void* stream) {
  if (int rc = check_handle(h)) return rc;
  h->stream = (cudaStream_t)stream;
  return PME_OK;
}

int pme_direct_setup(pme_direct* h, double boxx, double boxy, double boxz, double kappa, double roff,
                     double ron, double e14fac, int vdw_model, int elec_model) {
  if (int rc = check_handle(h)) return rc;
  if (vdw_model != PME_VDW_VSH && vdw_model != PME_VDW_NONE)
    return fail(PME_EUNSUPPORTED, "direct: only the VDW_VSH (and NONE) vdW model is built");
  if (elec_model != PME_ELEC_EWALD && elec_model != PME_ELEC_NONE)
    return fail(PME_EUNSUPPORTED, "direct: only the EWALD (and NONE) electrostatics model is built");
  if (!(kappa >= 0.0) || !std::isfinite(kappa) || !std::isfinite(e14fac) || !std::isfinite(ron))
    return fail(PME_EINVAL, "direct: kappa, ron and e14fac must be finite (kappa >= 0)");
  h->kappa = kappa;
  h->roff = roff;
  h->ron = ron;
  h->e14fac = e14fac;
  h->vdw_model = vdw_model;
  h->elec_model = elec_model;
  h->configured = false;
  if (int rc = pme_direct_set_box_size(h, boxx, boxy, boxz)) return rc;
  h->configured = true;
  return PME_OK;
}

int pme_direct_set_box_size(pme_direct* h, double boxx, double boxy, double boxz) {
  if (int rc = check_handle(h)) return rc;
  const double b[3] = {boxx, boxy, boxz};
  for (double v : b)
    if (!(v > 0.0) || !std::isfinite(v)) return fail(PME_EINVAL, "direct: box edges must be finite and positive");
  if (!(h->roff > 0.0) || 2.0 * h->roff > std::min(boxx, std::min(boxy, boxz)))
    return fail(PME_EINVAL, "direct: roff must be positive and at most half the shortest box edge");
  for (int d = 0; d < 3; d++) h->box[d] = b[d];
  return PME_OK;
}

int pme_direct_set_vdwparam(pme_direct* h, int nvdwparam, const float* hp) { return upload_vdw(h, nvdwparam, hp, false); }
int pme_direct_set_vdwparam14(pme_direct* h, int nvdwparam, const float* hp) { return upload_vdw(h, nvdwparam, hp, true); }

int pme_direct_set_vdwtype(pme_direct* h, int ncoord, const int* hv) {
  if (int rc = check_handle(h)) return rc;
  if (ncoord < 0 || (ncoord > 0 && !hv)) return fail(PME_EINVAL, "vdwtype: bad arguments");
  int mx = -1;
  for (int i = 0; i < ncoord; i++) {
    if (hv[i] < 0) return fail(PME_EINVAL, "vdwtype: negative type");
    mx = std::max(mx, hv[i]);
  }
  DeviceGuard dg(h->device);
  cudaError_t e = upload(&h->d_vdwtype, hv, (size_t)ncoord, h->stream);
  if (e != cudaSuccess) return cuda_fail(e, "vdwtype: upload");
  h->n_types = ncoord;
  h->max_type = mx;
  return PME_OK;
}

int pme_direct_set_exclusions(pme_direct* h, int ncoord, const int* iblo14, const int* inb14, const int* loc2glo) {
  if (int rc = check_handle(h)) return rc;
  if (ncoord < 0 || (ncoord > 0 && !iblo14)) return fail(PME_EINVAL, "exclusions: bad arguments");
  const int n = ncoord;
  std::vector<int> glob((size_t)n), glo2loc((size_t)n, -1);
  for (int i = 0; i < n; i++) {
    const int g = loc2glo ? loc2glo[i] : i;
    if (g < 0 || g >= n || glo2loc[g] >= 0) return fail(PME_EINVAL, "exclusions: loc2glo is not a permutation");
    glob[i] = g;
    glo2loc[g] = i;
  }
  std::vector<ulonglong2> win((size_t)n, make_ulonglong2(0ull, 1ull));   // bit 64: the atom itself
  std::vector<std::vector<int>> far((size_t)n);
  auto add = [&](int ga, int gb) {   // exclude gb from ga's list (global indices)
    const int i = glo2loc[ga];
    const int k = gb - ga + 64;
    if (k >= 0 && k < 128) {
      if (k < 64) win[i].x |= 1ull << k;
      else win[i].y |= 1ull << (k - 64);
    } else {
      far[i].push_back(gb);
    }
  };
  int prev = 0;
  for (int ga = 0; ga < n; ga++) {
    const int end = iblo14[ga];
    if (end < prev || (end > prev && !inb14)) return fail(PME_EINVAL, "exclusions: iblo14 must be non-decreasing");
    for (int k = prev; k < end; k++) {
      const int gb = std::abs(inb14[k]) - 1;
      if (gb < 0 || gb >= n) return fail(PME_EINVAL, "exclusions: inb14 entry out of range");
      add(ga, gb);
      add(gb, ga);
    }
    prev = end;
  }
  std::vector<int> ptr((size_t)n + 1, 0), idx;
  for (int i = 0; i < n; i++) {
    std::sort(far[i].begin(), far[i].end());
    far[i].erase(std::unique(far[i].begin(), far[i].end()), far[i].end());
    ptr[i + 1] = ptr[i] + (int)far[i].size();
    idx.insert(idx.end(), far[i].begin(), far[i].end());
  }
  DeviceGuard dg(h->device);
  cudaError_t e = upload(&h->d_win, win.data(), win.size(), h->stream);
  if (e == cudaSuccess) e = upload(&h->d_glob, glob.data(), glob.size(), h->stream);
  if (e == cudaSuccess) e = upload(&h->d_far_ptr, ptr.data(), ptr.size(), h->stream);
  if (e == cudaSuccess) e = upload(&h->d_far_idx, idx.data(), idx.size(), h->stream);
  if (e != cudaSuccess) return cuda_fail(e, "exclusions: upload");
  h->excl_set = true;
  h->n_excl = n;
  return PME_OK;
}

int pme_direct_set_14_list(pme_direct* h, int nin14, int nex14, const int* in14, const int* ex14) {
  if (int rc = check_handle(h)) return rc;
  if (nin14 < 0 || nex14 < 0 || (nin14 > 0 && !in14) || (nex14 > 0 && !ex14)) return fail(PME_EINVAL, "14 list: bad arguments");
  std::vector<int4> L;
  L.reserve((size_t)nin14 + nex14);
  int mx = -1;
  for (int pass = 0; pass < 2; pass++) {
    const int* s = pass == 0 ? in14 : ex14;
    const int n = pass == 0 ? nin14 : nex14;
    for (int k = 0; k < n; k++) {
      const int i = s[3 * k], j = s[3 * k + 1], ish = s[3 * k + 2];
      if (i < 0 || j < 0 || ish < 0 || ish > 26) return fail(PME_EINVAL, "14 list: bad entry");
      L.push_back(make_int4(i, j, ish, pass + 1));
      mx = std::max(mx, std::max(i, j));
    }
  }
  DeviceGuard dg(h->device);
  cudaError_t e = upload(&h->d_list14, L.data(), L.size(), h->stream);
  if (e != cudaSuccess) return cuda_fail(e, "14 list: upload");
  h->n14 = (int)L.size();
  h->max14 = mx;
  return PME_OK;
}

int pme_direct_calc_force(pme_direct* h, const void* xyzq, int ncoord, int calc_energy, int calc_virial, int stride,
                          long long* force) {
  if (int rc = check_handle(h)) return rc;
  if (!h->configured) return fail(PME_ESTATE, "direct: setup first");
  if (ncoord < 0 || (ncoord > 0 && (!xyzq || !force)) || stride < ncoord) return fail(PME_EINVAL, "direct: bad arguments");
  if (ncoord == 0) return PME_OK;
  if (h->vdw_model != PME_VDW_NONE) {
    if (!h->d_vdw || !h->d_vdwtype) return fail(PME_ESTATE, "direct: set vdwparam and vdwtype first");
    if (h->n_types != ncoord) return fail(PME_EINVAL, "direct: ncoord differs from the vdW types' count");
    if (h->max_type >= h->ntype) return fail(PME_EINVAL, "direct: a vdW type is beyond the parameter table");
  }
  if (h->excl_set && h->n_excl != ncoord) return fail(PME_EINVAL, "direct: ncoord differs from the exclusions' count");
  DeviceGuard dg(h->device);
  if (!h->excl_set) {   // no exclusion lists: every atom excludes only itself
    if (int rc = self_exclusions(h, ncoord)) return rc;
    h->excl_set = true;
    h->n_excl = ncoord;
  }
  if (h->n_types != ncoord) {   // no vdW: every atom type 0
    std::vector<int> zeros((size_t)ncoord, 0);
    cudaError_t e = upload(&h->d_vdwtype, zeros.data(), zeros.size(), h->stream);
    if (e != cudaSuccess) return cuda_fail(e, "direct: types");
    h->n_types = ncoord;
    h->max_type = 0;
  }
  if (int rc = ensure_table(h)) return rc;
  Params p = make_params(h);
  if (h->vdw_model == PME_VDW_NONE) p.npair = 0;
  const int ncell = p.nc[0] * p.nc[1] * p.nc[2];
  if (int rc = ensure_work(h, ncoord, ncell)) return rc;
  cudaStream_t s = h->stream;
  cudaError_t e = cudaMemsetAsync(h->d_count, 0, (2 * (size_t)ncell + 1) * sizeof(int), s);   // + task counter
  if (e != cudaSuccess) return cuda_fail(e, "direct: clear counts");
  const int nb = (ncoord + 255) / 256;
  k_direct_cell<<<nb, 256, 0, s>>>((const float4*)xyzq, ncoord, p, h->d_cell_of, h->d_count);
  k_direct_scan<<<1, 1024, 0, s>>>(h->d_count, ncell, h->d_start, h->d_start + ncell + 1);
  k_direct_fill<<<nb, 256, 0, s>>>(h->d_cell_of, ncoord, h->d_start, h->d_count + ncell, h->d_tmp);
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, h->device);
  const int og = std::min((ncell + 7) / 8, sms * 16);
  k_direct_order<<<og, 256, 0, s>>>(h->d_start, ncell, h->d_tmp, (const float4*)xyzq, h->d_vdwtype, h->d_glob,
                                    h->d_win, h->d_far_ptr, p.box[0], p.box[1], p.box[2], p.inv_box[0],
                                    p.inv_box[1], p.inv_box[2], h->d_pos, h->d_info, h->d_mask);
  // neighbour cells by periodic shift when every axis has distinct offsets, else minimum image
  const bool minimg = p.cnt[0] == p.nc[0] || p.cnt[1] == p.nc[1] || p.cnt[2] == p.nc[2];
  auto kern = minimg ? k_direct_pairs<true> : k_direct_pairs<false>;
  const size_t smem = (size_t)std::max(p.npair, 1) * sizeof(float2);
  e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)std::max<size_t>(smem, 48 * 1024));
  if (e != cudaSuccess) return cuda_fail(e, "direct: shared memory");
  // chunks are counted on the device: enough CTAs for every (chunk, z slice) task of a uniform
  // system, each warp striding over the rest
  // one wave of resident CTAs; their warps draw the (chunk, z slice) tasks from a counter
  int occ = 1;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, kWarps * 32, smem);
  if (e != cudaSuccess) return cuda_fail(e, "direct: occupancy");
  const long long tasks = (long long)((ncoord + 31) / 32 + ncell) * p.cnt[2];
  const int pg = (int)std::max<long long>(1, std::min<long long>((tasks + kWarps - 1) / kWarps,
                                                                 (long long)sms * std::max(occ, 1)));
  kern<<<pg, kWarps * 32, smem, s>>>(p, h->d_start, h->d_start + ncell + 1, h->d_pos, h->d_info, h->d_mask,
                                     h->d_far_ptr, h->d_far_idx, h->d_vdw, calc_energy ? 1 : 0, calc_virial ? 1 : 0,
                                     stride, force, h->d_acc, h->d_count + 2 * ncell);
  e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "direct: launch");
  return PME_OK;
}

int pme_direct_calc_14_force(pme_direct* h, const void* xyzq, int calc_energy, int calc_virial, int stride,
                             long long* force) {
  if (int rc = check_handle(h)) return rc;
  if (!h->configured) return fail(PME_ESTATE, "direct: setup first");
  if (h->n14 == 0) return PME_OK;
  if (!xyzq || !force || stride < 1) return fail(PME_EINVAL, "direct 14: bad arguments");
  if (h->max14 >= stride) return fail(PME_EINVAL, "direct 14: a list entry is beyond the force stride");
  if (h->max14 >= std::max(h->n_types, h->n_excl))
    return fail(PME_EINVAL, "direct 14: a list entry is beyond the atoms (set vdwtype or exclusions first)");
  if (h->vdw_model != PME_VDW_NONE) {
    if (!h->d_vdw14 || !h->d_vdwtype) return fail(PME_ESTATE, "direct 14: set vdwparam14 and vdwtype first");
    if (h->max14 >= h->n_types) return fail(PME_EINVAL, "direct 14: a list entry is beyond the vdW types");
    if (h->max_type >= h->ntype14) return fail(PME_EINVAL, "direct 14: a vdW type is beyond the 1-4 table");
  }
  DeviceGuard dg(h->device);
  const Params p = make_params(h);
  k_direct_14<<<(h->n14 + 255) / 256, 256, 0, h->stream>>>(p, h->d_list14, h->n14, (const float4*)xyzq, h->d_vdwtype,
                                                           h->d_vdw14, calc_energy ? 1 : 0, calc_virial ? 1 : 0,
                                                           stride, force, h->d_acc);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "direct 14: launch");
  return PME_OK;
}

int pme_direct_clear_energy_virial(pme_direct* h) {
  if (int rc = check_handle(h)) return rc;
  DeviceGuard dg(h->device);
  cudaError_t e = cudaMemsetAsync(h->d_acc, 0, kAccN * sizeof(long long), h->stream);
  return e == cudaSuccess ? PME_OK : cuda_fail(e, "direct: clear");
}

int pme_direct_get_energy_virial(pme_direct* h, double* e_vdw, double* e_elec, double* e_excl, double* vir9) {
  if (int rc = check_handle(h)) return rc;
  DeviceGuard dg(h->device);
  long long a[kAccN];
  cudaError_t e = cudaStreamSynchronize(h->stream);
  if (e == cudaSuccess) e = cudaMemcpy(a, h->d_acc, sizeof(a), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return cuda_fail(e, "direct: read energies");
  const double sc = 0.5 / 4294967296.0;   // doubled sums at 2^32
  if (e_vdw) *e_vdw = (double)a[kAccVdw] * sc;
  if (e_elec) *e_elec = (double)a[kAccElec] * sc;
  if (e_excl) *e_excl = (double)a[kAccExcl] * sc;
  if (vir9) {
    const double w[6] = {(double)a[3] * sc, (double)a[4] * sc, (double)a[5] * sc,
                         (double)a[6] * sc, (double)a[7] * sc, (double)a[8] * sc};
    const double t[9] = {w[0], w[1], w[2], w[1], w[3], w[4], w[2], w[4], w[5]};
    for (int k = 0; k < 9; k++) vir9[k] = t[k];
  }
  return PME_OK;
}

}  // extern "C"

// pme_kernels.cu -- sm_100a kernels of the smooth-PME reciprocal path.
//
// Two forms over the same tile functions (pme_tiles.cuh):
//  * staged kernels, one tile per CTA, one launch per reference stage (spread_charge, r2c_fft,
//    scalar_sum, c2r_fft, gather_force, calc_self_energy of CudaPMERecip.cu);
//  * the persistent fused kernel: one cooperative launch runs every phase of every system of a
//    batch, with bounded grid barriers between non-empty phases:
//      0 bin atoms by row block (records, sum q^2, max |q|) and the FP64 influence tables
//                                                                    (:479-580, :1252-1275)
//      1 spread into one row block in shared memory, x forward       (cuFFT R2C :2421)
//      2 y forward, or whole kx planes: y, z, solve, z and y inverse (:594-901)
//      3 z forward + solve with energy/virial + z inverse (no planes)
//      4 y inverse (no planes)
//      5 x inverse (C2R) and the energy/virial finalisation          (cuFFT C2R :2464)
//      6 gather by bin, writing the bin-sorted atom order            (:1031-1245)
//    It is compiled three times (latency, throughput and cluster builds, see k_fused_lat /
//    k_fused_tput / k_fused_cl); the cluster build runs phases 2-4 as one phase of cluster plane tiles.
// Both forms execute the same per-element arithmetic, so forces and energies agree bit for bit.
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <cstring>
#include <map>
#include <mutex>
#include <utility>

#include "pme_internal.h"
#include "pme_tiles.cuh"

namespace pme {

// Copy a descriptor (kernel parameter or global table entry) into shared memory.
// Copy a kernel's SysDesc parameter (a __grid_constant__, read in place from the parameter space)
// into shared memory, one word per thread.
__device__ __forceinline__ void load_desc(SysDesc& dst, const SysDesc& src_param) {
  const int n = (int)(sizeof(SysDesc) / sizeof(int));
  const int* s = reinterpret_cast<const int*>(&src_param);
  int* t = reinterpret_cast<int*>(&dst);
  for (int i = threadIdx.x; i < n; i += blockDim.x) t[i] = s[i];
  __syncthreads();
}

__device__ __forceinline__ void load_desc_global(SysDesc& dst, const SysDesc* src) {
  const int n = (int)(sizeof(SysDesc) / sizeof(int));
  const int* s = (const int*)src;
  int* t = (int*)&dst;
  for (int i = threadIdx.x; i < n; i += blockDim.x) t[i] = __ldg(&s[i]);
  __syncthreads();
}

// ------------------------------- staged kernels ----------------------------------------------
__global__ void __launch_bounds__(kThreads) k_spread(const __grid_constant__ SysDesc p) {
  __shared__ SysDesc d;
  extern __shared__ float2 smem[];
  load_desc(d, p);
  spread_dispatch(d, blockIdx.x, smem);
}

__global__ void __launch_bounds__(kThreads) k_gather(const __grid_constant__ SysDesc p) {
  __shared__ SysDesc d;
  load_desc(d, p);
  gather_dispatch(d, blockIdx.x);
}

// ------------------------------- fused persistent kernel --------------------------------------
// Grid barrier: arrival counter + generation word.  Waits are bounded: after spin_limit polls
// the CTA records kStatusBarrierTimeout in *status and the kernel returns (no trap, no hang).
__device__ __forceinline__ unsigned int ld_acquire(const unsigned int* p) {
  unsigned int v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ int ld_volatile(const int* p) { return *(const volatile int*)p; }

__device__ __forceinline__ unsigned long long globaltimer() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ void trace_mark(const FusedArgs& a, int ph, int which) {
  if (a.trace != nullptr && threadIdx.x == 0 && (int)blockIdx.x < a.trace_ctas)
    a.trace[((size_t)blockIdx.x * kPhases + ph) * 2 + which] = globaltimer();
}

__device__ __forceinline__ unsigned long long ld_acquire_u64(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ unsigned long long ld_relaxed_u64(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ void fence_acq_rel_gpu() { asm volatile("fence.acq_rel.gpu;" ::: "memory"); }

__device__ __forceinline__ void red_release_add_u64(unsigned long long* p, unsigned long long v) {
  asm volatile("red.release.gpu.global.add.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

// Grid barrier k of a launch: a monotonic 64-bit arrival counter.  Every CTA adds 1 with release
// semantics and waits (acquire) until the counter reaches base + (k+1) * gridDim.x, where base is
// the counter value at launch start (bar[1], advanced once per launch by CTA 0 after barrier 0,
// when every CTA has read it).  Waits are bounded: after spin_limit polls the CTA records
// kStatusBarrierTimeout in *status and the kernel returns (no trap, no hang).
__device__ bool grid_barrier(unsigned long long* bar, unsigned long long base, int k, int nbar,
                             int* status, unsigned int spin_limit, bool bump_parity = true) {
  __shared__ int ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    const unsigned long long target = base + (unsigned long long)(k + 1) * gridDim.x;
    red_release_add_u64(&bar[0], 1ull);
    int good = 1;
    unsigned int it = 0;
    // relaxed polls, then one acquire fence once the count is reached (the acquire pattern); the
    // status word (another CTA gave up) is looked at every 64 polls
    while (ld_relaxed_u64(&bar[0]) < target) {
      ++it;
      if (it > spin_limit || ((it & 63u) == 0u && ld_volatile(status) != 0)) {
        atomicCAS(status, 0, kStatusBarrierTimeout);
        good = 0;
        break;
      }
      if (it > 64) __nanosleep(32);
    }
    fence_acq_rel_gpu();
    if (good && k == 0 && blockIdx.x == 0) {
      bar[1] = base + (unsigned long long)nbar * gridDim.x;
      // launch counter (bin parity), advanced by the launches that bin atoms; every CTA read it
      // before barrier 0
      if (bump_parity) bar[3] = bar[3] + 1ull;
    }
    ok = good;
  }
  __syncthreads();
  return ok != 0;
}

__device__ __forceinline__ int find_system(const int* prefix, int nsys, int t) {
  int lo = 0, hi = nsys - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (__ldg(&prefix[mid]) <= t) lo = mid; else hi = mid - 1;
  }
  return lo;
}

// The fused evaluation's body; compiled three times (see k_fused_lat / k_fused_tput / k_fused_cl
// below).  CL: the build with the cluster plane tiles, launched with 4-CTA clusters.
template <bool LAT, bool CL = false>
__device__ __forceinline__ void fused_body(const FusedArgs& a) {
  __shared__ SysDesc d;
  __shared__ int cur;
  extern __shared__ float2 smem[];
  __shared__ unsigned long long base;
  __shared__ int parity;
  if (threadIdx.x == 0) {
    cur = -1;
    base = ld_acquire_u64(&a.bar[1]);
    parity = (int)(ld_acquire_u64(&a.bar[3]) & 1ull);
  }
  // a sticky error from an earlier interrupted evaluation: do nothing until the host clears it
  if (ld_volatile(a.status) != kStatusOk) return;
  if (a.table == nullptr) load_desc(d, a.single);
  __syncthreads();
  int k = 0;   // barriers passed
  for (int ph = 0; ph < kPhases; ph++) {
    if (a.total[ph] == 0) continue;
    const int* prefix = a.prefix ? a.prefix + ph * (a.nsys + 1) : nullptr;
    trace_mark(a, ph, 0);
    for (int t = blockIdx.x; t < a.total[ph]; t += gridDim.x) {
      int local = t;
      if (a.table != nullptr) {
        const int s = find_system(prefix, a.nsys, t);
        local = t - __ldg(&prefix[s]);
        if (s != cur) {
          __syncthreads();
          load_desc_global(d, a.table + s);
          if (threadIdx.x == 0) cur = s;
        }
      }
      switch (ph) {
        case 0:
          if (local < tiles_bin(d)) bin_tile(d, local, parity, (long long*)smem);
          else ktab_tile(d);
          break;
        case 1: spread_x_dispatch(d, local, parity, (char*)smem); break;
        case 2:
          if (CL && d.cplane) cplane_tile<kClusterPlane>(d, local, smem);
          else if (d.plane) plane_tile(d, local, smem);
          else y_tile(d, 0, local, smem);
          break;
        case 3: z_tile(d, 2, local, smem); break;
        case 4: y_tile(d, 1, local, smem); break;
        case 5:
          if (local < tiles_xpass(d)) x_inv_tile(d, local, smem);
          else if (threadIdx.x == 0) finalize_system(d, true, true);
          break;
        default:
          // with the inverse x pass in the gather tiles, the record is finalised by one extra tile here
          // (only the latency build has the fused variant; the host never gives gx to the other)
          if (LAT && d.gx) {
            if (local == tiles_blocks(d)) {
              if (threadIdx.x == 0) finalize_system(d, true, true);
            } else {
              gather_bin_order<true>(d, local, parity, (char*)smem);
            }
          } else if (!LAT && d.gsort) {
            // (throughput build only: large bins come with launches of many tiles per CTA)
            gather_bin_order<false, true>(d, local, parity, (char*)smem);
          } else {
            gather_bin_order<false>(d, local, parity, (char*)smem);
          }
          break;
      }
      __syncthreads();
    }
    trace_mark(a, ph, 1);
    if (a.inject == 1 && k == 0 && blockIdx.x == 0) return;
    if (k < a.nbar) {
      if (!grid_barrier(a.bar, base, k, a.nbar, a.status, a.spin_limit)) return;
      k++;
    }
  }
}

// Latency build: up to 128 registers, 2 CTAs of 256 threads per SM; for launches with about one
// tile per CTA in a phase.  Throughput build: at most 80 registers, 3 CTAs per SM (a few spills in
// the largest tiles); for launches with many tiles per CTA, where the extra resident warps hide
// more latency than the spills cost.
__global__ void __launch_bounds__(kThreads) k_fused_lat(const __grid_constant__ FusedArgs a) { fused_body<true>(a); }
__global__ void __launch_bounds__(kThreads, 3) k_fused_tput(const __grid_constant__ FusedArgs a) { fused_body<false>(a); }
// Cluster build: the latency build with the cluster plane tiles, only ever launched with clusters of
// kClusterPlane CTAs (kept apart so that the other launches run the latency build without the
// cluster code: compiled into one kernel, it made their evaluations 2-4 us slower).
__global__ void __launch_bounds__(kThreads) k_fused_cl(const __grid_constant__ FusedArgs a) { fused_body<true, true>(a); }

// ------------------------------- staged cooperative kernel -----------------------------------
// One reference-interface call (r2c_fft, scalar_sum, c2r_fft) as one cooperative launch over the
// same tile functions as the fused evaluation, with bounded grid barriers between its phases:
// one launch per call instead of three, the same arithmetic (so the same bits).  The launches do
// not bin atoms, so they leave the bin parity of the fused evaluations alone.
__global__ void __launch_bounds__(kThreads, 2) k_staged(const __grid_constant__ StagedArgs a) {
  __shared__ SysDesc d;
  extern __shared__ float2 smem[];
  __shared__ unsigned long long base;
  if (threadIdx.x == 0) base = ld_acquire_u64(&a.bar[1]);
  if (ld_volatile(a.status) != kStatusOk) return;
  load_desc(d, a.d);
  const int nbar = a.nphase - 1;
  for (int ph = 0; ph < a.nphase; ph++) {
    for (int t = blockIdx.x; t < a.total[ph]; t += gridDim.x) {
      switch (a.kind[ph]) {
        case kStgXFwdZero: x_fwd_tile(d, t, smem, true); break;
        case kStgYFwd: y_tile(d, 0, t, smem); break;
        case kStgZFwd: z_tile(d, 0, t, smem); break;
        case kStgZSolve: z_tile(d, 3, t, smem); break;
        case kStgZInv: z_tile(d, 1, t, smem); break;
        case kStgYInv: y_tile(d, 1, t, smem); break;
        default: x_inv_tile(d, t, smem); break;
      }
      __syncthreads();
    }
    if (ph < nbar && !grid_barrier(a.bar, base, ph, nbar, a.status, a.spin_limit, false)) return;
  }
  if (a.ticket != nullptr) {
    // the energy/virial sums of every CTA are in the accumulators once all have taken a ticket
    __shared__ bool last;
    __syncthreads();
    if (threadIdx.x == 0) {
      __threadfence();
      last = atomicAdd(a.ticket, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (last && threadIdx.x == 0) {
      __threadfence();
      finalize_system(d, true, false);
      *a.ticket = 0u;
    }
  }
}

// Self energy in one launch: per-CTA sums of q^2 (fixed point) into the accumulator; the last CTA
// to finish (ticket of an arrival counter) converts it into the record and re-arms the counter.
__global__ void __launch_bounds__(kThreads) k_self_energy(const __grid_constant__ SysDesc p, unsigned int* done) {
  __shared__ long long red[32];
  __shared__ bool last;
  long long q2 = 0;
  for (int i = blockIdx.x * kThreads + threadIdx.x; i < p.natom; i += gridDim.x * kThreads)
    q2 += q2_fixed(__ldg(&p.xyzq[i]).w);
  const long long sum = block_sum_ll(q2, red);
  if (threadIdx.x == 0) {
    if (sum != 0) atomicAdd((unsigned long long*)&p.acc[kAccQ2], (unsigned long long)sum);
    __threadfence();
    last = atomicAdd(done, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (last && threadIdx.x == 0) {
    __threadfence();
    finalize_system(p, false, true);
    *done = 0u;
  }
}

// Energy/virial records of every system of a batch set to zero in one launch (a memset per
// system would cost one operation each).
__global__ void k_clear_records(const SysDesc* __restrict__ table, int nsys) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int sys = i / kEvCount, slot = i - sys * kEvCount;
  if (sys < nsys) table[sys].ev[slot] = 0.0;
}

// ------------------------------- host launchers ----------------------------------------------
static size_t staged_fft_smem(int L, int tx) { return tile_smem_bytes(L, tx) + 32 * 7 * sizeof(long long); }
// z tiles also stage the y and z influence tables
static size_t staged_z_smem(const SysDesc& d) {
  return staged_fft_smem(d.g.nz, d.tx_z) + ktab_smem_bytes(d.g.ny, d.g.nz);
}

size_t spread_smem(int order) {
  switch (order) {
    case 4: return spread_smem_bytes<4>();
    case 6: return spread_smem_bytes<6>();
    default: return spread_smem_bytes<8>();
  }
}

size_t fused_smem_bytes(const SysDesc& d) {
  size_t m = 32 * sizeof(long long);
  size_t c[6] = {staged_fft_smem(d.g.nx, d.tx_rows), staged_fft_smem(d.g.ny, d.tx_y),
                 staged_z_smem(d), d.plane ? plane_smem_bytes(d.g.ny, d.g.nz) : 0,
                 spread_x_smem_bytes(d.g.nx, d.bry * d.brz, d.order),
                 d.cplane ? cplane_smem_bytes(d.g.ny, d.g.nz, d.cplane) : 0};
  for (size_t v : c) m = m > v ? m : v;
  if (d.gx) {
    const size_t v = gx_smem_bytes(d.g.nx, d.bry, d.brz, d.order);
    m = m > v ? m : v;
  }
  return m;
}

void fused_tile_counts(const SysDesc& d, int* counts) {
  counts[0] = tiles_bin(d) + 1;
  counts[1] = tiles_blocks(d);
  counts[2] = d.cplane ? tiles_plane(d) * d.cplane : (d.plane ? tiles_plane(d) : tiles_ypass(d));
  counts[3] = (d.plane || d.cplane) ? 0 : tiles_zpass(d);
  counts[4] = (d.plane || d.cplane) ? 0 : tiles_ypass(d);
  counts[5] = d.gx ? 0 : tiles_xpass(d) + 1;
  counts[6] = tiles_blocks(d) + (d.gx ? 1 : 0);
}

int fused_barriers(const int* total) {
  int nonempty = 0;
  for (int p = 0; p < kPhases; p++) nonempty += total[p] > 0 ? 1 : 0;
  return nonempty > 0 ? nonempty - 1 : 0;
}

cudaError_t staged_spread(const SysDesc& d, cudaStream_t s) {
  const int blocks = tiles_spread(d);
  if (blocks <= 0) return cudaSuccess;
  k_spread<<<blocks, kThreads, spread_smem(d.order), s>>>(d);
  return cudaGetLastError();
}

cudaError_t staged_self(const SysDesc& d, unsigned int* done, cudaStream_t s) {
  // one charge per thread up to 1184 CTAs: the sum is latency-bound (24,000 charges: 24 CTAs of
  // four loads per thread took 6.2 us with caches cold)
  int blocks = (d.natom + kThreads - 1) / kThreads;
  blocks = blocks < 1 ? 1 : (blocks > 1184 ? 1184 : blocks);
  k_self_energy<<<blocks, kThreads, 0, s>>>(d, done);
  return cudaGetLastError();
}

// Shared memory of a staged phase.
static size_t staged_phase_smem(const SysDesc& d, int kind) {
  switch (kind) {
    case kStgXFwdZero: case kStgXInv: return staged_fft_smem(d.g.nx, d.tx_rows);
    case kStgYFwd: case kStgYInv: return staged_fft_smem(d.g.ny, d.tx_y);
    case kStgZFwd: case kStgZSolve: case kStgZInv: return staged_z_smem(d);
    default: return 0;
  }
}

static int staged_phase_tiles(const SysDesc& d, int kind) {
  switch (kind) {
    case kStgXFwdZero: case kStgXInv: return tiles_xpass(d);
    case kStgYFwd: case kStgYInv: return tiles_ypass(d);
    case kStgZFwd: case kStgZSolve: case kStgZInv: return tiles_zpass(d);
    default: return 1;
  }
}

cudaError_t staged_launch(const SysDesc& d, const int* kinds, int nphase, const StagedCtx& c, cudaStream_t s,
                          unsigned int* ticket = nullptr) {
  static std::mutex mu;
  static std::map<std::pair<int, size_t>, int> occ_cache;
  StagedArgs a;
  std::memset(&a, 0, sizeof(a));
  a.d = d;
  a.nphase = nphase;
  a.bar = c.bar;
  a.status = c.status;
  a.spin_limit = c.spin_limit;
  a.ticket = ticket;
  size_t smem = 32 * sizeof(long long);
  int most = 1;
  for (int p = 0; p < nphase; p++) {
    a.kind[p] = kinds[p];
    a.total[p] = staged_phase_tiles(d, kinds[p]);
    smem = std::max(smem, staged_phase_smem(d, kinds[p]));
    most = std::max(most, a.total[p]);
  }
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  int occ = 0, sms = 0;
  {
    std::lock_guard<std::mutex> g(mu);
    auto it = occ_cache.find({dev, smem});
    if (it != occ_cache.end()) occ = it->second;
  }
  if (occ == 0) {
    if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_staged, kThreads, smem)) != cudaSuccess) return e;
    if (occ < 1) return cudaErrorInvalidConfiguration;
    std::lock_guard<std::mutex> g(mu);
    occ_cache[{dev, smem}] = occ;
  }
  if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
  const int grid = std::min(sms * occ, most);
  void* params[] = {&a};
  return cudaLaunchCooperativeKernel((const void*)k_staged, dim3(grid), dim3(kThreads), params, smem, s);
}

cudaError_t staged_r2c(const SysDesc& d, const StagedCtx& c, cudaStream_t s) {
  const int kinds[3] = {kStgXFwdZero, kStgYFwd, kStgZFwd};
  return staged_launch(d, kinds, 3, c, s);
}

// One phase: every z tile computes the influence tables it needs, and the last CTA to finish
// writes the record (no grid barrier).  The ticket counter is the handle's barrier word 5.
cudaError_t staged_solve(const SysDesc& d, const StagedCtx& c, cudaStream_t s) {
  const int kinds[1] = {kStgZSolve};
  return staged_launch(d, kinds, 1, c, s, (unsigned int*)(c.bar + 5));
}

cudaError_t staged_c2r(const SysDesc& d, const StagedCtx& c, cudaStream_t s) {
  const int kinds[3] = {kStgZInv, kStgYInv, kStgXInv};
  return staged_launch(d, kinds, 3, c, s);
}

cudaError_t clear_records(const SysDesc* d_table, int nsys, cudaStream_t s) {
  const int n = nsys * kEvCount;
  k_clear_records<<<(n + 255) / 256, 256, 0, s>>>(d_table, nsys);
  return cudaGetLastError();
}

cudaError_t staged_gather(const SysDesc& d, cudaStream_t s) {
  const int blocks = tiles_gather(d);
  if (blocks <= 0) return cudaSuccess;
  k_gather<<<blocks, kThreads, 0, s>>>(d);
  return cudaGetLastError();
}

static const void* fused_kernel(int variant) {
  return variant == kFusedThroughput ? (const void*)k_fused_tput : (const void*)k_fused_lat;
}

// Resident CTAs per SM of the two builds at a dynamic shared-memory size, and the SM count, per
// device (the occupancy queries cost host time on every launch-shape choice otherwise).
struct Occupancy {
  int sms, lat, tput;
};

static cudaError_t occupancy(size_t smem, Occupancy* out) {
  static std::mutex mu;
  static std::map<std::pair<int, size_t>, Occupancy> cache;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  {
    std::lock_guard<std::mutex> g(mu);
    auto it = cache.find({dev, smem});
    if (it != cache.end()) {
      *out = it->second;
      return cudaSuccess;
    }
  }
  Occupancy o;
  if ((e = cudaDeviceGetAttribute(&o.sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
  if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o.lat, k_fused_lat, kThreads, smem)) != cudaSuccess)
    return e;
  if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o.tput, k_fused_tput, kThreads, smem)) != cudaSuccess)
    return e;
  std::lock_guard<std::mutex> g(mu);
  cache[{dev, smem}] = o;
  *out = o;
  return cudaSuccess;
}

cudaError_t fused_shape(const int* total, size_t smem, int grid_cap, FusedShape* out) {
  Occupancy o;
  cudaError_t e = occupancy(smem, &o);
  if (e != cudaSuccess) return e;
  const int sms = o.sms, occ_lat = o.lat, occ_tput = o.tput;
  int most = 1;
  for (int p = 0; p < kPhases; p++) most = most > total[p] ? most : total[p];
  // many tiles per CTA: more resident CTAs pay; about one: fewer registers per thread cost
  const bool tput = occ_tput > occ_lat && most > 2 * sms * occ_lat;
  out->variant = tput ? kFusedThroughput : kFusedLatency;
  out->cluster = 0;
  int grid = sms * (tput ? occ_tput : occ_lat);
  grid = grid < most ? grid : most;
  if (grid_cap > 0 && grid > grid_cap) grid = grid_cap;
  out->grid = grid;
  return grid >= 1 ? cudaSuccess : cudaErrorInvalidConfiguration;
}

// The cooperative launch of the latency build with thread-block clusters of cs CTAs (the cluster
// plane tiles): the CTAs that can be co-resident as whole clusters, at most the largest phase's
// tile count rounded up to whole clusters, at most grid_cap (rounded down to whole clusters).
static void cluster_config(cudaLaunchConfig_t* cfg, cudaLaunchAttribute* at, int cs, size_t smem, cudaStream_t s) {
  std::memset(cfg, 0, sizeof(*cfg));
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = (unsigned)cs;
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  at[1].id = cudaLaunchAttributeCooperative;
  at[1].val.cooperative = 1;
  cfg->gridDim = dim3((unsigned)cs);
  cfg->blockDim = dim3(kThreads);
  cfg->dynamicSmemBytes = smem;
  cfg->stream = s;
  cfg->attrs = at;
  cfg->numAttrs = 2;
}

cudaError_t fused_shape_cluster(const int* total, size_t smem, int grid_cap, int cs, FusedShape* out) {
  cudaLaunchConfig_t cfg;
  cudaLaunchAttribute at[2];
  cluster_config(&cfg, at, cs, smem, nullptr);
  int ncl = 0;
  cudaError_t e = cudaOccupancyMaxActiveClusters(&ncl, (const void*)k_fused_cl, &cfg);
  if (e != cudaSuccess) return e;
  int most = 1;
  for (int p = 0; p < kPhases; p++) most = most > total[p] ? most : total[p];
  int grid = ncl * cs;
  const int want = (most + cs - 1) / cs * cs;
  grid = grid < want ? grid : want;
  if (grid_cap > 0 && grid > grid_cap) grid = grid_cap / cs * cs;
  out->variant = kFusedLatency;
  out->grid = grid;
  out->cluster = cs;
  return grid >= cs ? cudaSuccess : cudaErrorInvalidConfiguration;
}

cudaError_t fused_launch(const FusedArgs& a, const FusedShape& shape, size_t smem, cudaStream_t s) {
  FusedArgs args = a;
  if (shape.cluster > 0) {
    cudaLaunchConfig_t cfg;
    cudaLaunchAttribute at[2];
    cluster_config(&cfg, at, shape.cluster, smem, s);
    cfg.gridDim = dim3((unsigned)shape.grid);
    return cudaLaunchKernelEx(&cfg, k_fused_cl, args);
  }
  void* params[] = {&args};
  return cudaLaunchCooperativeKernel(fused_kernel(shape.variant), dim3(shape.grid), dim3(kThreads), params, smem, s);
}

// Opt every dynamic-shared-memory kernel in to the device's per-CTA budget (minus the kernel's
// own static shared memory).  Called on the current device.
template <class K>
static cudaError_t opt_in_smem(K kernel, int optin) {
  cudaFuncAttributes fa;
  cudaError_t e = cudaFuncGetAttributes(&fa, kernel);
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              optin - (int)fa.sharedSizeBytes);
}

cudaError_t configure_kernels(size_t* max_dyn_smem) {
  int dev = 0, optin = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  if (e != cudaSuccess) return e;
  if ((e = opt_in_smem(k_spread, optin)) != cudaSuccess) return e;
  if ((e = opt_in_smem(k_fused_lat, optin)) != cudaSuccess) return e;
  if ((e = opt_in_smem(k_fused_tput, optin)) != cudaSuccess) return e;
  if ((e = opt_in_smem(k_fused_cl, optin)) != cudaSuccess) return e;
  if ((e = opt_in_smem(k_staged, optin)) != cudaSuccess) return e;
  cudaFuncAttributes fa;
  if ((e = cudaFuncGetAttributes(&fa, k_fused_lat)) != cudaSuccess) return e;
  if (max_dyn_smem) *max_dyn_smem = (size_t)optin - fa.sharedSizeBytes;
  return cudaSuccess;
}

}  // namespace pme

// pme_server.cu -- a request loop for PME evaluations with continuous batching.
//
// The reference evaluates one system per CudaPMERecip instance, fed by CudaDomdecRecipLooper's
// receive / compute / send loop (CudaDomdecRecipLooper.cu:3-36).  This server takes many such
// requests at once: each request is a system (grid, order, box, kappa, coordinates) and a number
// of evaluations of it, each on the coordinates plus a deterministic Gaussian jitter.  A host
// worker thread admits requests in arrival order while an active slot and device memory (from
// one arena allocated at creation) are free, and then runs steps: every step is one fused
// persistent launch that evaluates the next evaluation of every active request.  Requests that
// arrive while others run join at the next step; requests leave as they finish, and their
// memory returns to the arena.  Each request keeps its grids, moduli, bins and bin-sorted atom
// order on the device for all its evaluations.
//
// The fused kernel computes every system independently and bit-exactly, so a request's results
// do not depend on which other requests share its steps.
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

#include "../../include/pme_recip.h"
#include "pme_internal.h"
#include "pme_state.h"

using namespace pme;

namespace {

// Per active request, what the step kernels need.
struct SlotDesc {
  const float4* base;        // coordinates as submitted
  float4* cur;               // coordinates of the current evaluation
  double* ev;                // the system's energy/virial record (filled by the fused kernel)
  double* hist;              // [n_evals][kEvCount] records of finished evaluations
  unsigned long long seed;
  float sigma;
  int natom;
  int k;                     // index of the current evaluation
  int pad;
};

// Counter-based uniform in (0, 1]: splitmix64 finaliser of (seed, evaluation, atom, axis).
__device__ __forceinline__ unsigned long long mix64(unsigned long long z) {
  z += 0x9e3779b97f4a7c15ull;
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  return z ^ (z >> 31);
}

// Standard normal deviate for (seed, k, atom, axis) by the Box-Muller transform.
__device__ __forceinline__ float gauss(unsigned long long seed, int k, int atom, int axis) {
  const unsigned long long h =
      mix64(seed ^ mix64(((unsigned long long)(unsigned)k << 34) ^ ((unsigned long long)(unsigned)atom << 2) ^ axis));
  const float u1 = ((float)(h >> 40) + 1.0f) * (1.0f / 16777216.0f);          // (0, 1]
  const float u2 = (float)((h >> 16) & 0xffffffull) * (1.0f / 16777216.0f);    // [0, 1)
  return sqrtf(-2.0f * logf(u1)) * cospif(2.0f * u2);
}

// Before a step: the coordinates of each active request's current evaluation.
__global__ void k_server_pre(const SlotDesc* __restrict__ slots) {
  const SlotDesc s = slots[blockIdx.y];
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < s.natom; i += gridDim.x * blockDim.x) {
    float4 a = s.base[i];
    if (s.sigma > 0.0f) {
      a.x += s.sigma * gauss(s.seed, s.k, i, 0);
      a.y += s.sigma * gauss(s.seed, s.k, i, 1);
      a.z += s.sigma * gauss(s.seed, s.k, i, 2);
    }
    s.cur[i] = a;
  }
}

// After a step: move each request's record to its history, clear it, advance the evaluation.
__global__ void k_server_post(SlotDesc* slots, int nslots) {
  const int s = blockIdx.x;
  if (s >= nslots) return;
  SlotDesc& d = slots[s];
  const int t = threadIdx.x;
  if (t < kEvCount) {
    d.hist[(size_t)d.k * kEvCount + t] = d.ev[t];
    d.ev[t] = 0.0;
  }
  __syncthreads();
  if (t == 0) d.k += 1;
}

// First-fit allocator over one device allocation (host bookkeeping only).
class Arena {
 public:
  void reset(size_t size) {
    size_ = size;
    free_.clear();
    if (size) free_[0] = size;
    used_ = 0;
  }
  bool alloc(size_t bytes, size_t* off) {
    bytes = align256(bytes);
    for (auto it = free_.begin(); it != free_.end(); ++it) {
      if (it->second >= bytes) {
        *off = it->first;
        const size_t rest = it->second - bytes, at = it->first + bytes;
        free_.erase(it);
        if (rest) free_[at] = rest;
        used_ += bytes;
        return true;
      }
    }
    return false;
  }
  void release(size_t off, size_t bytes) {
    bytes = align256(bytes);
    used_ -= bytes;
    auto it = free_.emplace(off, bytes).first;
    auto next = std::next(it);
    if (next != free_.end() && it->first + it->second == next->first) {
      it->second += next->second;
      free_.erase(next);
    }
    if (it != free_.begin()) {
      auto prev = std::prev(it);
      if (prev->first + prev->second == it->first) {
        prev->second += it->second;
        free_.erase(it);
      }
    }
  }
  size_t size() const { return size_; }
  size_t used() const { return used_; }

 private:
  size_t size_ = 0, used_ = 0;
  std::map<size_t, size_t> free_;
};

enum ReqState { kPending = 0, kActive = 1, kFinishing = 2, kDone = 3, kFailed = 4 };

struct Request {
  long long id = 0;
  pme_request r{};
  int state = kPending;
  int status = PME_OK;
  double t_submit = 0, t_admit = 0, t_done = 0;
  // host: pinned staging of the coordinates and of the results
  float* h_stage = nullptr;   // [natom*4 xyzq][n_evals*kEvCount doubles][natom*3 force]
  size_t stage_cap = 0;       // bytes of the h_stage buffer (a pooled buffer may be larger)
  bool stage_in_arena = false;   // h_stage is a block of the server's pinned host arena
  // device
  size_t off = 0, bytes = 0;
  SystemState st;
  float4* base = nullptr;
  float4* cur = nullptr;
  float* force = nullptr;
  double* hist = nullptr;
  int stride = 0;
  int k = 0;                  // evaluations issued
  cudaEvent_t done_ev = nullptr;

  double* h_ev() const { return (double*)(h_stage + (size_t)r.natom * 4); }
  float* h_force() const { return (float*)(h_ev() + (size_t)r.n_evals * kEvCount); }
  // twiddles (float2) then moduli (double) of the three axes
  char* h_tables() const { return (char*)(h_force() + (size_t)r.natom * 3); }
  static size_t stage_bytes(const pme_request& q) {
    return (size_t)q.natom * 16 + (size_t)q.n_evals * kEvCount * 8 + (size_t)q.natom * 12 +
           (size_t)(q.nfftx + q.nffty + q.nfftz) * 16 + 16;
  }
};

size_t request_bytes(const pme_request& q) {
  SystemState st;
  st.setup(q.nfftx, q.nffty, q.nfftz, q.order);
  const int n = std::max(q.natom, 1);
  const size_t stride = (size_t)((n + 63) / 64) * 64;
  return align256(SystemState::bytes(q.nfftx, q.nffty, q.nfftz)) + align256(st.bin_ints(n) * sizeof(int)) +
         2 * align256((size_t)n * 16) + align256(3 * stride * sizeof(float)) +
         align256((size_t)q.n_evals * kEvCount * sizeof(double));
}

double now_s() {
  using namespace std::chrono;
  return duration<double>(steady_clock::now().time_since_epoch()).count();
}

int check_request(const pme_request* q) {
  if (!q) return fail(PME_EINVAL, "request is NULL");
  if (int rc = check_grid(q->nfftx, q->nffty, q->nfftz, q->order)) return rc;
  if (q->natom < 1 || !q->xyzq) return fail(PME_EINVAL, "a request needs natom >= 1 and host xyzq");
  if (q->n_evals < 1 || q->n_evals > 1000000) return fail(PME_EINVAL, "n_evals must be in [1, 10^6]");
  if (!(q->box[0] > 0 && q->box[1] > 0 && q->box[2] > 0) || !(q->kappa > 0))
    return fail(PME_EINVAL, "box edges and kappa must be positive");
  if (!(q->sigma >= 0.0f) || !std::isfinite(q->sigma)) return fail(PME_EINVAL, "sigma must be finite and >= 0");
  if (!q->ev_out) return fail(PME_EINVAL, "ev_out is NULL");
  return PME_OK;
}

}  // namespace

struct HostTables {
  std::vector<float2> tw;
  std::vector<double> bmod;
};

struct pme_server {
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  char* d_arena = nullptr;
  Arena arena;
  int max_active = 0;
  size_t max_smem = 0;
  double t0 = 0;
  unsigned int spin_limit = 1u << 22;
  // launch state
  SysDesc* d_table = nullptr;
  int* d_prefix = nullptr;
  SlotDesc* d_slots = nullptr;
  unsigned long long* d_bar = nullptr;
  int* d_status = nullptr;
  std::vector<SysDesc> h_table;
  std::vector<SlotDesc> h_slots;
  std::vector<int> h_prefix;
  char* h_stage[2] = {nullptr, nullptr};   // pinned copies of the tables, alternating per rebuild
  size_t stage_bytes = 0;
  int stage_parity = 0;
  int* h_status = nullptr;                 // pinned: device status after each step, by parity
  int total[kPhases] = {0};
  size_t smem = 0;
  FusedShape shape{kFusedLatency, 0};
  cudaEvent_t step_ev[2] = {nullptr, nullptr};
  int step_parity = 0;
  // requests
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<Request*> pending;
  std::vector<Request*> active, finishing;
  std::map<long long, std::unique_ptr<Request>> reqs;
  long long next_id = 1;
  bool stop = false;
  bool failed = false;
  std::thread worker;
  // pinned staging buffers and completion events of finished requests, reused by later ones:
  // cudaHostAlloc is slow, and cudaFreeHost can synchronise the device under running steps
  char* h_arena = nullptr;                    // pinned host arena for request staging
  Arena harena;
  std::multimap<size_t, float*> stage_pool;   // capacity -> buffer (staging beyond the arena)
  size_t stage_pool_bytes = 0;
  std::vector<cudaEvent_t> event_pool;
  // twiddles and B-spline moduli by (nx, ny, nz, order): built once on the host (the moduli are an
  // O(n^2) sum per axis) and shared by every request of that grid
  std::map<std::array<int, 4>, HostTables> tables;
  const HostTables& tables_for(const SystemState& st) {
    const std::array<int, 4> key = {st.nx, st.ny, st.nz, st.order};
    auto it = tables.find(key);
    if (it == tables.end()) {
      HostTables t;
      st.host_tables(t.tw, t.bmod);
      it = tables.emplace(key, std::move(t)).first;
    }
    return it->second;
  }
  // statistics
  long long n_submitted = 0, n_completed = 0, n_evals = 0, n_steps = 0;
};

namespace {

constexpr size_t kHostArenaBytes = 256ull << 20;  // pinned staging arena (at most)
constexpr size_t kStagePoolMax = 512ull << 20;   // pinned bytes kept for reuse beyond the arena

// Take a pooled staging buffer of at least `need` bytes (at most twice that) and a pooled event,
// if there are any (lock held).
void take_staging(pme_server* s, Request* q, size_t need) {
  size_t off = 0;
  if (s->h_arena && s->harena.alloc(need, &off)) {
    q->h_stage = (float*)(s->h_arena + off);
    q->stage_cap = need;
    q->stage_in_arena = true;
  }
  auto it = q->h_stage ? s->stage_pool.end() : s->stage_pool.lower_bound(need);
  if (it != s->stage_pool.end() && it->first <= 2 * need + 65536) {
    q->h_stage = it->second;
    q->stage_cap = it->first;
    s->stage_pool_bytes -= it->first;
    s->stage_pool.erase(it);
  }
  if (!s->event_pool.empty()) {
    q->done_ev = s->event_pool.back();
    s->event_pool.pop_back();
  }
}

// Return a request's staging buffer and event to the pools (lock held); buffers beyond the
// pool's limit are freed.
void release_staging(pme_server* s, Request* q) {
  if (q->h_stage && q->stage_in_arena) {
    s->harena.release((size_t)((char*)q->h_stage - s->h_arena), q->stage_cap);
    q->h_stage = nullptr;
    q->stage_in_arena = false;
  }
  if (q->h_stage) {
    if (s->stage_pool_bytes + q->stage_cap <= kStagePoolMax) {
      s->stage_pool.emplace(q->stage_cap, q->h_stage);
      s->stage_pool_bytes += q->stage_cap;
    } else {
      cudaFreeHost(q->h_stage);
    }
    q->h_stage = nullptr;
  }
  if (q->done_ev) {
    s->event_pool.push_back(q->done_ev);
    q->done_ev = nullptr;
  }
}

// Allocate, clear and fill the device state of a pending request (worker thread, lock held).
int admit(pme_server* s, Request* q) {
  const pme_request& r = q->r;
  q->st.setup(r.nfftx, r.nffty, r.nfftz, r.order);
  const size_t sys = align256(SystemState::bytes(r.nfftx, r.nffty, r.nfftz));
  const size_t bins = align256(q->st.bin_ints(r.natom) * sizeof(int));
  const size_t xb = align256((size_t)r.natom * 16);
  q->stride = ((r.natom + 63) / 64) * 64;
  const size_t fb = align256(3 * (size_t)q->stride * sizeof(float));
  char* p = s->d_arena + q->off;
  cudaError_t e = cudaMemsetAsync(p, 0, q->bytes, s->stream);
  if (e != cudaSuccess) return cuda_fail(e, "server: clear request memory");
  q->st.carve(p);
  q->st.bins = (int*)(p + sys);
  q->st.atom_cap = r.natom;
  q->st.bin_cap = SystemState::cap_for(r.natom, q->st.nbins());
  q->base = (float4*)(p + sys + bins);
  q->cur = (float4*)(p + sys + bins + xb);
  q->force = (float*)(p + sys + bins + 2 * xb);
  q->hist = (double*)(p + sys + bins + 2 * xb + fb);
  // twiddles, moduli and coordinates from the request's pinned staging copy (stream-ordered after
  // the clear)
  const HostTables& tab = s->tables_for(q->st);
  const std::vector<float2>& twh = tab.tw;
  const std::vector<double>& bm = tab.bmod;
  char* ht = q->h_tables();
  std::memcpy(ht, twh.data(), twh.size() * sizeof(float2));
  std::memcpy(ht + twh.size() * sizeof(float2), bm.data(), bm.size() * sizeof(double));
  e = cudaMemcpyAsync(q->st.tw, ht, twh.size() * sizeof(float2), cudaMemcpyHostToDevice, s->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(q->st.bmod, ht + twh.size() * sizeof(float2), bm.size() * sizeof(double),
                        cudaMemcpyHostToDevice, s->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(q->base, q->h_stage, (size_t)r.natom * 16, cudaMemcpyHostToDevice, s->stream);
  if (e != cudaSuccess) return cuda_fail(e, "server: upload request");
  return PME_OK;
}

// Rebuild the launch tables of the active set and upload them (stream-ordered).
int rebuild(pme_server* s) {
  const int n = (int)s->active.size();
  s->h_table.resize(n);
  s->h_slots.resize(n);
  s->h_prefix.assign((size_t)kPhases * (n + 1), 0);
  s->smem = 0;
  for (int i = 0; i < n; i++) {
    Request* q = s->active[i];
    const pme_request& r = q->r;
    const double r3[3] = {1.0 / r.box[0], 1.0 / r.box[1], 1.0 / r.box[2]};
    SysDesc d = q->st.desc(r3, r.kappa, q->cur, r.natom, q->force, PME_FORCE_F32X3, q->stride,
                           (r.calc_energy || r.calc_virial) ? 1 : 0, r.calc_energy ? 1 : 0);
    s->h_table[i] = d;
    int cnt[kPhases];
    fused_tile_counts(d, cnt);
    for (int p = 0; p < kPhases; p++)
      s->h_prefix[(size_t)p * (n + 1) + i + 1] = s->h_prefix[(size_t)p * (n + 1) + i] + cnt[p];
    s->smem = std::max(s->smem, fused_smem_bytes(d));
    SlotDesc& sl = s->h_slots[i];
    sl.base = q->base;
    sl.cur = q->cur;
    sl.ev = q->st.ev;
    sl.hist = q->hist;
    sl.seed = r.seed;
    sl.sigma = r.sigma;
    sl.natom = r.natom;
    sl.k = q->k;
    sl.pad = 0;
  }
  for (int p = 0; p < kPhases; p++) s->total[p] = s->h_prefix[(size_t)p * (n + 1) + n];
  for (int i = 0; i < n; i++) s->h_table[i].gsort = gather_sorts(s->h_table[i], s->smem);
  if (n == 0) return PME_OK;
  // Stream order puts these copies after the previous step's launches, which read the tables.
  // The pinned source alternates per rebuild; the copies from the buffer's previous use were
  // queued before an earlier step that the worker has already waited for.
  char* st = s->h_stage[s->stage_parity];
  s->stage_parity ^= 1;
  const size_t tb = sizeof(SysDesc) * n, pb = sizeof(int) * s->h_prefix.size(), sb = sizeof(SlotDesc) * n;
  std::memcpy(st, s->h_table.data(), tb);
  std::memcpy(st + align256(tb), s->h_prefix.data(), pb);
  std::memcpy(st + align256(tb) + align256(pb), s->h_slots.data(), sb);
  cudaError_t e = cudaMemcpyAsync(s->d_table, st, tb, cudaMemcpyHostToDevice, s->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(s->d_prefix, st + align256(tb), pb, cudaMemcpyHostToDevice, s->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(s->d_slots, st + align256(tb) + align256(pb), sb, cudaMemcpyHostToDevice, s->stream);
  if (e != cudaSuccess) return cuda_fail(e, "server: upload tables");
  e = fused_shape(s->total, s->smem, 0, &s->shape);
  if (e != cudaSuccess) return cuda_fail(e, "server: launch shape");
  return PME_OK;
}

// One step: coordinates, the fused evaluation of every active request, records to history.
int step(pme_server* s) {
  const int n = (int)s->active.size();
  int maxatoms = 1;
  for (Request* q : s->active) maxatoms = std::max(maxatoms, q->r.natom);
  dim3 g1((unsigned)std::min((maxatoms + 255) / 256, 64), (unsigned)n);
  k_server_pre<<<g1, 256, 0, s->stream>>>(s->d_slots);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "server: coordinates");
  FusedArgs a;
  std::memset(&a, 0, sizeof(a));
  a.table = s->d_table;
  a.nsys = n;
  a.prefix = s->d_prefix;
  for (int p = 0; p < kPhases; p++) a.total[p] = s->total[p];
  a.nbar = fused_barriers(a.total);
  a.bar = s->d_bar;
  a.status = s->d_status;
  a.spin_limit = s->spin_limit;
  e = fused_launch(a, s->shape, s->smem, s->stream);
  if (e != cudaSuccess) return cuda_fail(e, "server: fused launch");
  k_server_post<<<n, 32, 0, s->stream>>>(s->d_slots, n);
  e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "server: records");
  for (Request* q : s->active) q->k++;
  s->n_steps++;
  s->n_evals += n;
  return PME_OK;
}

void finish_request(pme_server* s, Request* q) {
  const pme_request& r = q->r;
  cudaMemcpyAsync(q->h_ev(), q->hist, (size_t)r.n_evals * kEvCount * sizeof(double), cudaMemcpyDeviceToHost, s->stream);
  if (r.force_out)
    cudaMemcpyAsync(q->h_force(), q->force, (size_t)r.natom * 3 * sizeof(float), cudaMemcpyDeviceToHost, s->stream);
  cudaEventRecord(q->done_ev, s->stream);
  q->state = kFinishing;
}

void fail_all(pme_server* s, int status) {
  for (Request* q : s->active) {
    q->state = kFailed;
    q->status = status;
    q->t_done = now_s() - s->t0;
    s->arena.release(q->off, q->bytes);
  }
  s->active.clear();
  for (Request* q : s->pending) {
    q->state = kFailed;
    q->status = status;
  }
  s->pending.clear();
  s->failed = true;
}

void worker_loop(pme_server* s) {
  cudaSetDevice(s->device);
  std::unique_lock<std::mutex> lock(s->mu);
  bool dirty = false;
  while (true) {
    // results whose copies have landed
    for (auto it = s->finishing.begin(); it != s->finishing.end();) {
      Request* q = *it;
      if (cudaEventQuery(q->done_ev) == cudaSuccess) {
        q->t_done = now_s() - s->t0;
        std::memcpy(q->r.ev_out, q->h_ev(), (size_t)q->r.n_evals * kEvCount * sizeof(double));
        if (q->r.force_out) std::memcpy(q->r.force_out, q->h_force(), (size_t)q->r.natom * 3 * sizeof(float));
        s->arena.release(q->off, q->bytes);
        q->state = kDone;
        s->n_completed++;
        it = s->finishing.erase(it);
        s->cv_done.notify_all();
      } else {
        ++it;
      }
    }
    // admission in arrival order while a slot and memory are free
    while (!s->failed && !s->pending.empty() && (int)s->active.size() < s->max_active) {
      Request* q = s->pending.front();
      size_t off = 0;
      if (!s->arena.alloc(q->bytes, &off)) break;
      q->off = off;
      s->pending.pop_front();
      const int rc = admit(s, q);
      if (rc) {
        s->arena.release(q->off, q->bytes);
        q->state = kFailed;
        q->status = rc;
        s->cv_done.notify_all();
        continue;
      }
      q->t_admit = now_s() - s->t0;
      q->state = kActive;
      s->active.push_back(q);
      dirty = true;
    }
    if (s->active.empty()) {
      if (s->stop && s->pending.empty() && s->finishing.empty()) break;
      if (s->finishing.empty()) s->cv_work.wait(lock);
      else s->cv_work.wait_for(lock, std::chrono::microseconds(50));
      continue;
    }
    // keep at most two steps queued on the stream: wait for the step two back, whose status
    // word has then landed
    const int par = s->step_parity;
    lock.unlock();
    cudaEventSynchronize(s->step_ev[par]);
    lock.lock();
    if (s->h_status[par] != kStatusOk) {
      fail_all(s, PME_ETIMEOUT);
      s->cv_done.notify_all();
      continue;
    }
    if (dirty) {
      if (int rc = rebuild(s)) { fail_all(s, rc); s->cv_done.notify_all(); continue; }
      dirty = false;
    }
    if (int rc = step(s)) { fail_all(s, rc); s->cv_done.notify_all(); continue; }
    cudaMemcpyAsync(&s->h_status[par], s->d_status, sizeof(int), cudaMemcpyDeviceToHost, s->stream);
    cudaEventRecord(s->step_ev[par], s->stream);
    s->step_parity ^= 1;
    // requests whose last evaluation was just queued leave the active set
    for (auto it = s->active.begin(); it != s->active.end();) {
      Request* q = *it;
      if (q->k >= q->r.n_evals) {
        finish_request(s, q);
        s->finishing.push_back(q);
        it = s->active.erase(it);
        dirty = true;
      } else {
        ++it;
      }
    }
  }
}

}  // namespace

extern "C" {

size_t pme_request_device_bytes(const pme_request* r) {
  if (!r || check_grid(r->nfftx, r->nffty, r->nfftz, r->order) != PME_OK || r->natom < 0 || r->n_evals < 1) return 0;
  return request_bytes(*r);
}

int pme_server_create(size_t device_bytes, int max_active, void* stream, pme_server** out) {
  if (!out) return fail(PME_EINVAL, "out is NULL");
  *out = nullptr;
  if (device_bytes < (1u << 20)) return fail(PME_EINVAL, "device_bytes must be at least 1 MiB");
  if (max_active < 1 || max_active > 4096) return fail(PME_EINVAL, "max_active must be in [1, 4096]");
  pme_server* s = new (std::nothrow) pme_server();
  if (!s) return fail(PME_ENOMEM, "host allocation failed");
  cudaError_t e = cudaGetDevice(&s->device);
  if (e == cudaSuccess) e = configure_kernels(&s->max_smem);
  if (e == cudaSuccess) {
    if (stream) {
      s->stream = (cudaStream_t)stream;
    } else {
      e = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking);
      s->own_stream = e == cudaSuccess;
    }
  }
  const size_t table = align256(sizeof(SysDesc) * max_active) + align256(sizeof(int) * kPhases * (max_active + 1)) +
                       align256(sizeof(SlotDesc) * max_active);
  char* t = nullptr;
  if (e == cudaSuccess && cudaMalloc(&s->d_arena, device_bytes) != cudaSuccess) e = cudaErrorMemoryAllocation;
  if (e == cudaSuccess && cudaMalloc(&t, table) != cudaSuccess) e = cudaErrorMemoryAllocation;
  if (e == cudaSuccess && cudaMalloc(&s->d_bar, 4 * sizeof(unsigned long long)) != cudaSuccess)
    e = cudaErrorMemoryAllocation;
  if (e == cudaSuccess) e = cudaMemset(s->d_bar, 0, 4 * sizeof(unsigned long long));
  for (int i = 0; i < 2 && e == cudaSuccess; i++) e = cudaEventCreateWithFlags(&s->step_ev[i], cudaEventDisableTiming);
  s->stage_bytes = table;
  for (int i = 0; i < 2 && e == cudaSuccess; i++) e = cudaHostAlloc(&s->h_stage[i], table, cudaHostAllocDefault);
  if (e == cudaSuccess) e = cudaHostAlloc(&s->h_status, 2 * sizeof(int), cudaHostAllocDefault);
  if (e == cudaSuccess) s->h_status[0] = s->h_status[1] = kStatusOk;
  // pinned staging of submitted requests comes from one arena allocated here, so that submit
  // makes no pinned allocation (which holds the driver against the worker's launches); requests
  // beyond it allocate their own
  if (e == cudaSuccess) {
    const size_t hb = std::min<size_t>(kHostArenaBytes, std::max<size_t>(device_bytes / 16, 16u << 20));
    if (cudaHostAlloc(&s->h_arena, hb, cudaHostAllocDefault) == cudaSuccess) s->harena.reset(hb);
    else { cudaGetLastError(); s->h_arena = nullptr; }
  }
  if (e != cudaSuccess) {
    cudaGetLastError();
    cudaFree(s->d_arena);
    cudaFree(t);
    cudaFree(s->d_bar);
    for (cudaEvent_t ev : s->step_ev) if (ev) cudaEventDestroy(ev);
    for (char* h : s->h_stage) if (h) cudaFreeHost(h);
    if (s->h_status) cudaFreeHost(s->h_status);
    if (s->own_stream) cudaStreamDestroy(s->stream);
    delete s;
    return e == cudaErrorMemoryAllocation ? fail(PME_ENOMEM, "server: device allocation failed")
                                          : cuda_fail(e, "server: create");
  }
  s->d_table = (SysDesc*)t;
  s->d_prefix = (int*)(t + align256(sizeof(SysDesc) * max_active));
  s->d_slots = (SlotDesc*)(t + align256(sizeof(SysDesc) * max_active) + align256(sizeof(int) * kPhases * (max_active + 1)));
  s->d_status = (int*)(s->d_bar + 2);
  s->arena.reset(device_bytes);
  s->max_active = max_active;
  s->t0 = now_s();
  s->worker = std::thread(worker_loop, s);
  *out = s;
  return PME_OK;
}

int pme_server_submit(pme_server* s, const pme_request* r, long long* id) {
  if (!s) return fail(PME_EINVAL, "server is NULL");
  if (int rc = check_request(r)) return rc;
  const size_t bytes = request_bytes(*r);
  if (bytes > s->arena.size()) return fail(PME_ENOMEM, "request is larger than the server's device memory");
  std::unique_ptr<Request> q(new (std::nothrow) Request());
  if (!q) return fail(PME_ENOMEM, "host allocation failed");
  q->r = *r;
  q->bytes = bytes;
  const size_t need = Request::stage_bytes(*r);
  cudaError_t e = cudaSetDevice(s->device);
  {
    std::lock_guard<std::mutex> lock(s->mu);
    take_staging(s, q.get(), need);
  }
  if (e == cudaSuccess && !q->h_stage) {
    q->stage_cap = (need + 4095) & ~(size_t)4095;
    e = cudaHostAlloc(&q->h_stage, q->stage_cap, cudaHostAllocDefault);
    if (e != cudaSuccess) q->h_stage = nullptr;
  }
  if (e == cudaSuccess && !q->done_ev) e = cudaEventCreateWithFlags(&q->done_ev, cudaEventDisableTiming);
  if (e != cudaSuccess) {
    std::lock_guard<std::mutex> lock(s->mu);
    release_staging(s, q.get());
    return cuda_fail(e, "server: request staging");
  }
  std::memcpy(q->h_stage, r->xyzq, (size_t)r->natom * 16);
  std::lock_guard<std::mutex> lock(s->mu);
  if (s->stop) {
    release_staging(s, q.get());
    return fail(PME_ESTATE, "server is shutting down");
  }
  q->id = s->next_id++;
  q->t_submit = now_s() - s->t0;
  Request* raw = q.get();
  s->reqs[raw->id] = std::move(q);
  s->pending.push_back(raw);
  s->n_submitted++;
  if (id) *id = raw->id;
  s->cv_work.notify_all();
  return PME_OK;
}

int pme_server_wait(pme_server* s, long long id, double timeout_s, double* times3) {
  if (!s) return fail(PME_EINVAL, "server is NULL");
  std::unique_lock<std::mutex> lock(s->mu);
  auto it = s->reqs.find(id);
  if (it == s->reqs.end()) return fail(PME_EINVAL, "unknown request id");
  Request* q = it->second.get();
  auto finished = [&]() { return q->state == kDone || q->state == kFailed; };
  if (timeout_s < 0) {
    s->cv_done.wait(lock, finished);
  } else if (!s->cv_done.wait_for(lock, std::chrono::duration<double>(timeout_s), finished)) {
    return fail(PME_ETIMEOUT, "request not finished within the timeout");
  }
  if (times3) {
    times3[0] = q->t_submit;
    times3[1] = q->t_admit;
    times3[2] = q->t_done;
  }
  const int status = q->status;
  release_staging(s, q);
  s->reqs.erase(it);
  if (status != PME_OK) return fail(status, "request failed");
  return PME_OK;
}

int pme_server_get_stats(pme_server* s, pme_server_stats* out) {
  if (!s || !out) return fail(PME_EINVAL, "NULL argument");
  std::lock_guard<std::mutex> lock(s->mu);
  out->submitted = s->n_submitted;
  out->completed = s->n_completed;
  out->evals = s->n_evals;
  out->steps = s->n_steps;
  out->active = (long long)s->active.size();
  out->pending = (long long)s->pending.size();
  out->arena_bytes = s->arena.size();
  out->arena_used = s->arena.used();
  out->seconds = now_s() - s->t0;
  return PME_OK;
}

int pme_server_destroy(pme_server* s) {
  if (!s) return PME_OK;
  {
    std::lock_guard<std::mutex> lock(s->mu);
    s->stop = true;
    s->cv_work.notify_all();
  }
  if (s->worker.joinable()) s->worker.join();
  cudaSetDevice(s->device);
  cudaStreamSynchronize(s->stream);
  for (auto& kv : s->reqs) {
    if (kv.second->h_stage && !kv.second->stage_in_arena) cudaFreeHost(kv.second->h_stage);
    if (kv.second->done_ev) cudaEventDestroy(kv.second->done_ev);
  }
  for (auto& kv : s->stage_pool) cudaFreeHost(kv.second);
  if (s->h_arena) cudaFreeHost(s->h_arena);
  for (cudaEvent_t ev : s->event_pool) cudaEventDestroy(ev);
  cudaFree(s->d_arena);
  cudaFree(s->d_table);
  cudaFree(s->d_bar);
  for (cudaEvent_t ev : s->step_ev) if (ev) cudaEventDestroy(ev);
  for (char* h : s->h_stage) if (h) cudaFreeHost(h);
  if (s->h_status) cudaFreeHost(s->h_status);
  if (s->own_stream) cudaStreamDestroy(s->stream);
  delete s;
  return PME_OK;
}

}  // extern "C"

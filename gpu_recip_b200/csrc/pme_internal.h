// pme_internal.h -- host-side launch interface of the PME reciprocal-space kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "pme_common.cuh"
#include "pme_fft.cuh"
#include "pme_tiles.cuh"

namespace pme {

constexpr int kPhases = 7;

// Device status word values (fused kernel).
enum { kStatusOk = 0, kStatusBarrierTimeout = 1 };

// Arguments of the persistent fused kernel.  A single system travels by value (`single`, with
// table == nullptr); a batch uses a device table of descriptors and per-phase tile prefix sums
// prefix[ph * (nsys + 1) + s].
struct FusedArgs {
  const SysDesc* table;
  SysDesc single;
  int nsys;
  const int* prefix;
  int total[kPhases];
  unsigned long long* bar;   // [arrival counter, counter value at launch start], zero-initialised
  int* status;               // kStatus*; sticky until cleared by the host
  unsigned int spin_limit;   // barrier polls before giving up
  int inject;                // 1: CTA 0 leaves before the first barrier (failure-detection test)
  int nbar;                  // grid barriers per launch (non-empty phases - 1)
  unsigned long long* trace; // optional: [cta][phase][begin, end] %globaltimer stamps
  int trace_ctas;            // CTAs recorded (rows of trace)
};

cudaError_t configure_kernels(size_t* max_dyn_smem);

// Record the calling thread's last error message (returned by pme_last_error_string).
void set_last_error(const char* msg);

size_t spread_smem(int order);
size_t fused_smem_bytes(const SysDesc& d);
void fused_tile_counts(const SysDesc& d, int* counts);
int fused_barriers(const int* total);

// Phases of a staged cooperative launch (k_staged): one reference-interface call each.
// kStgXFwdZero reads the int64 charge grid and leaves it zero behind it (ready for the next
// atomic spread).
enum StagedKind {
  kStgXFwdZero = 0, kStgYFwd, kStgZFwd, kStgZSolve, kStgZInv, kStgYInv, kStgXInv
};
constexpr int kStagedMaxPhases = 4;

struct StagedArgs {
  SysDesc d;
  int nphase;
  int kind[kStagedMaxPhases];
  int total[kStagedMaxPhases];
  unsigned long long* bar;   // the handle's barrier words (shared with its fused evaluations)
  int* status;
  unsigned int spin_limit;
  unsigned int* ticket;      // non-null: the last CTA to finish finalises the solve's record
};

// The handle's barrier words and failure-detection settings for a staged launch.
struct StagedCtx {
  unsigned long long* bar;
  int* status;
  unsigned int spin_limit;
};

// Global-atomic spread of one tile per CTA into a cleared accumulation grid (exact int64 sums).
cudaError_t staged_spread(const SysDesc& d, cudaStream_t s);
// Reference-interface calls as cooperative launches: x (clearing the charge grid behind it), y, z
// forward passes; influence tables, solve with energy/virial and the record update; z, y, x
// inverse passes.
cudaError_t staged_r2c(const SysDesc& d, const StagedCtx& c, cudaStream_t s);
cudaError_t staged_solve(const SysDesc& d, const StagedCtx& c, cudaStream_t s);
cudaError_t staged_c2r(const SysDesc& d, const StagedCtx& c, cudaStream_t s);
// Self energy in one launch (done: an arrival counter, zero between launches).
cudaError_t staged_self(const SysDesc& d, unsigned int* done, cudaStream_t s);
cudaError_t staged_gather(const SysDesc& d, cudaStream_t s);
// Zero the energy/virial records of the nsys systems of a device descriptor table.
cudaError_t clear_records(const SysDesc* d_table, int nsys, cudaStream_t s);

// Launch shape of a fused evaluation: which build of the kernel and how many CTAs.
enum { kFusedLatency = 0, kFusedThroughput = 1 };
struct FusedShape {
  int variant;
  int grid;
  int cluster;   // > 0: launched with thread-block clusters of this many CTAs (latency build)
};
// Picks the build and the CTAs (at most the resident maximum, at most the largest phase's tile
// count, at most grid_cap when > 0) for phases of total[] tiles and smem bytes per CTA.
cudaError_t fused_shape(const int* total, size_t smem, int grid_cap, FusedShape* out);
cudaError_t fused_launch(const FusedArgs& a, const FusedShape& shape, size_t smem, cudaStream_t s);
// The same for a launch with clusters of cs CTAs (the cluster plane tiles).
cudaError_t fused_shape_cluster(const int* total, size_t smem, int grid_cap, int cs, FusedShape* out);

}  // namespace pme

/* pme_recip.h -- C ABI of the B200 smooth-PME reciprocal-space engine.
 *
 * Drop-in for the operator surface of the reference class CudaPMERecip<AT,CT,CT2>
 * (ap-hynninen/gpu_recip, CudaPMERecip.h:37-205) and of its MD adapter CudaDomdecRecip
 * (CudaDomdecRecip.h:9-83).  Plain pointers and sizes only; every device pointer argument is a
 * CUDA device address, every call is asynchronous on the handle's stream unless it says it
 * synchronises.  Units: Angstrom, elementary charge, kcal/mol (ccelec = 332.0716).
 *
 * Differences from the reference, by design:
 *  - errors are returned as a status code (never exit()); pme_last_error_string() explains;
 *  - the charge grid is always accumulated in int64 fixed point (scale 2^40), so it is exact
 *    and run-to-run deterministic; energy and virial reductions are deterministic too;
 *  - the energy/virial record is owned by the handle (slots "recip" and "self" plus a 3x3
 *    virial), accumulated like CudaEnergyVirial and cleared with pme_clear_energy_virial().
 */
#ifndef PME_RECIP_H
#define PME_RECIP_H

#include <stddef.h>

#if defined(__GNUC__)
#define PME_API __attribute__((visibility("default")))
#else
#define PME_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef struct pme_recip pme_recip;      /* opaque operator instance */

typedef enum {
  PME_OK = 0,
  PME_EINVAL = -1,        /* bad argument (null pointer, size, order, singular or non-finite box) */
  PME_EUNSUPPORTED = -2,  /* valid but not supported (grid length with a prime factor > 5) */
  PME_ECUDA = -3,         /* CUDA runtime error */
  PME_ETIMEOUT = -4,      /* a bounded wait gave up */
  PME_ENOMEM = -5,        /* device or host allocation failed */
  PME_ESTATE = -6         /* call out of order (e.g. no handle state for the request) */
} pme_status;

/* FFT decomposition of the reference (CudaPMERecip.h:30).  On one GPU all three give the same
 * result; this engine always runs its own single-GPU 3-D transform. */
typedef enum { PME_FFT_COLUMN = 0, PME_FFT_SLAB = 1, PME_FFT_BOX = 2 } pme_fft_type;

/* Force output kinds of gather_force<FT> (CudaPMERecip.cu:983-1024). */
typedef enum {
  PME_FORCE_F32_SOA = 0,       /* float x|y|z blocks at force, force+stride, force+2*stride; overwrite */
  PME_FORCE_F32X3 = 1,         /* float3 array (AoS); overwrite; stride ignored */
  PME_FORCE_I64_SOA_ACCUM = 2  /* long long fixed point 2^40, SoA with stride; atomically ADDED */
} pme_force_kind;

/* Energy/virial record slots (doubles), device resident. */
enum { PME_EV_RECIP = 0, PME_EV_SELF = 1, PME_EV_VIRIAL = 2, PME_EV_COUNT = 11 };

/* ---- lifetime (CudaPMERecip ctor/dtor, CudaPMERecip.h:166-170, CudaPMERecip.cu:1411-1493) ---- */
/* nnode must be 1 and mynode 0 (single GPU).  order in {4, 6, 8}; every grid length must be
 * 2/3/5-smooth, >= order and <= 512.  stream: cudaStream_t (0 = legacy default stream). */
PME_API int pme_create(int nfftx, int nffty, int nfftz, int order, int fft_type, int nnode, int mynode,
               void* stream, pme_recip** out);
PME_API int pme_destroy(pme_recip* h);

/* ---- configuration (CudaPMERecip.h:176-178, :198-201) ---- */
PME_API int pme_set_stream(pme_recip* h, void* stream);
PME_API int pme_get_stream(const pme_recip* h, void** stream);     /* the handle's cudaStream_t */
PME_API int pme_set_order(pme_recip* h, int order);                 /* recomputes the B-spline moduli */
PME_API int pme_get_nfft(const pme_recip* h, int* nfftx, int* nffty, int* nfftz);
PME_API int pme_get_order(const pme_recip* h, int* order);
PME_API int pme_print_info(const pme_recip* h);                    /* to stdout (CudaPMERecip.cu:1710) */

/* ---- stages (CudaPMERecip.h:180-197) ----
 * xyzq: device float4[ncoord] (x, y, z, q).  recip: HOST double[9], row-major 3x3 reciprocal
 * box R[j][d] = recip[3 j + d], the inverse of the matrix whose rows are the box vectors, so that
 * the fractional coordinate along d is sum_j x_j R[j][d].  A diagonal recip is the reference's
 * orthorhombic case (CudaPMERecip.cu:2042-2045) and must be positive; off-diagonals select the
 * triclinic forms of spread, solve and gather (an extension: the reference exits on them), which
 * need a finite, non-singular matrix.  Anything else returns PME_EINVAL. */
PME_API int pme_spread_charge(pme_recip* h, const void* xyzq, int ncoord, const double* recip);
PME_API int pme_r2c_fft(pme_recip* h);
PME_API int pme_scalar_sum(pme_recip* h, const double* recip, double kappa, int calc_energy,
                   int calc_virial);
PME_API int pme_c2r_fft(pme_recip* h);
/* gather_force<FT>: force is a device pointer of the kind's element type. */
PME_API int pme_gather_force(pme_recip* h, const void* xyzq, int ncoord, const double* recip, int stride,
                     int kind, void* force);
PME_API int pme_calc_self_energy(pme_recip* h, const void* xyzq, int ncoord, double kappa);

/* ---- energy / virial record (CudaEnergyVirial.h:13-53) ---- */
PME_API int pme_clear_energy_virial(pme_recip* h);                 /* async memset on the stream */
/* Synchronises the stream, then copies.  Any output pointer may be NULL. */
PME_API int pme_get_energy_virial(pme_recip* h, double* energy_recip, double* energy_self,
                          double* virial9);
/* Enqueue a copy of the record (double[PME_EV_COUNT]) to dst (host pinned or device memory)
 * on the stream, without synchronising. */
PME_API int pme_copy_energy_virial_async(pme_recip* h, double* dst);
/* Device address of the record: double[PME_EV_COUNT]. */
PME_API int pme_energy_virial_device_ptr(pme_recip* h, double** dev_ptr);
/* Opt-in (no counterpart in the reference): every later fused evaluation (pme_eval,
 * pme_eval_ortho) also stores its own record [E_recip, E_self, W_xx .. W_zz] (not the accumulated
 * one; zeros for terms not asked for) at host_mapped, pinned host memory mapped at the same
 * address (cudaHostAlloc / cudaMallocHost with unified addressing), readable once the stream has
 * passed the evaluation.  The device record accumulates as before.  NULL turns it off. */
PME_API int pme_set_energy_virial_mirror(pme_recip* h, double* host_mapped);

/* ---- fused evaluation: the CudaDomdecRecip::calc sequence (CudaDomdecRecip.h:17-81) ----
 * spread, R2C, scalar sum (energy/virial if asked), C2R, gather into `force` of `kind`, and the
 * self energy when calc_energy.  Energy/virial ACCUMULATE into the record.  Same results as the
 * staged calls, bit for bit. */
PME_API int pme_eval_ortho(pme_recip* h, double inv_boxx, double inv_boxy, double inv_boxz,
                   const void* xyzq, int ncoord, double kappa, int calc_energy, int calc_virial,
                   int kind, void* force, int stride);
/* The same for any box: recip as for pme_spread_charge (orthorhombic or triclinic).  With a
 * diagonal recip it is pme_eval_ortho.  No counterpart in the reference, which only takes
 * orthorhombic boxes (CudaDomdecRecip.h:20-23 builds a diagonal recip). */
PME_API int pme_eval(pme_recip* h, const double* recip, const void* xyzq, int ncoord, double kappa,
                   int calc_energy, int calc_virial, int kind, void* force, int stride);
/* pme_eval from and to host buffers: xyzq_host is page-locked host memory mapped at the same
 * address (cudaHostAlloc / cudaMallocHost with unified addressing), which the evaluation reads
 * directly over the bus, in index order, while it bins the atoms; force_host is page-locked host
 * memory that receives the forces by one copy on the handle's stream after the evaluation (for
 * PME_FORCE_F32_SOA only the ncoord entries of each of the three rows).  Float kinds only
 * (PME_EUNSUPPORTED for PME_FORCE_I64_SOA_ACCUM); PME_EINVAL for memory that is not page-locked.
 * Asynchronous: the forces are in force_host once the stream has passed the call.  Same results
 * as pme_eval bit for bit.  No counterpart in the reference, whose calls take device buffers. */
PME_API int pme_eval_host(pme_recip* h, const double* recip, const void* xyzq_host, int ncoord,
                          double kappa, int calc_energy, int calc_virial, int kind, void* force_host,
                          int stride);

/* ---- fixed-point force conversion (Force<long long>, Force.cu:103-190) ----
 * An MD step accumulates reciprocal (PME_FORCE_I64_SOA_ACCUM), direct and 1-4 forces into one
 * int64 SoA array at scale 2^40 and converts it once (CudaPMEForcefield.cu:514).  Every value
 * becomes the int64 rounded once to the output type times 2^-40 (exact), i.e. the reference's
 * ((T)v) * INV_FORCE_SCALE (reduce.cu:15-53).  Only the ncoord entries of each of the three rows
 * are read and written (stride padding is left alone).  Asynchronous on `stream`. */
enum { PME_REAL_F32 = 0, PME_REAL_F64 = 1 };
/* Force<long long>::convert<T2>(Force<T2>&) (Force.cu:103-128): rows at in + k in_stride to rows
 * at out + k out_stride of out_type.  out == in converts in place (PME_REAL_F64 and the same
 * stride only), as Force<long long>::convert<double>() (Force.cu:143-157); other overlaps are
 * PME_EINVAL. */
PME_API int pme_force_convert(const long long* in, int in_stride, int ncoord, void* out, int out_stride,
                              int out_type, void* stream);
/* Force<long long>::convert_add<double, T>(Force<T>&) (Force.cu:167-184, reduce.cu:152-170): in
 * place, each int64 entry v of inout becomes the double v 2^-40 + add, with add float or double
 * (add_type) SoA rows at add + k add_stride. */
PME_API int pme_force_convert_add(long long* inout, int stride, int ncoord, const void* add, int add_stride,
                                  int add_type, void* stream);

/* ---- recip-node request loop (CudaDomdecRecipLooper::run, CudaDomdecRecipLooper.cu:3-36) ----
 * The loop of a pure reciprocal-space node: receive a header (DomdecRecipComm.h:11-15), stop on
 * a negative coordinate count, receive the coordinates, evaluate (pme_eval_ortho into a float3
 * force buffer that grows with the count, as reallocate<float3> does), send the forces, repeat.
 * The transport is the caller's, as callbacks (the role of CudaDomdecRecipComm); each returns 0
 * on success, anything else ends the loop with PME_ESTATE. */
typedef struct {
  double inv_boxx, inv_boxy, inv_boxz;   /* inverse box edges (1/A) */
  int ncoord;                            /* coordinates of this step; < 0: STOP */
  int calc_energy, calc_virial;
} pme_recip_header;

typedef struct {
  void* user;                            /* passed back to every callback */
  int (*recv_header)(void* user, pme_recip_header* header);
  /* The step's coordinates: *xyzq = a device float4[ncoord] (the callback may copy them there
   * on `stream`, the handle's stream, which the evaluation then follows). */
  int (*recv_coord)(void* user, int ncoord, void* stream, const void** xyzq);
  /* After the step (stream synchronised): force = device float3[ncoord] (+dE/dx, overwritten by
   * the next step), energy_virial = host double[PME_EV_COUNT], this step's own record. */
  int (*send_force)(void* user, int ncoord, const void* force, const double* energy_virial);
} pme_recip_comm;

/* Runs the loop on the handle (its grid, order and stream) with Ewald kappa until STOP; *steps
 * (may be NULL) receives the number of steps served.  Synchronous. */
PME_API int pme_recip_loop_run(pme_recip* h, double kappa, const pme_recip_comm* comm, long long* steps);

/* ---- grid read-back for parity checks (synchronise the stream; host outputs) ----
 * Layouts follow the reference: real grids [z][y][x]; half-complex grid [z][y][kx],
 * kx = 0..nfftx/2, interleaved (re, im). */
PME_API int pme_copy_charge_grid_fixed(pme_recip* h, long long* host_out);   /* nx*ny*nz int64, 2^40 */
PME_API int pme_copy_charge_grid(pme_recip* h, float* host_out);             /* nx*ny*nz float */
PME_API int pme_copy_fft_grid(pme_recip* h, float* host_out);                /* 2*(nx/2+1)*ny*nz float */
PME_API int pme_copy_solved_grid(pme_recip* h, float* host_out);             /* nx*ny*nz float */
/* Replace the accumulated charge grid (e.g. to test the transforms on a known grid): host
 * float nx*ny*nz values rounded to the 2^40 fixed point; synchronous. */
PME_API int pme_load_charge_grid(pme_recip* h, const float* host_in);

/* ---- device status of the fused evaluation ----
 * The fused evaluation (pme_eval_ortho) runs as one cooperative kernel whose grid barriers wait
 * at most a bounded number of polls.  If a wait gives up, the kernel stops early, leaves a sticky
 * status on the device and later evaluations do nothing until it is cleared.  pme_get_status
 * synchronises the stream, reports the status (PME_ETIMEOUT if a wait gave up) and clears it,
 * together with the barrier words and the accumulation grid, so the handle is usable again. */
PME_API int pme_get_status(pme_recip* h, int* device_status);
PME_API int pme_set_barrier_spin_limit(pme_recip* h, unsigned int polls);   /* default 2^22 */
/* The fused evaluation bins atoms by grid row block; its bin storage grows (synchronously) the
 * first time a call has more atoms than any earlier one.  Call this with the largest atom count
 * before capturing evaluations in a CUDA graph, so that no capture needs to allocate. */
PME_API int pme_reserve_atoms(pme_recip* h, int natom);
/* Schedule of the fused evaluation's y/z transforms: PME_SCHED_PLANES runs y, z and the solve
 * as whole-plane tiles (one CTA per kx plane, where a plane fits in shared memory),
 * PME_SCHED_PASSES as separate y and z passes (more, smaller tiles), PME_SCHED_CLUSTER as kx
 * planes split over a cluster of 4 CTAs (y lines and z lines exchanged through distributed shared
 * memory; single systems in the latency build, orthorhombic boxes, ny and nz multiples of 4, else
 * passes), PME_SCHED_AUTO (default) picks planes when there are at least as many planes as SMs,
 * else the cluster form where it applies and there are at least 32 planes, else passes.  Results
 * are identical. */
enum { PME_SCHED_AUTO = 0, PME_SCHED_PLANES = 1, PME_SCHED_PASSES = 2, PME_SCHED_CLUSTER = 3 };

/* ---- autotuner ----
 * No counterpart in the reference (its launch shapes are fixed).  The fused evaluation's launch
 * shape: the y/z schedule, the lines of the x-, y- and z-pass tiles and the number of CTAs of the
 * persistent launch.  Every shape gives the same results bit for bit; only the time differs.
 * pme_autotune measures candidate shapes on the caller's own system (coordinates, box, kappa as
 * for pme_eval_ortho) by coordinate descent, `reps` timed evaluations per candidate, keeps the
 * fastest in the handle and in a process-wide cache keyed by (device, grid, order) that later
 * pme_create calls of the same key start from.  It synchronises the stream, allocates a
 * temporary force buffer and leaves the energy/virial record as it found it. */
typedef struct {
  int schedule;        /* PME_SCHED_* */
  int x_lines;         /* grid lines per x-pass tile */
  int y_lines;         /* grid lines per y-pass tile */
  int z_columns;       /* grid columns per z-pass tile */
  int grid_ctas;       /* CTAs of the persistent launch; 0 = as many as are resident */
  float us_per_eval;   /* measured time of this shape (pme_autotune), else 0 */
  int candidates;      /* shapes measured (pme_autotune), else 0 */
} pme_tune_config;

PME_API int pme_autotune(pme_recip* h, const void* xyzq, int ncoord, double inv_boxx, double inv_boxy,
                         double inv_boxz, double kappa, int reps, pme_tune_config* out);
PME_API int pme_get_tune_config(const pme_recip* h, pme_tune_config* out);
/* Set a shape explicitly (checked against the shared-memory limits; PME_EINVAL if it does not fit). */
PME_API int pme_set_tune_config(pme_recip* h, const pme_tune_config* cfg);
PME_API int pme_tune_cache_clear(void);
PME_API int pme_set_fft_schedule(pme_recip* h, int schedule);

/* Where the fused evaluation runs the inverse x pass.  AUTO (default): inside the gather tiles,
 * each transforming the rows its atoms reach (halo rows again for every tile that reaches them),
 * when those rows fit in the shared memory the other phases take (each tile also stores its own
 * rows, so the solved grid is complete afterwards, as the staged calls expect).  OFF: as a phase
 * of its own before the gather.  Results are identical bit for bit; only the time differs. */
enum { PME_XGATHER_AUTO = 0, PME_XGATHER_OFF = 1 };
PME_API int pme_set_x_gather_fusion(pme_recip* h, int mode);

/* Test hook for failure detection: PME_INJECT_SKIP_BARRIER makes CTA 0 of the next fused
 * evaluations leave before the first grid barrier, so the other CTAs' bounded waits run out
 * (no fault, no hang).  PME_INJECT_NONE turns it off. */
enum { PME_INJECT_NONE = 0, PME_INJECT_SKIP_BARRIER = 1 };
PME_API int pme_set_fault_injection(pme_recip* h, int what);

/* Profiling hook: while set, every fused evaluation writes, for each CTA c < max_ctas and each of
 * its 7 phases p (spread, x fwd, y fwd, z fwd+solve+inv, y inv, x inv, gather), the %globaltimer
 * (ns) at the phase's start and end to dev_buf[(c * 7 + p) * 2 + {0, 1}] (device memory,
 * max_ctas * 14 entries), followed by 32 entries of step stamps inside CTA 0's first tiles.
 * NULL turns it off. */
PME_API int pme_set_trace(pme_recip* h, unsigned long long* dev_buf, int max_ctas);

/* ---- batches: many independent systems in one persistent launch ----
 * Each system has its own grid, spline order, box, kappa, coordinates and force output; all
 * device state (grids, plans, moduli, records) is allocated once at creation, so repeated
 * evaluations allocate nothing.  This path has no counterpart in the reference (which evaluates
 * one system per CudaPMERecip instance). */
typedef struct pme_batch pme_batch;
typedef struct {
  int nfftx, nffty, nfftz, order;
  int natom;
  double box[3];          /* orthorhombic box edges (A) */
  double kappa;
  const void* xyzq;       /* device float4[natom] */
  void* force;            /* device output of force_kind */
  int force_kind;
  int stride;             /* SoA stride (>= natom) for PME_FORCE_F32_SOA / I64 kinds */
  int calc_energy, calc_virial;
} pme_system_desc;

PME_API int pme_batch_create(const pme_system_desc* systems, int nsys, void* stream, pme_batch** out);
PME_API int pme_batch_destroy(pme_batch* b);
PME_API int pme_batch_set_stream(pme_batch* b, void* stream);
/* Change one system's box (NULL keeps it), coordinates or force pointer (NULL keeps them);
 * takes effect at the next pme_batch_commit. */
PME_API int pme_batch_set_system(pme_batch* b, int sys, const double* box3, const void* xyzq, void* force);
PME_API int pme_batch_commit(pme_batch* b);      /* uploads descriptors (synchronises the stream) */
PME_API int pme_batch_eval(pme_batch* b);        /* one launch: every system, every stage */
PME_API int pme_batch_clear_energy_virial(pme_batch* b);
/* Synchronises; out = nsys * PME_EV_COUNT doubles, system-major. */
PME_API int pme_batch_get_energy_virial(pme_batch* b, double* out);
PME_API int pme_batch_info(const pme_batch* b, int* nsys, int* grid_ctas, size_t* device_bytes);
PME_API int pme_batch_set_trace(pme_batch* b, unsigned long long* dev_buf, int max_ctas);
/* Autotune the batch's launch: the y/z schedule of every system (planes where they fit, or
 * passes), the lines per x/y/z pass tile (each system's default times 1, 2 or 4, within the
 * shared-memory budget) and the CTAs of the launch, `reps` timed evaluations per candidate; the
 * fastest is kept (and committed).  The evaluations write the systems' force outputs as
 * pme_batch_eval does (int64 outputs accumulate every tuning evaluation: clear them afterwards);
 * the energy/virial records are left as they were.  out may be NULL; out->x_lines, y_lines and
 * z_columns hold the chosen multiplier. */
PME_API int pme_batch_autotune(pme_batch* b, int reps, pme_tune_config* out);
/* Device bytes one system of this grid occupies (for admission by HBM footprint). */
PME_API size_t pme_system_device_bytes(int nfftx, int nffty, int nfftz);

/* ---- request server: continuous batching of PME evaluations ----
 * No counterpart in the reference, whose CudaDomdecRecipLooper (CudaDomdecRecipLooper.cu:3-36)
 * serves one system's evaluations at a time.  A server owns a device arena of device_bytes and a
 * worker thread.  A request is one orthorhombic system and n_evals evaluations of it; evaluation k
 * uses the submitted coordinates plus sigma * N(0,1) per coordinate, drawn from (seed, k, atom,
 * axis), so a request's results depend only on the request.  Requests are admitted in arrival
 * order while fewer than max_active run and their device footprint (pme_request_device_bytes)
 * fits in the arena; every step evaluates the next evaluation of all running requests in one
 * fused launch; requests that arrive meanwhile join at the next step.  A request's grids, moduli,
 * bins and bin-sorted atom order stay on the device for all its evaluations. */
typedef struct pme_server pme_server;
typedef struct {
  int nfftx, nffty, nfftz, order;
  int natom;
  double box[3];            /* orthorhombic box edges (A) */
  double kappa;
  const float* xyzq;        /* host float[natom][4]; copied by pme_server_submit */
  int n_evals;              /* >= 1 */
  float sigma;              /* coordinate jitter (A) of every evaluation; 0 = none */
  unsigned long long seed;
  int calc_energy, calc_virial;
  double* ev_out;           /* host n_evals * PME_EV_COUNT doubles: each evaluation's record */
  float* force_out;         /* host natom * 3 floats (x, y, z per atom) of the last evaluation, or NULL */
} pme_request;

typedef struct {
  long long submitted, completed, evals, steps, active, pending;
  size_t arena_bytes, arena_used;
  double seconds;           /* since the server was created */
} pme_server_stats;

/* stream NULL: the server makes its own non-blocking stream. */
PME_API int pme_server_create(size_t device_bytes, int max_active, void* stream, pme_server** out);
/* Finishes every admitted and pending request, then releases everything. */
PME_API int pme_server_destroy(pme_server* s);
PME_API size_t pme_request_device_bytes(const pme_request* r);   /* 0 if the request is invalid */
/* Queue a request (PME_ENOMEM if it can never fit in the arena); the host buffers ev_out and
 * force_out must stay valid until pme_server_wait for its id returns. */
PME_API int pme_server_submit(pme_server* s, const pme_request* r, long long* id);
/* Block until request `id` is done (timeout_s < 0: no limit); its results are then in ev_out /
 * force_out; times3 (may be NULL) receives its submit, admission and completion times (seconds
 * since the server was created).  Each id can be waited for once. */
PME_API int pme_server_wait(pme_server* s, long long id, double timeout_s, double* times3);
PME_API int pme_server_get_stats(pme_server* s, pme_server_stats* out);

/* ---- spreading without device allocation ----
 * No counterpart in the reference.  For callers that must not allocate device memory when they
 * need a charge grid: hosts whose own memory manager owns all device memory and forbids plug-ins
 * to call cudaMalloc, and latency-critical loops that cannot take allocator locks or let an
 * allocation synchronise the device.  Same spreading kernel and exact int64 fixed-point
 * accumulation as pme_spread_charge, but the accumulation grid is a fixed array compiled into
 * this library (8 MiB on every GPU that loads it, held until the process exits, so
 * nfftx*nffty*nfftz <= 1048576; larger grids return PME_EINVAL).  The caller passes the
 * coordinates (device float4[ncoord]), the host recip[9] (orthorhombic: a positive diagonal,
 * off-diagonals return PME_EINVAL) and the output: grid_out, a device float[nfftz][nffty][nfftx]
 * that receives the converted charge grid.  Asynchronous on `stream`; it calls no cudaMalloc or
 * cudaFree.  The first call on a device (and the first after that device's context was replaced,
 * e.g. by cudaDeviceReset) looks up the array's device address (cudaGetSymbolAddress): make it
 * before any stream capture.  All calls share the array and each clears it before use: calls
 * whose work overlaps on the GPU race and corrupt each other's grid. */
PME_API int pme_spread_charge_noalloc(const void* xyzq, int ncoord, const double* recip, int nfftx,
                                      int nffty, int nfftz, int order, float* grid_out, void* stream);

/* ---- errors / version ---- */
PME_API const char* pme_last_error_string(void);     /* thread-local message of the last failure */
PME_API const char* pme_status_string(int status);
PME_API int pme_version(void);                       /* 10000*major + 100*minor + patch */

#ifdef __cplusplus
}
#endif

#endif /* PME_RECIP_H */

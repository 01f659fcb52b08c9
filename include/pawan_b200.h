/* pawan_b200 -- C ABI of the B200 (sm_100a) implementation of pawan's hot
 * path: the all-pairs vortex-particle interaction and the RK4 integration
 * that drives it.
 *
 * Plain C types only (pointers, sizes, doubles); no CUDA or C++ types cross
 * this boundary.  Every call returns a status (PAWAN_OK == 0); the text of the
 * last failure on a context is pawan_ctx_last_error().  No C++ exception
 * crosses the ABI.  Host pointers are borrowed for the duration of the call
 * only.  A context is used from one host thread at a time (the serving
 * engine runs its own worker thread on a context it owns).
 *
 * Layout conventions (the reference's, src/wake/wake.cpp:87-120):
 *   - a system's particles are the union of its wakes in wake order;
 *   - position / vorticity arrays are N x 3 row-major doubles;
 *   - a state or rate vector has size 6*N ("_size", src/system/system.h:22)
 *     and holds, per wake, [x (N_w x 3) | alpha (N_w x 3)], wakes concatenated
 *     (src/interaction/interaction.cpp:204-229).
 *
 * Each entry point names the reference interface it replaces.
 */
#ifndef PAWAN_B200_H
#define PAWAN_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------ status codes */
#define PAWAN_OK 0
#define PAWAN_ERR_INVALID 1     /* bad argument, size or handle */
#define PAWAN_ERR_CUDA 2        /* CUDA runtime error (text in last_error) */
#define PAWAN_ERR_NOMEM 3       /* device or host allocation failed */
#define PAWAN_ERR_STATE 4       /* call not valid in the object's state */
#define PAWAN_ERR_BUDGET 5      /* serving: request can never fit the budget */
#define PAWAN_ERR_TIMEOUT 6     /* serving: wait ran out */
#define PAWAN_ERR_NOTFOUND 7    /* serving: unknown request id */
#define PAWAN_ERR_REJECTED 8    /* serving: queue full or engine stopped */

/* ---------------------------------------------------------- pair precision */
#define PAWAN_PREC_F32 0        /* FP32 pair math, FP64 per-tile accumulation */
#define PAWAN_PREC_F64 1        /* FP64, same algebra as the FP32 kernel */
#define PAWAN_PREC_F64_PLAIN 2  /* FP64, the reference's formula term by term */

/* Tiling of the pair kernel (the compiled variants are listed by
 * pawan_system_autotune's candidates; set_tiling rejects others). */
typedef struct {
  int threads;            /* threads per block = sources per shared-memory tile: 128 or 256 */
  int threads_per_target; /* threads sharing one target's sources: 1, 2 or 4 */
  int targets_per_thread; /* targets per thread: 1 or 2 */
  int unroll;             /* unroll depth of the source loop */
  int blocks_per_sm;      /* blocks per SM the registers are bounded for, 0 = default */
  int items_per_slot;     /* work items per resident block (source chunking) */
  int packed;             /* far tiles two sources per FP32x2 instruction: 1 with
                             1/rho^2 from the MUFU reciprocal, 2 from rsqrt
                             squared; 0: one source per instruction */
  int split_near;         /* FP32: 1 computes the near tile pairs in a pass of
                             their own before the far pass (each kernel with its
                             own registers; faster where near pairs are many),
                             2 the same with the near pass two sources per
                             FP32x2 instruction; 0: one pass */
} pawan_tiling;

typedef struct pawan_ctx pawan_ctx;
typedef struct pawan_system pawan_system;
typedef struct pawan_batch pawan_batch;
typedef struct pawan_server pawan_server;

/* ---------------------------------------------------------------- context */
/* One device, one stream.  No reference counterpart: the reference has no
 * device state. */
int pawan_ctx_create(int device, pawan_ctx **out);
void pawan_ctx_destroy(pawan_ctx *ctx);
const char *pawan_ctx_last_error(const pawan_ctx *ctx);
const char *pawan_status_name(int status);
/* sm_count, compute capability, total device memory in bytes. */
int pawan_ctx_info(pawan_ctx *ctx, int *sm_count, int *cc_major, int *cc_minor,
                   size_t *total_mem);
int pawan_ctx_synchronize(pawan_ctx *ctx);
/* Number of this library's kernels launched on the context so far. */
unsigned long long pawan_ctx_launch_count(const pawan_ctx *ctx);
/* Time every pair-kernel launch with CUDA events on the launching stream. */
int pawan_ctx_profile(pawan_ctx *ctx, int enable);
/* Totals since profiling was (re)enabled: summed pair-kernel time (ms),
 * pair launches, and pair interactions counted as N^2 per solve per launch. */
int pawan_ctx_profile_read(pawan_ctx *ctx, double *pair_ms, unsigned long long *pair_launches,
                           double *pair_interactions);
/* The same for the per-particle stage kernel (RK4 stage update and repack):
 * summed time (ms), launches, and algorithmic HBM bytes (what each launch must
 * read and write: the summed rates, FP64 state vectors, packed tile data). */
int pawan_ctx_profile_stage(pawan_ctx *ctx, double *stage_ms, unsigned long long *stage_launches,
                            double *stage_bytes);
/* Timing marks on the context's stream (CUDA events, slots 0..15) and the
 * device time between two of them, in ms (waits for the later mark). */
int pawan_ctx_mark(pawan_ctx *ctx, int slot);
int pawan_ctx_elapsed(pawan_ctx *ctx, int slot0, int slot1, double *ms);
/* Overwrites `bytes` of device scratch on the context's stream, evicting the
 * L2 cache between timed iterations. */
int pawan_ctx_flush_l2(pawan_ctx *ctx, size_t bytes);
/* Pinned host memory (for host<->device copies at full bandwidth). */
int pawan_host_alloc(pawan_ctx *ctx, size_t bytes, void **out);
int pawan_host_free(pawan_ctx *ctx, void *ptr);

/* ----------------------------------------------------------------- system */
/* A system is the reference's __interaction (src/interaction/interaction.h:21-235)
 * with its wakes: all-pairs over the union of the wakes, viscosity nu.
 * Replaces __interaction(W) / __interaction(W1,W2) / addWake
 * (interaction.cpp:11-39) and __parallel(W), __parallel(W1,W2)
 * (src/interaction/parallel.cpp:10-11).  The reference hard-codes
 * nu = 2.5e-3 (interaction.cpp:13); here it is an argument. */
int pawan_system_create(pawan_ctx *ctx, size_t n_wakes, const size_t *num_particles, double nu,
                        int precision, pawan_system **out);
void pawan_system_destroy(pawan_system *sys);
/* __system::_size (src/system/system.h:22): 6 * total particles. */
size_t pawan_system_size(const pawan_system *sys);
size_t pawan_system_num_particles(const pawan_system *sys);
/* Particle data of all wakes (union, N x 3 / N): the fields of __wake
 * (src/wake/wake.h:35-41) that the interaction reads. */
int pawan_system_set_particles(pawan_system *sys, const double *position, const double *vorticity,
                               const double *radius, const double *volume);
/* __interaction::setStates / getStates (interaction.cpp:204-211, 222-229). */
int pawan_system_set_states(pawan_system *sys, const double *state, size_t size);
int pawan_system_get_states(pawan_system *sys, double *state, size_t size);
/* __interaction::solve -> interact() (interaction.cpp:41-43, 95-108) and
 * __parallel::interact (parallel.cpp:13-85): velocity and vorticity rate of
 * every particle.  Asynchronous; read the result with get_rates. */
int pawan_system_solve(pawan_system *sys);
/* __interaction::getRates (interaction.cpp:213-220): [u | dalpha] per wake. */
int pawan_system_get_rates(pawan_system *sys, double *rate, size_t size);
/* W->_velocity and W->_retvorcity of one wake (N_w x 3 each; wake.h:36,38). */
int pawan_system_get_wake_rates(pawan_system *sys, size_t wake, double *velocity,
                                double *retvorcity);
/* nsteps of __rk4::step (src/integration/rk4.cpp:12-76), state kept on the
 * device between steps; read it back with get_states. */
int pawan_system_rk4(pawan_system *sys, double dt, size_t nsteps);
/* The same with the step's four (pair, stage) launch pairs captured once in a
 * CUDA graph and replayed per step (bit-identical to pawan_system_rk4; the
 * pair launches are not timed by pawan_ctx_profile). */
int pawan_system_rk4_graph(pawan_system *sys, double dt, size_t nsteps);
/* nsteps of __integration::step (src/integration/integration.cpp:37-45). */
int pawan_system_euler(pawan_system *sys, double dt, size_t nsteps);
/* __interaction::diagnose (interaction.cpp:49-93), FP64 on the device.
 * out[0..2] total vorticity, [3..5] linear impulse, [6..8] angular impulse,
 * [9] enstrophy, [10] helicity.  quadratic = 0 skips the O(N^2) terms
 * (out[9], out[10] then 0). */
int pawan_system_diagnose(pawan_system *sys, double *out, int quadratic);
/* Smoothing kernel: PAWAN_KERNEL_HIGHORDER (src/interaction/highorder.h, the
 * reference's default) or PAWAN_KERNEL_GAUSSIAN (src/interaction/gaussian.h,
 * which the reference selects with #define GAUSSIAN 1 in
 * interaction_utils.h:13-24).  Applies to solve, RK4/Euler, diagnostics (with
 * the Gaussian kernel the enstrophy is 0, as the reference's ENST stub
 * returns, gaussian.h:67-86) and the vorticity field.  Systems of one batch
 * share their kernel; the serving engine and pawan_interact_noalloc use the
 * high-order kernel. */
#define PAWAN_KERNEL_HIGHORDER 0
#define PAWAN_KERNEL_GAUSSIAN 1
int pawan_system_set_kernel(pawan_system *sys, int kernel);
int pawan_system_get_kernel(pawan_system *sys, int *kernel);
/* calculateKineticEnergy over all wakes (interaction.cpp:351-383). */
int pawan_system_kinetic_energy(pawan_system *sys, double *ke);
/* __interaction::resolve -> influence (interaction.cpp:45-47, 110-155): the
 * smoothed vorticity field of every particle, FP64 on the device, into
 * `field` (3N doubles, the wakes' _vorticityfield rows in wake order).  The
 * influence-matrix path of __resolve::rebuild (src/resolve/resolve.cpp:10-57)
 * calls it once per state component. */
int pawan_system_influence(pawan_system *sys, double *field, size_t size);
/* The vorticity field of ncols strength vectors at once, over the system's
 * current positions and radii: alpha holds ncols blocks of N x 3 doubles
 * (wake order, the rows of every wake's _vorticity), field receives the same
 * shape (size = ncols * 3N for both).  These are the influence-matrix columns
 * of __resolve::rebuild (resolve.cpp:19-31), which differ only in strength;
 * each column is bit-identical to pawan_system_influence with that strength.
 * The system's own strengths are not changed. */
int pawan_system_influence_columns(pawan_system *sys, size_t ncols, const double *alpha,
                                   double *field, size_t size);
/* The protected __interaction::_nu (interaction.h:24). */
int pawan_system_set_nu(pawan_system *sys, double nu);
int pawan_system_set_precision(pawan_system *sys, int precision);
/* Appends (append != 0) or writes one .wake frame: t (f64), nWake (size_t),
 * then per wake N (size_t), position (N x 3 f64), vorticity (N x 3 f64),
 * radius (N f64): __integration::integrate's per-step output
 * (integration.cpp:20-21, 28-29; interaction.cpp:197-202; wake.cpp:68-73). */
int pawan_system_write_frame(pawan_system *sys, const char *path, double t, int append);
/* __integration::integrate (src/integration/integration.cpp:16-35): n steps of
 * dt = T/n -- RK4 as __rk4::step (PAWAN_INTEGRATE_RK4) or Euler as
 * __integration::step (PAWAN_INTEGRATE_EULER) -- with a .wake frame at t = 0 and
 * after every step at t = i*dt, in the reference's frame format, written to
 * `path` (created or truncated).  The steps stay on the device; each frame is
 * copied out through a pinned ring and written by a background thread while
 * the next steps run.  The _file variant writes to an open FILE* (a
 * `FILE *` of the caller's C library, e.g. from __io::create_binary_file, which
 * stays open). */
#define PAWAN_INTEGRATE_RK4 0
#define PAWAN_INTEGRATE_EULER 1
int pawan_system_integrate(pawan_system *sys, double T, size_t n, const char *path, int method);
int pawan_system_integrate_file(pawan_system *sys, double T, size_t n, void *file, int method);
int pawan_system_set_tiling(pawan_system *sys, const pawan_tiling *tiling);
int pawan_system_get_tiling(pawan_system *sys, pawan_tiling *tiling);
/* Times the candidate tilings and chunkings on this system -- each one
 * right-hand side as an RK4 stage runs it: the pair launch and the reduction
 * of its chunk partials -- and keeps the fastest.  The state is unchanged; the
 * last rates (pawan_system_get_rates) are left as those of the current state,
 * computed with one of the candidates. */
int pawan_system_autotune(pawan_system *sys);
/* The tilings pawan_system_autotune / pawan_batch_autotune time for a
 * precision and smoothing kernel (each at the default chunking): *count is
 * their number, the first min(cap, *count) are written to out.  The
 * autotuner then times the chunkings pawan_tile_chunkings lists
 * (items_per_slot) for the fastest.  Host-only; no device needed. */
int pawan_tile_candidates(int precision, int kernel, pawan_tiling *out, size_t cap, size_t *count);
int pawan_tile_chunkings(int *out, size_t cap, size_t *count);
/* Device-side snapshot of the state (checkpoint) and its restore, for
 * resuming a run or repeating steps from one state.  The reference's
 * file-based save()/read() (src/wake/wake.cpp:58-85) is the on-disk
 * counterpart; pawan_system_write_frame writes the .wake frames. */
int pawan_system_checkpoint(pawan_system *sys);
int pawan_system_restore(pawan_system *sys);
/* Device address of the state [x | alpha] in union layout (6N doubles,
 * x = first 3N) for callers that keep data on the device. */
int pawan_system_device_state(pawan_system *sys, double **state);

/* ------------------------------------------------------- target sharding */
/* One system over `world` processes, one GPU each.  No reference counterpart
 * (the reference runs in one process); the reference's OpenMP path splits the
 * targets of each source over threads (parallel.cpp:21), this splits them
 * over GPUs.  Every process holds the whole state.  Process `rank` computes the
 * rates of its block of targets [rank*S, min(N, (rank+1)*S)), S =
 * pawan_shard_size(N, world) (a multiple of 512); the blocks are exchanged
 * through caller-owned device buffers -- `send` (6*S doubles: this process's
 * block) and `recv` (6*S*world doubles: every block in rank order, each laid
 * out [6][S]) -- by an all-gather of send into recv on every process (e.g.
 * torch.distributed / NCCL), ordered on the library's stream between the two
 * calls below.  Every process then applies the same update to all N
 * particles, so the states stay identical across processes.  One RK4 step:
 * for stage in 1..4 { shard_rates; all-gather; shard_stage(stage) }.
 * world = 0 clears the sharding; a sharded system refuses the unsharded
 * solve / rk4 / euler and batches. */
size_t pawan_shard_size(size_t n, int world);
int pawan_system_set_shard(pawan_system *sys, int rank, int world, double *send, double *recv);
/* Pair kernel over this process's targets, its block of rates into send. */
int pawan_system_shard_rates(pawan_system *sys);
/* After the all-gather: stage 1..4 of an RK4 step (rk4.cpp:24-66) for every
 * particle from the gathered rates; stage 0 stores the rates (as a solve()). */
int pawan_system_shard_stage(pawan_system *sys, int stage, double dt);
/* The context's CUDA stream (cudaStream_t), for ordering a caller's
 * collective with the library's kernels. */
int pawan_ctx_stream(pawan_ctx *ctx, void **stream);

/* ------------------------------------------------------------------ batch */
/* Many independent systems in one persistent pair launch per RK4 stage
 * (ragged segments), the four stages optionally captured in a CUDA graph.
 * No reference counterpart (the reference integrates one system at a time).
 * Each system's result matches its own pawan_system_rk4 result up to the
 * FP64 rounding of how its source chunks are grouped; graph and non-graph
 * runs of one batch agree bit for bit. */
int pawan_batch_create(pawan_ctx *ctx, size_t n, pawan_system *const *systems, pawan_batch **out);
void pawan_batch_destroy(pawan_batch *batch);
/* dt[i] for system i (NULL: every system uses dt0). */
int pawan_batch_rk4(pawan_batch *batch, const double *dt, double dt0, size_t nsteps,
                    int use_graph);
int pawan_batch_solve(pawan_batch *batch);
int pawan_batch_set_tiling(pawan_batch *batch, const pawan_tiling *tiling);
/* The same over the batch's systems together. */
int pawan_batch_autotune(pawan_batch *batch);

/* ---------------------------------------------------------------- serving */
/* A request loop with device-resident state and continuous batching: each
 * engine iteration advances every admitted request by one or more RK4 steps
 * (as many as fit in iteration_seconds of device work without passing any
 * active request's last step), one batched launch sequence per step (a CUDA
 * graph per plan when it runs several); requests that
 * arrive meanwhile are admitted when the HBM budget and the per-iteration
 * work cap allow.  The engine takes request memory from the device's default
 * memory pool (stream-ordered) and keeps freed memory there until it is
 * destroyed.  No reference counterpart. */
typedef struct {
  double budget_bytes;          /* device memory the admitted requests may hold */
  double max_step_interactions; /* cap on sum N^2 of the requests in one iteration (0: none) */
  int max_active;               /* cap on admitted requests (0: none) */
  int max_queue;                /* waiting requests beyond this are rejected (0: none) */
  int precision;                /* PAWAN_PREC_* */
  double iteration_seconds;     /* device time one iteration may take before new arrivals
                                   are admitted (0: 20 ms; tiny: one step per iteration) */
  int policy;                   /* admission order: PAWAN_SERVE_FIFO (arrival) or
                                   PAWAN_SERVE_SHORTEST_FIRST (least N^2 x steps first; under
                                   overload large requests can wait indefinitely) */
} pawan_serve_config;

#define PAWAN_SERVE_FIFO 0
#define PAWAN_SERVE_SHORTEST_FIRST 1

typedef struct {
  unsigned long long submitted, admitted, completed, rejected, queued, active;
  unsigned long long iterations;
  double interactions;          /* pair interactions computed (N^2 per solve per RHS) */
  double busy_seconds;          /* wall time the engine spent in iterations */
  double bytes_in_use;
  double admit_seconds;         /* engine time creating and uploading admitted requests */
  double plan_seconds;          /* engine time building batched plans */
  double retire_seconds;        /* engine time copying out and releasing finished requests */
} pawan_serve_stats;

#define PAWAN_REQ_QUEUED 0
#define PAWAN_REQ_ACTIVE 1
#define PAWAN_REQ_DONE 2
#define PAWAN_REQ_REJECTED 3
#define PAWAN_REQ_CANCELLED 4

int pawan_server_create(pawan_ctx *ctx, const pawan_serve_config *cfg, pawan_server **out);
/* Stops the worker (in-flight iteration finishes) and frees everything. */
void pawan_server_destroy(pawan_server *srv);
/* Copies the request's particles; returns its id.  nsteps RK4 steps of dt. */
int pawan_server_submit(pawan_server *srv, size_t n_wakes, const size_t *num_particles,
                        const double *position, const double *vorticity, const double *radius,
                        const double *volume, double nu, double dt, size_t nsteps,
                        long long *id);
int pawan_server_poll(pawan_server *srv, long long id, int *state);
/* Blocks until the request is done, rejected or cancelled, or timeout_s passes. */
int pawan_server_wait(pawan_server *srv, long long id, double timeout_s);
/* Final state (reference layout, 6N) and timing of a finished request; the
 * request is forgotten afterwards.  Times are seconds since the server was
 * created. */
int pawan_server_fetch(pawan_server *srv, long long id, double *state, size_t size,
                       double *t_submit, double *t_admit, double *t_done);
int pawan_server_cancel(pawan_server *srv, long long id);
int pawan_server_stats(pawan_server *srv, pawan_serve_stats *out);
/* The tiling the engine's pair launches use (FP32: 128 threads, packed far
 * path mode 1, the packed near pass; sources in fixed 8,192-source chunks, so
 * items_per_slot is not used), for running a request alone with the same
 * arithmetic. */
int pawan_server_get_tiling(pawan_server *srv, pawan_tiling *out);
/* Host-side fault injection, for testing how callers and the engine recover
 * (no GPU fault is made).  PAWAN_FAULT_ALLOC: the next `count` admissions
 * fail as an out-of-memory from the device allocator would (the request is
 * rejected, the others go on).  PAWAN_FAULT_ITERATION: the next `count`
 * iterations fail as a failed launch would (every request active in it is
 * rejected; the engine carries on with the next).  PAWAN_FAULT_SLOW: the next
 * `count` iterations first sleep `seconds` on the host (at most 60). */
#define PAWAN_FAULT_ALLOC 1
#define PAWAN_FAULT_ITERATION 2
#define PAWAN_FAULT_SLOW 3
int pawan_server_inject(pawan_server *srv, int fault, int count, double seconds);

/* ------------------------------------------------- allocation-free solve */
/* No counterpart in the reference.  For callers that must not allocate device
 * memory -- inside a host callback, under an allocator that owns the whole
 * device, or in a latency-critical loop where cudaMalloc's implicit
 * synchronisation is not acceptable.  One FP32 solve (all pairs over the n
 * particles with the high-order smoothing kernel, whatever
 * pawan_system_set_kernel chose elsewhere) from caller-owned DEVICE arrays:
 * position and vorticity n x 3, radius and volume n; writes velocity and
 * vorticity rate (n x 3, device).  The pair kernel is pawan_system_solve's
 * with PAWAN_PREC_F32, but the FP32 positions are relative to particle 0
 * rather than the centroid, so results agree with pawan_system_solve within
 * the FP32 tolerance, not bit for bit.  All working memory is one static
 * device array reserved by every GPU that loads the library (about 4.2 MB),
 * so n <= PAWAN_NOALLOC_MAX_PARTICLES; larger n, n < 2 or a negative or
 * non-finite nu returns PAWAN_ERR_INVALID.  The first call on a device
 * resolves that array's address (make it before any stream capture).  Calls
 * share the array: calls that may overlap on the GPU race and must be
 * serialised by the caller.  `stream` is a cudaStream_t (NULL: the default
 * stream); the call is asynchronous on it and allocates nothing. */
#define PAWAN_NOALLOC_MAX_PARTICLES 16384
int pawan_interact_noalloc(const double *position, const double *vorticity, const double *radius,
                           const double *volume, size_t n, double nu, double *velocity,
                           double *retvorcity, void *stream);

/* ----------------------------------------------------- throughput probes */
/* Measured FP32 / FP64 FMA throughput of the device, GFLOP/s (FMA = 2
 * flops), over `seconds` of back-to-back probe launches.  The FP32 figure is
 * the larger of scalar FFMA and packed FP32x2 FFMA2 chains. */
int pawan_peak_fp32(pawan_ctx *ctx, double seconds, double *gflops);
int pawan_peak_fp64(pawan_ctx *ctx, double seconds, double *gflops);

#ifdef __cplusplus
}
#endif

#endif /* PAWAN_B200_H */

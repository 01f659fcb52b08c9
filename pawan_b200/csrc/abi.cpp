// C ABI of the pawan B200 library (include/pawan_b200.h): contexts, systems,
// batches, sharding, diagnostics, the vorticity field, profiling and
// throughput probes, over the engine in runtime.cpp.
#include "runtime.h"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <numeric>

using namespace pawan;

size_t pawan_system::device_bytes() const {
  return X.bytes() + Xs.bytes() + K1.bytes() + K2.bytes() + R.bytes() + rad.bytes() +
         vol.bytes() + wake_id.bytes() + pos32.bytes() + vor32.bytes() + poslo.bytes() +
         vorlo.bytes() + pos64.bytes() +
         vor64.bytes() + diag_scratch.bytes() + diag_out.bytes() + Xc.bytes() + field.bytes() +
         (plan ? plan->partial.bytes() + plan->rates.bytes() + plan->tile_count.bytes() : 0);
}

// =================================================================== C ABI

#define CHECK_CTX(ctx) \
  if (!(ctx)) return PAWAN_ERR_INVALID
#define CHECK_SYS(sys) \
  if (!(sys) || !(sys)->ctx) return PAWAN_ERR_INVALID

static int pack_after_state(pawan_system *sys) {
  PAWAN_TRY(system_ensure_plan(sys));
  return launch_stage_mode(sys->ctx, *sys->plan, STAGE_PACK);
}

// Origin of the FP32 positions (centroid) and the near-tile radius: tile pairs
// closer than max(4 s_max, 0.03 * extent) use the hi/lo pair formulation.
static void set_geometry(pawan_system *sys, const double *pos, const double *rad) {
  const size_t N = sys->n;
  double c[3] = {0, 0, 0};
  for (size_t i = 0; i < N; ++i)
    for (int k = 0; k < 3; ++k) c[k] += pos[3 * i + k];
  for (int k = 0; k < 3; ++k) c[k] /= (double)N;
  double ext2 = 0, smax = 0;
  for (size_t i = 0; i < N; ++i) {
    double r2 = 0;
    for (int k = 0; k < 3; ++k) r2 += (pos[3 * i + k] - c[k]) * (pos[3 * i + k] - c[k]);
    ext2 = std::max(ext2, r2);
    smax = std::max(smax, rad[i]);
  }
  sys->ox = c[0];
  sys->oy = c[1];
  sys->oz = c[2];
  sys->r_near = std::max(4.0 * smax, 0.03 * std::sqrt(ext2));
  sys->geometry_version++;
}

static int create_system(pawan_ctx *ctx, size_t n_wakes, const size_t *num_particles, double nu,
                         int precision, bool ordered, pawan_system **out) {
  CHECK_CTX(ctx);
  if (!out || n_wakes == 0 || !num_particles)
    return fail(ctx, PAWAN_ERR_INVALID, "system needs at least one wake");
  if (precision < PAWAN_PREC_F32 || precision > PAWAN_PREC_F64_PLAIN)
    return fail(ctx, PAWAN_ERR_INVALID, "unknown precision");
  if (!std::isfinite(nu) || nu < 0.0) return fail(ctx, PAWAN_ERR_INVALID, "nu must be >= 0");
  *out = nullptr;
  std::unique_ptr<pawan_system> sys(new pawan_system());
  sys->ctx = ctx;
  sys->ordered_alloc = ordered;
  size_t off = 0;
  for (size_t w = 0; w < n_wakes; ++w) {
    if (num_particles[w] == 0) return fail(ctx, PAWAN_ERR_INVALID, "empty wake");
    sys->counts.push_back(num_particles[w]);
    sys->offsets.push_back(off);
    off += num_particles[w];
  }
  if (off < 2) return fail(ctx, PAWAN_ERR_INVALID, "a system needs at least two particles");
  if (off > (size_t)(1 << 28)) return fail(ctx, PAWAN_ERR_INVALID, "too many particles");
  sys->n = off;
  sys->nu = nu;
  sys->precision = precision;
  sys->tile = default_tile(precision);
  PAWAN_CUDA(ctx, cudaSetDevice(ctx->device));
  PAWAN_TRY(system_alloc(sys.get()));
  *out = sys.release();
  return PAWAN_OK;
}

int pawan::system_create_ordered(pawan_ctx *ctx, size_t n_wakes, const size_t *num_particles,
                                 double nu, int precision, pawan_system **out) {
  return create_system(ctx, n_wakes, num_particles, nu, precision, true, out);
}

int pawan::system_upload(pawan_system *sys, const double *position, const double *vorticity,
                         const double *radius, const double *volume) {
  CHECK_SYS(sys);
  pawan_ctx *ctx = sys->ctx;
  if (!position || !vorticity || !radius || !volume)
    return fail(ctx, PAWAN_ERR_INVALID, "null particle array");
  const size_t N = sys->n;
  for (size_t i = 0; i < N; ++i)
    if (!(radius[i] > 0.0) || !std::isfinite(radius[i]))
      return fail(ctx, PAWAN_ERR_INVALID, "smoothing radii must be positive");
  for (size_t i = 0; i < 3 * N; ++i)
    if (!std::isfinite(position[i]) || !std::isfinite(vorticity[i]))
      return fail(ctx, PAWAN_ERR_INVALID, "non-finite position or vorticity");
  set_geometry(sys, position, radius);
  PAWAN_CUDA(ctx, cudaMemcpyAsync(sys->X.p, position, 3 * N * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
  PAWAN_CUDA(ctx, cudaMemcpyAsync(sys->X.p + 3 * N, vorticity, 3 * N * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
  PAWAN_CUDA(ctx, cudaMemcpyAsync(sys->rad.p, radius, N * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
  PAWAN_CUDA(ctx, cudaMemcpyAsync(sys->vol.p, volume, N * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
  sys->has_particles = true;
  return PAWAN_OK;
}

extern "C" {

const char *pawan_status_name(int status) {
  switch (status) {
    case PAWAN_OK: return "ok";
    case PAWAN_ERR_INVALID: return "invalid argument";
    case PAWAN_ERR_CUDA: return "cuda error";
    case PAWAN_ERR_NOMEM: return "out of memory";
    case PAWAN_ERR_STATE: return "invalid state";
    case PAWAN_ERR_BUDGET: return "exceeds budget";
    case PAWAN_ERR_TIMEOUT: return "timeout";
    case PAWAN_ERR_NOTFOUND: return "not found";
    case PAWAN_ERR_REJECTED: return "rejected";
    default: return "unknown status";
  }
}

int pawan_ctx_create(int device, pawan_ctx **out) {
  if (!out) return PAWAN_ERR_INVALID;
  *out = nullptr;
  std::unique_ptr<pawan_ctx> ctx(new pawan_ctx());
  ctx->device = device;
  int count = 0;
  cudaError_t e = cudaGetDeviceCount(&count);
  if (e != cudaSuccess || device < 0 || device >= count) return PAWAN_ERR_CUDA;
  if (cudaSetDevice(device) != cudaSuccess) return PAWAN_ERR_CUDA;
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return PAWAN_ERR_CUDA;
  ctx->sm_count = prop.multiProcessorCount;
  ctx->cc_major = prop.major;
  ctx->cc_minor = prop.minor;
  ctx->total_mem = prop.totalGlobalMem;
  if (prop.major != 10) return PAWAN_ERR_CUDA;  // built for sm_100a only
  if (cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess)
    return PAWAN_ERR_CUDA;
  if (cudaMalloc(&ctx->d_counter, 2 * sizeof(int)) != cudaSuccess) {
    cudaStreamDestroy(ctx->stream);
    return PAWAN_ERR_NOMEM;
  }
  *out = ctx.release();
  return PAWAN_OK;
}

void pawan_ctx_destroy(pawan_ctx *ctx) {
  if (!ctx) return;
  cudaSetDevice(ctx->device);
  cudaStreamSynchronize(ctx->stream);
  for (auto *pend : {&ctx->pending, &ctx->stage_pending})
    for (auto &pr : *pend) {
      cudaEventDestroy(pr.first);
      cudaEventDestroy(pr.second);
    }
  for (auto e : ctx->event_pool) cudaEventDestroy(e);
  for (auto e : ctx->marks)
    if (e) cudaEventDestroy(e);
  if (ctx->flush_buf) cudaFree(ctx->flush_buf);
  if (ctx->d_counter) cudaFree(ctx->d_counter);
  if (ctx->stream) cudaStreamDestroy(ctx->stream);
  delete ctx;
}

const char *pawan_ctx_last_error(const pawan_ctx *ctx) { return ctx ? ctx->err.c_str() : ""; }

int pawan_ctx_info(pawan_ctx *ctx, int *sm_count, int *cc_major, int *cc_minor, size_t *total_mem) {
  CHECK_CTX(ctx);
  if (sm_count) *sm_count = ctx->sm_count;
  if (cc_major) *cc_major = ctx->cc_major;
  if (cc_minor) *cc_minor = ctx->cc_minor;
  if (total_mem) *total_mem = ctx->total_mem;
  return PAWAN_OK;
}

int pawan_ctx_synchronize(pawan_ctx *ctx) {
  CHECK_CTX(ctx);
  PAWAN_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return PAWAN_OK;
}

unsigned long long pawan_ctx_launch_count(const pawan_ctx *ctx) {
  return ctx ? ctx->launches.load() : 0ull;
}

int pawan_ctx_profile(pawan_ctx *ctx, int enable) {
  CHECK_CTX(ctx);
  PAWAN_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  for (auto *pend : {&ctx->pending, &ctx->stage_pending}) {
    for (auto &pr : *pend) {
      ctx->event_pool.push_back(pr.first);
      ctx->event_pool.push_back(pr.second);
    }
    pend->clear();
  }
  ctx->pair_ms = 0.0;
  ctx->pair_launches = 0;
  ctx->pair_interactions = 0.0;
  ctx->stage_ms = 0.0;
  ctx->stage_launches = 0;
  ctx->stage_bytes = 0.0;
  ctx->profile = enable != 0;
  return PAWAN_OK;
}

int pawan_ctx_profile_read(pawan_ctx *ctx, double *pair_ms, unsigned long long *pair_launches,
                           double *pair_interactions) {
  CHECK_CTX(ctx);
  PAWAN_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  for (auto &pr : ctx->pending) {
    float ms = 0.f;
    PAWAN_CUDA(ctx, cudaEventElapsedTime(&ms, pr.first, pr.second));
    ctx->pair_ms += ms;
    ctx->event_pool.push_back(pr.first);
    ctx->event_pool.push_back(pr.second);
  }
  ctx->pending.clear();
  if (pair_ms) *pair_ms = ctx->pair_ms;
  if (pair_launches) *pair_launches = ctx->pair_launches;
  if (pair_interactions) *pair_interactions = ctx->pair_interactions;
  return PAWAN_OK;
}

int pawan_ctx_profile_stage(pawan_ctx *ctx, double *stage_ms, unsigned long long *stage_launches,
                            double *stage_bytes) {
  CHECK_CTX(ctx);
  PAWAN_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  for (auto &pr : ctx->stage_pending) {
    float ms = 0.f;
    PAWAN_CUDA(ctx, cudaEventElapsedTime(&ms, pr.first, pr.second));
    ctx->stage_ms += ms;
    ctx->event_pool.push_back(pr.first);
    ctx->event_pool.push_back(pr.second);
  }
  ctx->stage_pending.clear();
  if (stage_ms) *stage_ms = ctx->stage_ms;
  if (stage_launches) *stage_launches = ctx->stage_launches;
  if (stage_bytes) *stage_bytes = ctx->stage_bytes;
  return PAWAN_OK;
}

int pawan_ctx_mark(pawan_ctx *ctx, int slot) {
  CHECK_CTX(ctx);
  if (slot < 0 || slot >= 16) return fail(ctx, PAWAN_ERR_INVALID, "mark slot must be 0..15");
  if (!ctx->marks[slot]) PAWAN_CUDA(ctx, cudaEventCreate(&ctx->marks[slot]));
  PAWAN_CUDA(ctx, cudaEventRecord(ctx->marks[slot], ctx->stream));
  return PAWAN_OK;
}

int pawan_ctx_elapsed(pawan_ctx *ctx, int slot0, int slot1, double *ms) {
  CHECK_CTX(ctx);
  if (!ms || slot0 < 0 || slot0 >= 16 || slot1 < 0 || slot1 >= 16 || !ctx->marks[slot0] ||
      !ctx->marks[slot1])
    return fail(ctx, PAWAN_ERR_INVALID, "unrecorded mark");
  PAWAN_CUDA(ctx, cudaEventSynchronize(ctx->marks[slot1]));
  float f = 0.f;
  PAWAN_CUDA(ctx, cudaEventElapsedTime(&f, ctx->marks[slot0], ctx->marks[slot1]));
  *ms = f;
  return PAWAN_OK;
}

int pawan_ctx_flush_l2(pawan_ctx *ctx, size_t bytes) {
  CHECK_CTX(ctx);
  if (bytes > ctx->flush_bytes) {
    if (ctx->flush_buf) cudaFree(ctx->flush_buf);
    ctx->flush_buf = nullptr;
    ctx->flush_bytes = 0;
    PAWAN_CUDA(ctx, cudaMalloc(&ctx->flush_buf, bytes));
    ctx->flush_bytes = bytes;
  }
  PAWAN_CUDA(ctx, cudaMemsetAsync(ctx->flush_buf, (int)(ctx->launches.load() & 0xff), bytes, ctx->stream));
  return PAWAN_OK;
}

int pawan_host_alloc(pawan_ctx *ctx, size_t bytes, void **out) {
  CHECK_CTX(ctx);
  if (!out) return PAWAN_ERR_INVALID;
  PAWAN_CUDA(ctx, cudaHostAlloc(out, bytes ? bytes : 1, cudaHostAllocDefault));
  return PAWAN_OK;
}

int pawan_host_free(pawan_ctx *ctx, void *ptr) {
  CHECK_CTX(ctx);
  PAWAN_CUDA(ctx, cudaFreeHost(ptr));
  return PAWAN_OK;
}

int pawan_system_create(pawan_ctx *ctx, size_t n_wakes, const size_t *num_particles, double nu,
                        int precision, pawan_system **out) {
  return create_system(ctx, n_wakes, num_particles, nu, precision, false, out);
}

// Device buffers are released with cudaFree, which waits for outstanding
// work on them; the context is not touched, so a system may outlive it
// (except one created by the serving engine, whose buffers go back to the
// memory pool on the context's stream).
void pawan_system_destroy(pawan_system *sys) {
  if (!sys) return;
  delete sys;
}

size_t pawan_system_size(const pawan_system *sys) { return sys ? 6 * sys->n : 0; }
size_t pawan_system_num_particles(const pawan_system *sys) { return sys ? sys->n : 0; }

int pawan_system_set_particles(pawan_system *sys, const double *position, const double *vorticity,
                               const double *radius, const double *volume) {
  PAWAN_TRY(system_upload(sys, position, vorticity, radius, volume));
  PAWAN_TRY(pack_after_state(sys));
  PAWAN_CUDA(sys->ctx, cudaStreamSynchronize(sys->ctx->stream));
  return PAWAN_OK;
}

int pawan_system_set_states(pawan_system *sys, const double *state, size_t size) {
  CHECK_SYS(sys);
  if (!state || size != 6 * sys->n)
    return fail(sys->ctx, PAWAN_ERR_INVALID, "state size must be 6*N");
  PAWAN_TRY(state_to_device(sys, state));
  PAWAN_TRY(pack_after_state(sys));
  PAWAN_CUDA(sys->ctx, cudaStreamSynchronize(sys->ctx->stream));
  return PAWAN_OK;
}

int pawan_system_get_states(pawan_system *sys, double *state, size_t size) {
  CHECK_SYS(sys);
  if (!state || size != 6 * sys->n)
    return fail(sys->ctx, PAWAN_ERR_INVALID, "state size must be 6*N");
  return state_from_device(sys, sys->X.p, state);
}

#define CHECK_UNSHARDED(sys)                                                        \
  if ((sys)->shard.active)                                                          \
  return fail((sys)->ctx, PAWAN_ERR_STATE,                                          \
              "system is sharded over processes: use pawan_system_shard_rates / shard_stage")

int pawan_system_solve(pawan_system *sys) {
  CHECK_SYS(sys);
  CHECK_UNSHARDED(sys);
  PAWAN_TRY(system_ensure_plan(sys));
  PAWAN_TRY(launch_pairs(sys->ctx, *sys->plan));
  return launch_stage_mode(sys->ctx, *sys->plan, STAGE_RATES);
}

int pawan_system_get_rates(pawan_system *sys, double *rate, size_t size) {
  CHECK_SYS(sys);
  if (!rate || size != 6 * sys->n)
    return fail(sys->ctx, PAWAN_ERR_INVALID, "rate size must be 6*N");
  return state_from_device(sys, sys->R.p, rate);
}

int pawan_system_get_wake_rates(pawan_system *sys, size_t wake, double *velocity,
                                double *retvorcity) {
  CHECK_SYS(sys);
  pawan_ctx *ctx = sys->ctx;
  if (wake >= sys->counts.size() || !velocity || !retvorcity)
    return fail(ctx, PAWAN_ERR_INVALID, "bad wake index or null output");
  const size_t o = sys->offsets[wake], c = sys->counts[wake], N = sys->n;
  PAWAN_CUDA(ctx, cudaMemcpyAsync(velocity, sys->R.p + 3 * o, 3 * c * sizeof(double),
                                  cudaMemcpyDeviceToHost, ctx->stream));
  PAWAN_CUDA(ctx, cudaMemcpyAsync(retvorcity, sys->R.p + 3 * N + 3 * o, 3 * c * sizeof(double),
                                  cudaMemcpyDeviceToHost, ctx->stream));
  PAWAN_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return PAWAN_OK;
}

int pawan_system_rk4(pawan_system *sys, double dt, size_t nsteps) {
  CHECK_SYS(sys);
  CHECK_UNSHARDED(sys);
  PAWAN_TRY(system_ensure_plan(sys));
  PAWAN_TRY(set_plan_dt(sys->ctx, *sys->plan, nullptr, dt));
  return rk4_steps(sys->ctx, *sys->plan, nsteps, false);
}

int pawan_system_rk4_graph(pawan_system *sys, double dt, size_t nsteps) {
  CHECK_SYS(sys);
  CHECK_UNSHARDED(sys);
  PAWAN_TRY(system_ensure_plan(sys));
  PAWAN_TRY(set_plan_dt(sys->ctx, *sys->plan, nullptr, dt));
  return rk4_steps(sys->ctx, *sys->plan, nsteps, true);
}

int pawan_system_euler(pawan_system *sys, double dt, size_t nsteps) {
  CHECK_SYS(sys);
  CHECK_UNSHARDED(sys);
  PAWAN_TRY(system_ensure_plan(sys));
  PAWAN_TRY(set_plan_dt(sys->ctx, *sys->plan, nullptr, dt));
  for (size_t k = 0; k < nsteps; ++k) {
    PAWAN_TRY(launch_pairs(sys->ctx, *sys->plan));
    PAWAN_TRY(launch_stage_mode(sys->ctx, *sys->plan, STAGE_EULER));
  }
  return PAWAN_OK;
}

static int run_diagnostics(pawan_system *sys, bool quadratic, double *out12) {
  pawan_ctx *ctx = sys->ctx;
  if (!sys->has_particles) return fail(ctx, PAWAN_ERR_STATE, "particles not set");
  cudaError_t e = launch_diagnostics((int)sys->n, sys->kernel, sys->pos64.p, sys->vor64.p, sys->wake_id.p,
                                     sys->diag_scratch.p, sys->diag_out.p, quadratic, ctx->stream);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "diagnostics launch");
  ctx->launches += quadratic ? 4 : 2;
  double h[12] = {0};
  PAWAN_CUDA(ctx, cudaMemcpyAsync(h, sys->diag_out.p, 12 * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  PAWAN_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  if (!quadratic) h[9] = h[10] = h[11] = 0.0;
  std::memcpy(out12, h, sizeof(h));
  return PAWAN_OK;
}

int pawan_system_diagnose(pawan_system *sys, double *out, int quadratic) {
  CHECK_SYS(sys);
  if (!out) return fail(sys->ctx, PAWAN_ERR_INVALID, "null output");
  double h[12];
  PAWAN_TRY(run_diagnostics(sys, quadratic != 0, h));
  std::memcpy(out, h, 11 * sizeof(double));
  return PAWAN_OK;
}

int pawan_system_kinetic_energy(pawan_system *sys, double *ke) {
  CHECK_SYS(sys);
  if (!ke) return fail(sys->ctx, PAWAN_ERR_INVALID, "null output");
  double h[12];
  PAWAN_TRY(run_diagnostics(sys, true, h));
  *ke = h[11];
  return PAWAN_OK;
}

int pawan_system_influence(pawan_system *sys, double *field, size_t size) {
  CHECK_SYS(sys);
  pawan_ctx *ctx = sys->ctx;
  if (!field || size != 3 * sys->n) return fail(ctx, PAWAN_ERR_INVALID, "field size must be 3*N");
  if (!sys->has_particles) return fail(ctx, PAWAN_ERR_STATE, "particles not set");
  if (!sys->field.p) PAWAN_CUDA(ctx, sys->field.alloc(3 * sys->n));
  // pos64 / vor64 hold pack(X) between API calls
  PAWAN_CUDA(ctx, launch_influence((int)sys->n, sys->kernel, sys->pos64.p, sys->vor64.p, sys->field.p,
                                   ctx->stream));
  ctx->launches++;
  PAWAN_CUDA(ctx, cudaMemcpyAsync(field, sys->field.p, 3 * sys->n * sizeof(double),
                                  cudaMemcpyDeviceToHost, ctx->stream));
  PAWAN_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return PAWAN_OK;
}

// Device scratch bound of pawan_system_influence_columns (strength columns
// plus their fields): larger requests run in several launches.
constexpr size_t kInfluenceColumnBytes = size_t(256) << 20;
constexpr size_t kMaxInfluenceColumnsPerLaunch = size_t(65535) * kInfluenceColumnGroup;

static int influence_columns(pawan_system *sys, size_t ncols, const double *alpha, double *field,
                             DBuf<double> &cols, DBuf<double> &out) {
  pawan_ctx *ctx = sys->ctx;
  const size_t per = 3 * sys->n;
  const size_t fit = std::max<size_t>(1, kInfluenceColumnBytes / (2 * per * sizeof(double)));
  const size_t chunk = std::min(ncols, std::min(fit, kMaxInfluenceColumnsPerLaunch));
  PAWAN_CUDA(ctx, cols.alloc(chunk * per));
  PAWAN_CUDA(ctx, out.alloc(chunk * per));
  for (size_t c0 = 0; c0 < ncols; c0 += chunk) {
    const size_t nc = std::min(chunk, ncols - c0);
    PAWAN_CUDA(ctx, cudaMemcpyAsync(cols.p, alpha + c0 * per, nc * per * sizeof(double),
                                    cudaMemcpyHostToDevice, ctx->stream));
    PAWAN_CUDA(ctx, launch_influence_columns((int)sys->n, (int)nc, sys->kernel, sys->pos64.p, cols.p,
                                             out.p, ctx->stream));
    ctx->launches++;
    PAWAN_CUDA(ctx, cudaMemcpyAsync(field + c0 * per, out.p, nc * per * sizeof(double),
                                    cudaMemcpyDeviceToHost, ctx->stream));
  }
  return PAWAN_OK;
}

int pawan_system_influence_columns(pawan_system *sys, size_t ncols, const double *alpha,
                                   double *field, size_t size) {
  CHECK_SYS(sys);
  pawan_ctx *ctx = sys->ctx;
  if (ncols == 0) return fail(ctx, PAWAN_ERR_INVALID, "ncols must be positive");
  if (!alpha || !field || size / ncols != 3 * sys->n || size % ncols != 0)
    return fail(ctx, PAWAN_ERR_INVALID, "alpha and field must hold ncols * 3N doubles");
  if (!sys->has_particles) return fail(ctx, PAWAN_ERR_STATE, "particles not set");
  DBuf<double> cols, out;
  const int st = influence_columns(sys, ncols, alpha, field, cols, out);
  // the scratch is freed on return: wait for the copies and launches first
  const cudaError_t e = cudaStreamSynchronize(ctx->stream);
  if (st != PAWAN_OK) return st;
  if (e != cudaSuccess) return cuda_fail(ctx, e, "influence columns");
  return PAWAN_OK;
}

size_t pawan_shard_size(size_t n, int world) {
  if (world < 1 || n == 0) return 0;
  const size_t per = (n + (size_t)world - 1) / (size_t)world;
  return (per + kShardAlign - 1) / kShardAlign * kShardAlign;
}

static bool device_pointer(const void *p) {
  cudaPointerAttributes a{};
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

int pawan_system_set_shard(pawan_system *sys, int rank, int world, double *send, double *recv) {
  CHECK_SYS(sys);
  pawan_ctx *ctx = sys->ctx;
  if (world == 0) {
    sys->shard = pawan_system::Shard{};
    sys->plan.reset();
    return PAWAN_OK;
  }
  if (world < 1 || rank < 0 || rank >= world)
    return fail(ctx, PAWAN_ERR_INVALID, "shard rank must be in [0, world)");
  if (!send || !recv || !device_pointer(send) || !device_pointer(recv))
    return fail(ctx, PAWAN_ERR_INVALID, "shard exchange buffers must be device memory");
  pawan_system::Shard sh;
  sh.active = true;
  sh.rank = rank;
  sh.world = world;
  sh.size = pawan_shard_size(sys->n, world);
  sh.send = send;
  sh.recv = recv;
  sys->shard = sh;
  sys->plan.reset();  // the next plan covers this process's targets
  return PAWAN_OK;
}

int pawan_system_shard_rates(pawan_system *sys) {
  CHECK_SYS(sys);
  if (!sys->shard.active) return fail(sys->ctx, PAWAN_ERR_STATE, "system is not sharded");
  PAWAN_TRY(system_ensure_plan(sys));
  Plan &p = *sys->plan;
  PAWAN_TRY(launch_pairs(sys->ctx, p));
  cudaError_t e = launch_stage(STAGE_SHARD, p.n_shard_blocks, p.shard_items.p, p.stage_descs.p,
                               sys->ctx->stream);
  if (e != cudaSuccess) return cuda_fail(sys->ctx, e, "shard reduce launch");
  if (p.n_shard_blocks > 0) sys->ctx->launches++;
  return PAWAN_OK;
}

int pawan_system_shard_stage(pawan_system *sys, int stage, double dt) {
  CHECK_SYS(sys);
  if (!sys->shard.active) return fail(sys->ctx, PAWAN_ERR_STATE, "system is not sharded");
  static const int modes[5] = {STAGE_RATES, STAGE_K1, STAGE_K2, STAGE_K3, STAGE_FINAL};
  if (stage < 0 || stage > 4) return fail(sys->ctx, PAWAN_ERR_INVALID, "stage must be 0..4");
  PAWAN_TRY(system_ensure_plan(sys));
  Plan &p = *sys->plan;
  if (stage > 0) PAWAN_TRY(set_plan_dt(sys->ctx, p, nullptr, dt));
  return launch_stage_mode(sys->ctx, p, modes[stage]);
}

int pawan_ctx_stream(pawan_ctx *ctx, void **stream) {
  CHECK_CTX(ctx);
  if (!stream) return PAWAN_ERR_INVALID;
  *stream = ctx->stream;
  return PAWAN_OK;
}

int pawan_system_set_kernel(pawan_system *sys, int kernel) {
  CHECK_SYS(sys);
  if (kernel != PAWAN_KERNEL_HIGHORDER && kernel != PAWAN_KERNEL_GAUSSIAN)
    return fail(sys->ctx, PAWAN_ERR_INVALID, "unknown smoothing kernel");
  if (kernel != sys->kernel) {
    sys->kernel = kernel;
    if (!tile_supported(sys->precision, sys->tile.pc, kernel)) {
      sys->tile = default_tile(sys->precision);
      sys->fixed_tile = false;
    }
    sys->plan.reset();
  }
  return PAWAN_OK;
}

int pawan_system_get_kernel(pawan_system *sys, int *kernel) {
  CHECK_SYS(sys);
  if (!kernel) return PAWAN_ERR_INVALID;
  *kernel = sys->kernel;
  return PAWAN_OK;
}

int pawan_system_set_nu(pawan_system *sys, double nu) {
  CHECK_SYS(sys);
  if (!std::isfinite(nu) || nu < 0.0) return fail(sys->ctx, PAWAN_ERR_INVALID, "nu must be >= 0");
  sys->nu = nu;
  return PAWAN_OK;
}

int pawan_system_set_precision(pawan_system *sys, int precision) {
  CHECK_SYS(sys);
  if (precision < PAWAN_PREC_F32 || precision > PAWAN_PREC_F64_PLAIN)
    return fail(sys->ctx, PAWAN_ERR_INVALID, "unknown precision");
  if (precision != sys->precision) {
    sys->precision = precision;
    if (!sys->fixed_tile || !tile_supported(precision, sys->tile.pc, sys->kernel))
      sys->tile = default_tile(precision);
  }
  return PAWAN_OK;
}

int pawan_system_write_frame(pawan_system *sys, const char *path, double t, int append) {
  CHECK_SYS(sys);
  pawan_ctx *ctx = sys->ctx;
  if (!path) return fail(ctx, PAWAN_ERR_INVALID, "null path");
  const size_t N = sys->n;
  std::vector<double> x(6 * N), s(N);
  PAWAN_CUDA(ctx, cudaMemcpyAsync(x.data(), sys->X.p, 6 * N * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  PAWAN_CUDA(ctx, cudaMemcpyAsync(s.data(), sys->rad.p, N * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  PAWAN_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  FILE *f = std::fopen(path, append ? "ab" : "wb");
  if (!f) return fail(ctx, PAWAN_ERR_INVALID, std::string("cannot open ") + path);
  bool ok = std::fwrite(&t, sizeof(double), 1, f) == 1;
  const size_t nw = sys->counts.size();
  ok = ok && std::fwrite(&nw, sizeof(size_t), 1, f) == 1;
  for (size_t w = 0; w < nw && ok; ++w) {
    const size_t o = sys->offsets[w], c = sys->counts[w];
    ok = ok && std::fwrite(&c, sizeof(size_t), 1, f) == 1;
    ok = ok && std::fwrite(x.data() + 3 * o, sizeof(double), 3 * c, f) == 3 * c;
    ok = ok && std::fwrite(x.data() + 3 * N + 3 * o, sizeof(double), 3 * c, f) == 3 * c;
    ok = ok && std::fwrite(s.data() + o, sizeof(double), c, f) == c;
  }
  std::fclose(f);
  if (!ok) return fail(ctx, PAWAN_ERR_INVALID, std::string("short write to ") + path);
  return PAWAN_OK;
}

static int tile_from_abi(pawan_ctx *ctx, int precision, int kernel, const pawan_tiling *t,
                         TileChoice *out) {
  if (!t) return fail(ctx, PAWAN_ERR_INVALID, "null tiling");
  TileChoice c;
  c.pc = PairConfig{t->threads, t->threads_per_target, t->unroll, t->targets_per_thread,
                    t->blocks_per_sm, t->packed, t->split_near};
  c.items_per_slot = t->items_per_slot;
  if (t->items_per_slot < 1 || t->targets_per_thread < 1 || t->blocks_per_sm < 0 || t->packed < 0 ||
      t->split_near < 0 || (t->split_near > 0 && precision != PAWAN_PREC_F32) ||
      !tile_supported(precision, c.pc, kernel))
    return fail(ctx, PAWAN_ERR_INVALID, "tiling not compiled for this precision and kernel");
  *out = c;
  return PAWAN_OK;
}

int pawan_system_set_tiling(pawan_system *sys, const pawan_tiling *tiling) {
  CHECK_SYS(sys);
  TileChoice t;
  PAWAN_TRY(tile_from_abi(sys->ctx, sys->precision, sys->kernel, tiling, &t));
  sys->tile = t;
  sys->fixed_tile = true;
  return PAWAN_OK;
}

int pawan_system_get_tiling(pawan_system *sys, pawan_tiling *tiling) {
  CHECK_SYS(sys);
  if (!tiling) return PAWAN_ERR_INVALID;
  tiling->threads = sys->tile.pc.tb;
  tiling->threads_per_target = sys->tile.pc.p;
  tiling->targets_per_thread = sys->tile.pc.r;
  tiling->unroll = sys->tile.pc.unroll;
  tiling->blocks_per_sm = sys->tile.pc.minb;
  tiling->packed = sys->tile.pc.packed;
  tiling->split_near = sys->tile.pc.split;
  tiling->items_per_slot = sys->tile.items_per_slot;
  return PAWAN_OK;
}

int pawan_tile_candidates(int precision, int kernel, pawan_tiling *out, size_t cap, size_t *count) {
  if (!count || (cap > 0 && !out)) return PAWAN_ERR_INVALID;
  if (precision < PAWAN_PREC_F32 || precision > PAWAN_PREC_F64_PLAIN) return PAWAN_ERR_INVALID;
  if (kernel != PAWAN_KERNEL_HIGHORDER && kernel != PAWAN_KERNEL_GAUSSIAN) return PAWAN_ERR_INVALID;
  const std::vector<TileChoice> v = tile_candidates(precision, kernel);
  *count = v.size();
  for (size_t i = 0; i < v.size() && i < cap; ++i) {
    out[i].threads = v[i].pc.tb;
    out[i].threads_per_target = v[i].pc.p;
    out[i].targets_per_thread = v[i].pc.r;
    out[i].unroll = v[i].pc.unroll;
    out[i].blocks_per_sm = v[i].pc.minb;
    out[i].packed = v[i].pc.packed;
    out[i].split_near = v[i].pc.split;
    out[i].items_per_slot = v[i].items_per_slot;
  }
  return PAWAN_OK;
}

int pawan_tile_chunkings(int *out, size_t cap, size_t *count) {
  if (!count || (cap > 0 && !out)) return PAWAN_ERR_INVALID;
  *count = kTuneItemsPerSlot.size();
  for (size_t i = 0; i < kTuneItemsPerSlot.size() && i < cap; ++i) out[i] = kTuneItemsPerSlot[i];
  return PAWAN_OK;
}

int pawan_system_autotune(pawan_system *sys) {
  CHECK_SYS(sys);
  if (!sys->has_particles) return fail(sys->ctx, PAWAN_ERR_STATE, "particles not set");
  TileChoice best;
  PAWAN_TRY(autotune_plan(sys->ctx, {sys}, sys->precision, &best));
  sys->tile = best;
  sys->fixed_tile = true;
  sys->plan.reset();
  const double n2 = (double)sys->n * (double)sys->n;
  sys->ctx->tune_cache[std::make_tuple(sys->precision, sys->nu != 0.0 ? 1 : 0,
                                       (int)std::log2(std::max(1.0, n2)), 0)] = best;
  return system_ensure_plan(sys);
}

int pawan_system_checkpoint(pawan_system *sys) {
  CHECK_SYS(sys);
  pawan_ctx *ctx = sys->ctx;
  if (!sys->has_particles) return fail(ctx, PAWAN_ERR_STATE, "particles not set");
  if (!sys->Xc.p) PAWAN_CUDA(ctx, sys->Xc.alloc(6 * sys->n));
  PAWAN_CUDA(ctx, cudaMemcpyAsync(sys->Xc.p, sys->X.p, 6 * sys->n * sizeof(double),
                                  cudaMemcpyDeviceToDevice, ctx->stream));
  return PAWAN_OK;
}

int pawan_system_restore(pawan_system *sys) {
  CHECK_SYS(sys);
  pawan_ctx *ctx = sys->ctx;
  if (!sys->Xc.p) return fail(ctx, PAWAN_ERR_STATE, "no checkpoint taken");
  PAWAN_CUDA(ctx, cudaMemcpyAsync(sys->X.p, sys->Xc.p, 6 * sys->n * sizeof(double),
                                  cudaMemcpyDeviceToDevice, ctx->stream));
  return pack_after_state(sys);
}

int pawan_system_device_state(pawan_system *sys, double **state) {
  CHECK_SYS(sys);
  if (!state) return PAWAN_ERR_INVALID;
  *state = sys->X.p;
  return PAWAN_OK;
}

// ------------------------------------------------------------------ batch

struct pawan_batch {
  pawan_ctx *ctx = nullptr;
  std::vector<pawan_system *> systems;
  int precision = PAWAN_PREC_F32;
  TileChoice tile;
  std::unique_ptr<Plan> plan;
};

static int batch_ensure_plan(pawan_batch *b) {
  for (auto *s : b->systems)
    if (!s->has_particles) return fail(b->ctx, PAWAN_ERR_STATE, "a batch system has no particles");
  if (b->plan && !b->plan->stale() && b->plan->tile == b->tile) return PAWAN_OK;
  b->plan.reset();
  return build_plan(b->ctx, b->systems, b->precision, b->tile, b->plan);
}

int pawan_batch_create(pawan_ctx *ctx, size_t n, pawan_system *const *systems, pawan_batch **out) {
  CHECK_CTX(ctx);
  if (!out || n == 0 || !systems) return fail(ctx, PAWAN_ERR_INVALID, "empty batch");
  std::unique_ptr<pawan_batch> b(new pawan_batch());
  b->ctx = ctx;
  b->precision = systems[0] ? systems[0]->precision : PAWAN_PREC_F32;
  for (size_t i = 0; i < n; ++i) {
    if (!systems[i] || systems[i]->ctx != ctx)
      return fail(ctx, PAWAN_ERR_INVALID, "batch systems must share the context");
    if (systems[i]->precision != b->precision)
      return fail(ctx, PAWAN_ERR_INVALID, "batch systems must share one precision");
    if (systems[i]->shard.active)
      return fail(ctx, PAWAN_ERR_INVALID, "a sharded system cannot join a batch");
    if (systems[i]->kernel != systems[0]->kernel)
      return fail(ctx, PAWAN_ERR_INVALID, "batch systems must share one smoothing kernel");
    b->systems.push_back(systems[i]);
  }
  b->tile = default_tile(b->precision);
  *out = b.release();
  return PAWAN_OK;
}

void pawan_batch_destroy(pawan_batch *b) {
  if (!b) return;
  delete b;
}

int pawan_batch_rk4(pawan_batch *b, const double *dt, double dt0, size_t nsteps, int use_graph) {
  if (!b) return PAWAN_ERR_INVALID;
  PAWAN_TRY(batch_ensure_plan(b));
  PAWAN_TRY(set_plan_dt(b->ctx, *b->plan, dt, dt0));
  return rk4_steps(b->ctx, *b->plan, nsteps, use_graph != 0);
}

int pawan_batch_solve(pawan_batch *b) {
  if (!b) return PAWAN_ERR_INVALID;
  PAWAN_TRY(batch_ensure_plan(b));
  PAWAN_TRY(launch_pairs(b->ctx, *b->plan));
  return launch_stage_mode(b->ctx, *b->plan, STAGE_RATES);
}

int pawan_batch_set_tiling(pawan_batch *b, const pawan_tiling *tiling) {
  if (!b) return PAWAN_ERR_INVALID;
  TileChoice t;
  PAWAN_TRY(tile_from_abi(b->ctx, b->precision, b->systems[0]->kernel, tiling, &t));
  b->tile = t;
  return PAWAN_OK;
}

int pawan_batch_autotune(pawan_batch *b) {
  if (!b) return PAWAN_ERR_INVALID;
  for (auto *s : b->systems)
    if (!s->has_particles) return fail(b->ctx, PAWAN_ERR_STATE, "a batch system has no particles");
  TileChoice best;
  PAWAN_TRY(autotune_plan(b->ctx, b->systems, b->precision, &best));
  b->tile = best;
  b->plan.reset();
  return batch_ensure_plan(b);
}

// ------------------------------------------------------------ throughput

// kind: 0 = FP32 FFMA, 1 = FP64 DFMA, 2 = packed FP32x2 FFMA2
static int run_peak(pawan_ctx *ctx, double seconds, double *gflops, int kind) {
  const bool fp64 = kind == 1;
  CHECK_CTX(ctx);
  if (!gflops) return PAWAN_ERR_INVALID;
  const int threads = 256;
  const int blocks = ctx->sm_count * 8;
  const int iters = fp64 ? 2048 : 4096;
  DBuf<double> sink;
  PAWAN_CUDA(ctx, sink.alloc((size_t)blocks));
  cudaEvent_t e0, e1;
  PAWAN_CUDA(ctx, cudaEventCreate(&e0));
  PAWAN_CUDA(ctx, cudaEventCreate(&e1));
  auto launch = [&]() -> cudaError_t {
    ctx->launches++;
    if (kind == 1) return launch_dfma_peak(blocks, threads, iters, sink.p, ctx->stream);
    if (kind == 2)
      return launch_ffma2_peak(blocks, threads, iters, reinterpret_cast<float *>(sink.p),
                               ctx->stream);
    return launch_ffma_peak(blocks, threads, iters, reinterpret_cast<float *>(sink.p), ctx->stream);
  };
  cudaError_t e = launch();  // warm-up
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  int launches = 0;
  double ms_total = 0.0;
  auto t0 = std::chrono::steady_clock::now();
  while (e == cudaSuccess) {
    e = cudaEventRecord(e0, ctx->stream);
    for (int k = 0; k < 4 && e == cudaSuccess; ++k) e = launch();
    if (e == cudaSuccess) e = cudaEventRecord(e1, ctx->stream);
    if (e == cudaSuccess) e = cudaEventSynchronize(e1);
    float ms = 0.f;
    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
    ms_total += ms;
    launches += 4;
    if (std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count() >= seconds)
      break;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "peak probe");
  const double fmas = (double)launches * blocks * threads * (double)iters * 16.0 * kPeakChains;
  *gflops = 2.0 * fmas / (ms_total * 1e-3) * 1e-9;
  return PAWAN_OK;
}

int pawan_peak_fp32(pawan_ctx *ctx, double seconds, double *gflops) {
  if (!gflops) return PAWAN_ERR_INVALID;
  double a = 0, b = 0;
  PAWAN_TRY(run_peak(ctx, 0.5 * seconds, &a, 0));
  PAWAN_TRY(run_peak(ctx, 0.5 * seconds, &b, 2));
  *gflops = a > b ? a : b;
  return PAWAN_OK;
}

int pawan_peak_fp64(pawan_ctx *ctx, double seconds, double *gflops) {
  return run_peak(ctx, seconds, gflops, 1);
}

}  // extern "C"

// Serving engine: a request loop with device-resident particle state and
// continuous batching.
//
// Each request is a system (one ring, a ring pair, ...) with its own nu, dt
// and step count.  The worker thread repeats: admit waiting requests in
// arrival order (or least work first, N^2 x steps, with the shortest-first
// policy) while the device-memory budget, the active-request cap and the
// per-iteration work cap (sum N^2) allow; advance every admitted request by
// k RK4 steps in one batched launch sequence per step (one persistent pair
// launch per stage over all of them); retire the finished ones (state copied
// to the host, device memory released).  Requests that arrive while others
// run join at the next iteration, so their work overlaps on the device.
//
// k is the largest step count that neither runs past the first active
// request's last step nor makes the iteration longer than the configured
// target (kIterTarget by default) at the device rate measured so far, so a
// new arrival waits at most
// about that long for admission while few or small active requests do not
// pay one host round trip per step.
//
// A request whose single RK4 step would take longer than the target ("large",
// decided at admission) does not step with the others: it has its own plan
// and advances by slices of its stages' work items, the large requests taking
// turns at about one target of work per iteration.  Small requests
// then keep their pace beside arbitrarily large ones, as with chunked
// prefill in language-model serving.  Its result is unchanged, bit for bit:
// every work item writes its own partial slot whichever launch runs it, and
// a target tile's slots are summed in chunk order by the item that completes
// the tile, in whichever launch that is.
//
// The engine's systems and plans take their device memory from the device's
// memory pool in the order of the engine's stream (cudaMallocAsync /
// cudaFreeAsync): admitting and retiring requests never synchronises the
// device, and a request's particles are packed by the batched plan built
// after its admission instead of a plan of its own.
//
// Sources are chunked in fixed-size chunks per request, so a request's
// arithmetic does not depend on which other requests share its launches: its
// result is the same alone and in the mix, bit for bit.
//
// The engine owns its own context (stream, scheduler counter) on the device of
// the context it was created from, so its worker never shares a stream with
// the caller's thread.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstdint>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <thread>

#include "runtime.h"

using namespace pawan;

namespace {

constexpr int kServeChunkSources = 8192;
constexpr double kIterTarget = 0.02;     // default seconds of device work per iteration
constexpr double kRateGuess = 3e11;      // interactions/s before the first measurement

double now_since(std::chrono::steady_clock::time_point t0) {
  return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

struct Request {
  long long id = 0;
  int state = PAWAN_REQ_QUEUED;
  std::vector<size_t> counts;
  std::vector<double> pos, vor, rad, vol;
  double nu = 0.0, dt = 0.0;
  size_t nsteps = 0, steps_done = 0;
  size_t n = 0;
  double bytes = 0.0;
  double t_submit = 0.0, t_admit = -1.0, t_done = -1.0;
  bool cancel = false;
  pawan_system *sys = nullptr;
  // a request whose RK4 step costs more than an iteration ("large"): its own
  // plan, and the stage / work item it has reached
  bool large = false;
  std::unique_ptr<Plan> plan;
  int stage = 0, next_item = 0;
  std::vector<double> result;
};

// Device bytes a request holds while active: the system's buffers plus its
// rates and partial slots in a batched plan (fixed chunk size; slots cover
// whole target tiles of at most 512 particles).
double request_bytes(size_t n, const TileChoice &tile) {
  const int tb = tile.pc.tb;
  const double per = 5 * 48.0 + 16.0 + 4.0 + 64.0 + 64.0 + 1.0 + 48.0;
  const size_t chunk = ((kServeChunkSources + tb - 1) / tb) * (size_t)tb;
  const size_t nch = (n + chunk - 1) / chunk;
  const double slots = nch > 1 ? 48.0 * (double)(n + 512) * (double)nch : 0.0;
  // a separate near pass keeps its sums in slots of its own (every chunk, one
  // chunk included) with a flag byte each
  const double near = tile.pc.split > 0 ? 49.0 * (double)(n + 512) * (double)nch : 0.0;
  return (double)n * per + slots + near + 4096.0;
}

// The engine's tiling: for FP32 the packed far path with the packed near pass
// (requests are rings of a few thousand to a few hundred thousand particles,
// where the near tile pairs are a tenth of the work for the small ones); the
// library default otherwise.
TileChoice serve_tile(int precision) {
  TileChoice t = default_tile(precision);
  if (precision == PAWAN_PREC_F32) t.pc = PairConfig{128, 1, 4, 1, 0, 1, 2};
  return t;
}

}  // namespace

struct pawan_server {
  pawan_ctx *ctx = nullptr;  // owned, worker-thread only
  pawan_serve_config cfg{};
  std::thread worker;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  bool stop = false;
  std::deque<long long> queue;
  std::map<long long, std::unique_ptr<Request>> reqs;
  std::vector<Request *> active;
  long long next_id = 1;
  std::chrono::steady_clock::time_point t0;
  pawan_serve_stats stats{};
  double bytes_in_use = 0.0;
  std::string worker_error;
  TileChoice tile;
  double rate = kRateGuess;  // measured interactions/s of the iterations (worker only)
  cudaMemPool_t pool = nullptr;
  // host-side fault injection (pawan_server_inject), under `mu`
  int fail_alloc = 0, fail_iteration = 0, slow_iterations = 0;
  double slow_seconds = 0.0;
};

namespace {

// Consumes one pending injected fault of a kind (call with `mu` held).
bool take(int &pending) {
  if (pending <= 0) return false;
  --pending;
  return true;
}

void finish(pawan_server *srv, Request *r, int state) {
  r->state = state;
  r->t_done = now_since(srv->t0);
}

// Builds the batched plan over the admitted requests (when the set changed);
// called without the lock.
int plan_iteration(pawan_server *srv, std::vector<Request *> &act, std::unique_ptr<Plan> &plan,
                   bool rebuild) {
  pawan_ctx *ctx = srv->ctx;
  if (rebuild || !plan) {
    plan.reset();
    std::vector<pawan_system *> sys;
    for (Request *r : act) sys.push_back(r->sys);
    int st = build_plan(ctx, sys, srv->cfg.precision, srv->tile, plan, kServeChunkSources, true);
    if (st != PAWAN_OK) return st;
  }
  std::vector<double> dts;
  for (Request *r : act) dts.push_back(r->dt);
  return set_plan_dt(ctx, *plan, dts.data(), 0.0);
}

// A slice of a large request's stage work, about `budget` interactions (at
// least one work item per resident block of the pair kernel, so the slice
// fills the device; on into the following stages while the budget lasts).
// Each work item writes its own partial slot and the tile counters carry over
// between launches, so splitting a stage over launches changes nothing in the
// result.  Adds the interactions done to *work.
int large_slice(pawan_server *srv, Request *r, double budget, double *work) {
  static const int modes[4] = {STAGE_K1, STAGE_K2, STAGE_K3, STAGE_FINAL};
  pawan_ctx *ctx = srv->ctx;
  Plan &p = *r->plan;
  double used = 0.0;
  while (r->steps_done < r->nsteps) {
    // at least one work item per resident block (a slice fills the device)
    int b = r->next_item;
    double acc = 0.0;
    while (b < p.n_items &&
           (b - r->next_item < p.grid || used + acc + p.item_costs[b] <= budget)) {
      acc += p.item_costs[b];
      ++b;
    }
    int st = launch_pairs_range(ctx, p, r->next_item, b - r->next_item);
    if (st != PAWAN_OK) return st;
    used += acc;
    r->next_item = b;
    if (b < p.n_items) break;  // budget spent mid-stage
    st = launch_stage_mode(ctx, p, modes[r->stage]);
    if (st != PAWAN_OK) return st;
    r->next_item = 0;
    if (++r->stage == 4) {
      r->stage = 0;
      r->steps_done++;
    }
    if (used >= budget) break;
  }
  *work += used;
  return PAWAN_OK;
}

// Steps per iteration (see the file comment).
size_t steps_per_iteration(const pawan_server *srv, const std::vector<Request *> &act) {
  size_t min_left = ~(size_t)0;
  double n2 = 0.0;
  for (const Request *r : act) {
    min_left = std::min(min_left, r->nsteps - r->steps_done);
    n2 += (double)r->n * (double)r->n;
  }
  const double step_s = 4.0 * n2 / std::max(1e9, srv->rate);
  const double target = srv->cfg.iteration_seconds > 0.0 ? srv->cfg.iteration_seconds : kIterTarget;
  const double fit = std::floor(target / std::max(1e-9, step_s));
  const size_t k = fit < 1.0 ? 1 : (fit > 1e6 ? (size_t)1000000 : (size_t)fit);
  return std::max<size_t>(1, std::min(k, min_left));
}

void worker_main(pawan_server *srv) {
  cudaSetDevice(srv->ctx->device);
  std::unique_ptr<Plan> plan;
  bool set_changed = true;
  size_t large_turn = 0;  // the large request that goes first this iteration
  for (;;) {
    std::vector<Request *> admit;
    {
      std::unique_lock<std::mutex> lk(srv->mu);
      if (srv->cfg.policy == PAWAN_SERVE_SHORTEST_FIRST && srv->queue.size() > 1) {
        // least work (N^2 x steps) first; arrival order among equals
        std::stable_sort(srv->queue.begin(), srv->queue.end(), [&](long long a, long long b) {
          const Request *ra = srv->reqs[a].get(), *rb = srv->reqs[b].get();
          return (double)ra->n * (double)ra->n * (double)ra->nsteps <
                 (double)rb->n * (double)rb->n * (double)rb->nsteps;
        });
      }
      for (;;) {
        // admission in queue order (arrival order, or least work first), no
        // overtaking of a request the caps hold back, within all caps
        if (srv->queue.empty()) break;
        Request *r = srv->reqs[srv->queue.front()].get();
        const size_t na = srv->active.size() + admit.size();
        double n2 = (double)r->n * (double)r->n;
        for (Request *a : srv->active) n2 += (double)a->n * (double)a->n;
        for (Request *a : admit) n2 += (double)a->n * (double)a->n;
        const bool empty = na == 0;
        if (srv->bytes_in_use + r->bytes > srv->cfg.budget_bytes) break;
        if (srv->cfg.max_active > 0 && (int)na >= srv->cfg.max_active) break;
        if (srv->cfg.max_step_interactions > 0 && n2 > srv->cfg.max_step_interactions && !empty)
          break;
        srv->queue.pop_front();
        srv->bytes_in_use += r->bytes;
        r->state = PAWAN_REQ_ACTIVE;
        r->t_admit = now_since(srv->t0);
        admit.push_back(r);
      }
      if (srv->active.empty() && admit.empty()) {
        if (srv->stop) break;
        srv->cv_work.wait_for(lk, std::chrono::milliseconds(50));
        continue;
      }
      if (srv->stop && admit.empty() && srv->active.empty()) break;
    }
    // create device state of newly admitted requests (outside the lock)
    const auto ta0 = std::chrono::steady_clock::now();
    for (Request *r : admit) {
      bool injected;
      {
        std::lock_guard<std::mutex> lk(srv->mu);
        injected = take(srv->fail_alloc);
      }
      int st = injected ? fail(srv->ctx, PAWAN_ERR_NOMEM, "injected allocation failure")
                        : system_create_ordered(srv->ctx, r->counts.size(), r->counts.data(),
                                                r->nu, srv->cfg.precision, &r->sys);
      if (st == PAWAN_OK)
        st = system_upload(r->sys, r->pos.data(), r->vor.data(), r->rad.data(), r->vol.data());
      std::lock_guard<std::mutex> lk(srv->mu);
      if (st != PAWAN_OK) {
        srv->worker_error = srv->ctx->err;
        if (r->sys) pawan_system_destroy(r->sys);
        r->sys = nullptr;
        srv->bytes_in_use -= r->bytes;
        finish(srv, r, PAWAN_REQ_REJECTED);
        srv->stats.rejected++;
        srv->cv_done.notify_all();
        continue;
      }
      // (the pageable particle copies were staged before system_upload returned)
      std::vector<double>().swap(r->pos);
      std::vector<double>().swap(r->vor);
      const double target = srv->cfg.iteration_seconds > 0.0 ? srv->cfg.iteration_seconds : kIterTarget;
      r->large = 4.0 * (double)r->n * (double)r->n / std::max(1e9, srv->rate) > target;
      srv->active.push_back(r);
      srv->stats.admitted++;
      set_changed = true;
    }
    if (!admit.empty()) {
      std::lock_guard<std::mutex> lk(srv->mu);
      srv->stats.admit_seconds +=
          std::chrono::duration<double>(std::chrono::steady_clock::now() - ta0).count();
    }
    std::vector<Request *> act;
    {
      std::lock_guard<std::mutex> lk(srv->mu);
      act = srv->active;
    }
    if (act.empty()) continue;
    // requests that step together, and large ones that advance by slices
    std::vector<Request *> reg, big;
    for (Request *r : act) (r->large ? big : reg).push_back(r);
    const auto tp0 = std::chrono::steady_clock::now();
    int st = PAWAN_OK;
    if (!reg.empty()) {
      st = plan_iteration(srv, reg, plan, set_changed);
    } else {
      plan.reset();
    }
    for (Request *r : big) {
      if (st != PAWAN_OK || r->plan) continue;
      st = build_plan(srv->ctx, {r->sys}, srv->cfg.precision, srv->tile, r->plan, kServeChunkSources, true);
      if (st == PAWAN_OK) st = set_plan_dt(srv->ctx, *r->plan, &r->dt, 0.0);
    }
    set_changed = false;
    const auto it0 = std::chrono::steady_clock::now();
    size_t k = 0;
    double n2 = 0.0, work = 0.0;
    for (Request *r : reg) n2 += (double)r->n * (double)r->n;
    bool inj_fail = false, inj_slow = false;
    double slow_s = 0.0;
    {
      std::lock_guard<std::mutex> lk(srv->mu);
      inj_fail = take(srv->fail_iteration);
      inj_slow = take(srv->slow_iterations);
      slow_s = srv->slow_seconds;
    }
    if (inj_slow) std::this_thread::sleep_for(std::chrono::duration<double>(slow_s));
    if (st == PAWAN_OK && inj_fail) st = fail(srv->ctx, PAWAN_ERR_CUDA, "injected iteration failure");
    if (st == PAWAN_OK && !reg.empty()) {
      k = steps_per_iteration(srv, reg);
      st = rk4_steps(srv->ctx, *plan, k, k >= 3);
      work += 4.0 * n2 * (double)k;
    }
    if (st == PAWAN_OK && !big.empty()) {
      // about one iteration target of work for the large requests, in turn
      // (round robin over iterations), so that each slice is large enough to
      // fill the device
      const double target = srv->cfg.iteration_seconds > 0.0 ? srv->cfg.iteration_seconds : kIterTarget;
      double budget = target * std::max(1e9, srv->rate);
      for (size_t j = 0; j < big.size() && budget > 0.0 && st == PAWAN_OK; ++j) {
        Request *r = big[(large_turn + j) % big.size()];
        const double before = work;
        st = large_slice(srv, r, budget, &work);
        budget -= work - before;
      }
      large_turn = (large_turn + 1) % std::max<size_t>(1, big.size());
    }
    if (st == PAWAN_OK) {
      cudaError_t e = cudaStreamSynchronize(srv->ctx->stream);
      if (e != cudaSuccess) st = cuda_fail(srv->ctx, e, "serving iteration");
    }
    const auto it1 = std::chrono::steady_clock::now();
    const double busy = std::chrono::duration<double>(it1 - it0).count();
    if (st == PAWAN_OK && busy > 0.0 && work > 0.0) {
      // device rate of this iteration, smoothed (for the next step counts)
      srv->rate = 0.5 * srv->rate + 0.5 * work / busy;
    }
    // retire finished / cancelled requests
    std::vector<Request *> done;
    {
      std::lock_guard<std::mutex> lk(srv->mu);
      srv->stats.iterations++;
      srv->stats.busy_seconds += busy;
      srv->stats.plan_seconds += std::chrono::duration<double>(it0 - tp0).count();
      if (st != PAWAN_OK) srv->worker_error = srv->ctx->err;
      if (st == PAWAN_OK) {
        for (Request *r : reg) r->steps_done += k;
        srv->stats.interactions += work;
      }
      for (Request *r : act)
        if (st != PAWAN_OK || r->cancel || r->steps_done >= r->nsteps) done.push_back(r);
    }
    const auto tr0 = std::chrono::steady_clock::now();
    for (Request *r : done) {
      int state = PAWAN_REQ_DONE;
      if (st != PAWAN_OK) {
        state = PAWAN_REQ_REJECTED;
      } else if (r->cancel) {
        state = PAWAN_REQ_CANCELLED;
      } else {
        r->result.resize(6 * r->n);
        if (pawan_system_get_states(r->sys, r->result.data(), r->result.size()) != PAWAN_OK)
          state = PAWAN_REQ_REJECTED;
      }
      r->plan.reset();
      pawan_system_destroy(r->sys);
      r->sys = nullptr;
      std::lock_guard<std::mutex> lk(srv->mu);
      srv->active.erase(std::find(srv->active.begin(), srv->active.end(), r));
      srv->bytes_in_use -= r->bytes;
      finish(srv, r, state);
      if (state == PAWAN_REQ_DONE) srv->stats.completed++;
      else if (state == PAWAN_REQ_REJECTED) srv->stats.rejected++;
      set_changed = true;
    }
    if (!done.empty()) {
      std::lock_guard<std::mutex> lk(srv->mu);
      srv->stats.retire_seconds +=
          std::chrono::duration<double>(std::chrono::steady_clock::now() - tr0).count();
      srv->cv_done.notify_all();
    }
  }
  plan.reset();
  cudaStreamSynchronize(srv->ctx->stream);  // the plan's buffers are back in the pool
}

}  // namespace

extern "C" {

int pawan_server_get_tiling(pawan_server *srv, pawan_tiling *out) {
  if (!srv || !out) return PAWAN_ERR_INVALID;
  const TileChoice &t = srv->tile;
  out->threads = t.pc.tb;
  out->threads_per_target = t.pc.p;
  out->targets_per_thread = t.pc.r;
  out->unroll = t.pc.unroll;
  out->blocks_per_sm = t.pc.minb;
  out->packed = t.pc.packed;
  out->split_near = t.pc.split;
  out->items_per_slot = t.items_per_slot;
  return PAWAN_OK;
}

int pawan_server_create(pawan_ctx *ctx, const pawan_serve_config *cfg, pawan_server **out) {
  if (!ctx || !cfg || !out) return PAWAN_ERR_INVALID;
  if (!(cfg->budget_bytes > 0) || cfg->precision < PAWAN_PREC_F32 ||
      cfg->precision > PAWAN_PREC_F64_PLAIN || !(cfg->iteration_seconds >= 0.0) ||
      (cfg->policy != PAWAN_SERVE_FIFO && cfg->policy != PAWAN_SERVE_SHORTEST_FIRST))
    return fail(ctx, PAWAN_ERR_INVALID, "bad serving configuration");
  std::unique_ptr<pawan_server> srv(new pawan_server());
  srv->cfg = *cfg;
  srv->tile = serve_tile(cfg->precision);
  int st = pawan_ctx_create(ctx->device, &srv->ctx);
  if (st != PAWAN_OK) return fail(ctx, st, "cannot create the serving context");
  // freed request memory stays in the device's pool for the next admission
  // (it goes back to the system when the engine is destroyed)
  if (cudaDeviceGetDefaultMemPool(&srv->pool, srv->ctx->device) == cudaSuccess) {
    uint64_t keep = UINT64_MAX;
    cudaMemPoolSetAttribute(srv->pool, cudaMemPoolAttrReleaseThreshold, &keep);
  } else {
    srv->pool = nullptr;
  }
  srv->t0 = std::chrono::steady_clock::now();
  pawan_server *raw = srv.get();
  try {
    srv->worker = std::thread(worker_main, raw);
  } catch (...) {
    pawan_ctx_destroy(srv->ctx);
    return fail(ctx, PAWAN_ERR_NOMEM, "cannot start the serving thread");
  }
  *out = srv.release();
  return PAWAN_OK;
}

void pawan_server_destroy(pawan_server *srv) {
  if (!srv) return;
  {
    std::lock_guard<std::mutex> lk(srv->mu);
    srv->stop = true;
    // queued requests never start; active ones are cancelled at the next iteration
    for (long long id : srv->queue) finish(srv, srv->reqs[id].get(), PAWAN_REQ_CANCELLED);
    srv->queue.clear();
    for (Request *r : srv->active) r->cancel = true;
  }
  srv->cv_work.notify_all();
  if (srv->worker.joinable()) srv->worker.join();
  for (auto &kv : srv->reqs) {
    kv.second->plan.reset();
    if (kv.second->sys) pawan_system_destroy(kv.second->sys);
  }
  cudaStreamSynchronize(srv->ctx->stream);
  if (srv->pool) cudaMemPoolTrimTo(srv->pool, 0);
  pawan_ctx_destroy(srv->ctx);
  delete srv;
}

int pawan_server_submit(pawan_server *srv, size_t n_wakes, const size_t *num_particles,
                        const double *position, const double *vorticity, const double *radius,
                        const double *volume, double nu, double dt, size_t nsteps,
                        long long *id) {
  if (!srv || !id || n_wakes == 0 || !num_particles || !position || !vorticity || !radius ||
      !volume || nsteps == 0 || !(dt > 0) || !(nu >= 0))
    return PAWAN_ERR_INVALID;
  std::unique_ptr<Request> r(new Request());
  size_t n = 0;
  for (size_t w = 0; w < n_wakes; ++w) {
    if (num_particles[w] == 0) return PAWAN_ERR_INVALID;
    r->counts.push_back(num_particles[w]);
    n += num_particles[w];
  }
  if (n < 2) return PAWAN_ERR_INVALID;
  r->n = n;
  r->nu = nu;
  r->dt = dt;
  r->nsteps = nsteps;
  r->bytes = request_bytes(n, srv->tile);
  std::lock_guard<std::mutex> lk(srv->mu);
  r->id = srv->next_id++;
  r->t_submit = now_since(srv->t0);
  *id = r->id;
  srv->stats.submitted++;
  if (srv->stop) {
    finish(srv, r.get(), PAWAN_REQ_REJECTED);
    srv->stats.rejected++;
    srv->reqs[r->id] = std::move(r);
    return PAWAN_ERR_REJECTED;
  }
  if (r->bytes > srv->cfg.budget_bytes) {
    finish(srv, r.get(), PAWAN_REQ_REJECTED);
    srv->stats.rejected++;
    srv->reqs[r->id] = std::move(r);
    return PAWAN_ERR_BUDGET;
  }
  if (srv->cfg.max_queue > 0 && (int)srv->queue.size() >= srv->cfg.max_queue) {
    finish(srv, r.get(), PAWAN_REQ_REJECTED);
    srv->stats.rejected++;
    srv->reqs[r->id] = std::move(r);
    return PAWAN_ERR_REJECTED;
  }
  r->pos.assign(position, position + 3 * n);
  r->vor.assign(vorticity, vorticity + 3 * n);
  r->rad.assign(radius, radius + n);
  r->vol.assign(volume, volume + n);
  srv->queue.push_back(r->id);
  srv->reqs[r->id] = std::move(r);
  srv->cv_work.notify_all();
  return PAWAN_OK;
}

int pawan_server_poll(pawan_server *srv, long long id, int *state) {
  if (!srv || !state) return PAWAN_ERR_INVALID;
  std::lock_guard<std::mutex> lk(srv->mu);
  auto it = srv->reqs.find(id);
  if (it == srv->reqs.end()) return PAWAN_ERR_NOTFOUND;
  *state = it->second->state;
  return PAWAN_OK;
}

int pawan_server_wait(pawan_server *srv, long long id, double timeout_s) {
  if (!srv) return PAWAN_ERR_INVALID;
  std::unique_lock<std::mutex> lk(srv->mu);
  auto deadline = std::chrono::steady_clock::now() +
                  std::chrono::duration_cast<std::chrono::steady_clock::duration>(
                      std::chrono::duration<double>(std::max(0.0, timeout_s)));
  for (;;) {
    auto it = srv->reqs.find(id);
    if (it == srv->reqs.end()) return PAWAN_ERR_NOTFOUND;
    const int s = it->second->state;
    if (s == PAWAN_REQ_DONE || s == PAWAN_REQ_REJECTED || s == PAWAN_REQ_CANCELLED)
      return PAWAN_OK;
    if (srv->cv_done.wait_until(lk, deadline) == std::cv_status::timeout) {
      auto it2 = srv->reqs.find(id);
      if (it2 != srv->reqs.end()) {
        const int s2 = it2->second->state;
        if (s2 == PAWAN_REQ_DONE || s2 == PAWAN_REQ_REJECTED || s2 == PAWAN_REQ_CANCELLED)
          return PAWAN_OK;
      }
      return PAWAN_ERR_TIMEOUT;
    }
  }
}

int pawan_server_fetch(pawan_server *srv, long long id, double *state, size_t size,
                       double *t_submit, double *t_admit, double *t_done) {
  if (!srv) return PAWAN_ERR_INVALID;
  std::lock_guard<std::mutex> lk(srv->mu);
  auto it = srv->reqs.find(id);
  if (it == srv->reqs.end()) return PAWAN_ERR_NOTFOUND;
  Request *r = it->second.get();
  if (r->state == PAWAN_REQ_QUEUED || r->state == PAWAN_REQ_ACTIVE) return PAWAN_ERR_STATE;
  if (t_submit) *t_submit = r->t_submit;
  if (t_admit) *t_admit = r->t_admit;
  if (t_done) *t_done = r->t_done;
  const int s = r->state;
  if (s == PAWAN_REQ_DONE) {
    if (!state || size != r->result.size()) return PAWAN_ERR_INVALID;
    std::memcpy(state, r->result.data(), size * sizeof(double));
  }
  srv->reqs.erase(it);
  return s == PAWAN_REQ_DONE ? PAWAN_OK : (s == PAWAN_REQ_CANCELLED ? PAWAN_ERR_STATE : PAWAN_ERR_REJECTED);
}

int pawan_server_cancel(pawan_server *srv, long long id) {
  if (!srv) return PAWAN_ERR_INVALID;
  std::lock_guard<std::mutex> lk(srv->mu);
  auto it = srv->reqs.find(id);
  if (it == srv->reqs.end()) return PAWAN_ERR_NOTFOUND;
  Request *r = it->second.get();
  if (r->state == PAWAN_REQ_QUEUED) {
    srv->queue.erase(std::find(srv->queue.begin(), srv->queue.end(), id));
    finish(srv, r, PAWAN_REQ_CANCELLED);
    srv->cv_done.notify_all();
  } else if (r->state == PAWAN_REQ_ACTIVE) {
    r->cancel = true;
  }
  return PAWAN_OK;
}

int pawan_server_inject(pawan_server *srv, int fault, int count, double seconds) {
  if (!srv || count < 0) return PAWAN_ERR_INVALID;
  std::lock_guard<std::mutex> lk(srv->mu);
  switch (fault) {
    case PAWAN_FAULT_ALLOC:
      srv->fail_alloc = count;
      break;
    case PAWAN_FAULT_ITERATION:
      srv->fail_iteration = count;
      break;
    case PAWAN_FAULT_SLOW:
      if (!(seconds >= 0.0) || seconds > 60.0) return PAWAN_ERR_INVALID;
      srv->slow_iterations = count;
      srv->slow_seconds = seconds;
      break;
    default:
      return PAWAN_ERR_INVALID;
  }
  srv->cv_work.notify_all();
  return PAWAN_OK;
}

int pawan_server_stats(pawan_server *srv, pawan_serve_stats *out) {
  if (!srv || !out) return PAWAN_ERR_INVALID;
  std::lock_guard<std::mutex> lk(srv->mu);
  *out = srv->stats;
  out->queued = srv->queue.size();
  out->active = srv->active.size();
  out->bytes_in_use = srv->bytes_in_use;
  return PAWAN_OK;
}

}  // extern "C"

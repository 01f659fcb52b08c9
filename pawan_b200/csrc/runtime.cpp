// Host runtime and C ABI of the pawan B200 library: contexts, systems (the
// reference's __interaction with its wakes), execution plans over one or many
// systems, RK4 driving, diagnostics, autotuning and throughput probes.
#include "runtime.h"

#include <nvtx3/nvToolsExt.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <numeric>

using namespace pawan;

namespace pawan {

int fail(pawan_ctx *ctx, int code, const std::string &msg) {
  if (ctx) ctx->err = msg;
  return code;
}

int cuda_fail(pawan_ctx *ctx, cudaError_t e, const char *where) {
  std::string m = std::string(where) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")";
  if (e == cudaErrorMemoryAllocation) return fail(ctx, PAWAN_ERR_NOMEM, m);
  return fail(ctx, PAWAN_ERR_CUDA, m);
}

#define PAWAN_CUDA(ctx, expr)                                  \
  do {                                                         \
    cudaError_t e_ = (expr);                                   \
    if (e_ != cudaSuccess) return cuda_fail((ctx), e_, #expr); \
  } while (0)

#define PAWAN_TRY(expr)             \
  do {                              \
    int s_ = (expr);                \
    if (s_ != PAWAN_OK) return s_;  \
  } while (0)

// Defaults measured on the ring pair and the helical wake (N = 131,072 and
// 262,144): two targets per thread, 256 threads, shallow unroll, fine chunks.
TileChoice default_tile(int precision) {
  TileChoice t;
  if (precision == PAWAN_PREC_F32) {
    t.pc = PairConfig{128, 1, 4, 1, 0, 2};  // packed far path, unroll 4
  } else {
    t.pc = PairConfig{128, 1, 1};
  }
  t.items_per_slot = 32;
  return t;
}

std::vector<TileChoice> tile_candidates(int precision, int kernel) {
  std::vector<TileChoice> v;
  if (precision == PAWAN_PREC_F32) {
    // (threads per target, targets per thread, unroll, blocks per SM) as
    // compiled in pair_f32.cu (0 = the default register bound)
    // (.., packed) among those compiled in pair_f32.cu: the ones that led on
    // some workload (threads per target > 1 for small systems, two targets
    // per thread or packed pairs for large ones)
    const int shapes[][5] = {{1, 1, 4, 0, 0}, {2, 1, 4, 0, 0}, {4, 1, 4, 0, 0}, {1, 2, 1, 0, 0},
                             {1, 2, 2, 0, 0}, {1, 1, 4, 5, 0}, {1, 1, 1, 0, 1}, {1, 1, 2, 0, 1},
                             {1, 1, 4, 0, 1}, {1, 1, 2, 5, 1}, {1, 1, 2, 0, 2}, {1, 1, 4, 0, 2}};
    for (int tb : {128, 256})
      for (const auto &sh : shapes) {
        TileChoice t;
        t.pc = PairConfig{tb, sh[0], sh[2], sh[1], sh[3], sh[4]};
        if (pairs_f32_supported(t.pc, kernel)) v.push_back(t);
      }
  } else {
    for (int tb : {128, 256}) {
      TileChoice t;
      t.pc = PairConfig{tb, 1, 1};
      v.push_back(t);
    }
  }
  return v;
}

Plan::~Plan() {
  if (graph_exec) cudaGraphExecDestroy(graph_exec);
  if (graph) cudaGraphDestroy(graph);
}

bool Plan::stale() const {
  for (size_t s = 0; s < systems.size(); ++s)
    if (systems[s]->nu != nus[s] || systems[s]->geometry_version != geometry_versions[s])
      return true;
  return false;
}

static int occupancy(pawan_ctx *ctx, int precision, const PairConfig &pc, bool diffusion,
                     int kernel, int *bps) {
  cudaError_t e;
  if (precision == PAWAN_PREC_F32)
    e = pairs_f32_occupancy(pc, diffusion, kernel, bps);
  else if (precision == PAWAN_PREC_F64)
    e = pairs_f64_occupancy(pc, diffusion, kernel, bps);
  else
    e = pairs_plain_occupancy(pc, kernel, bps);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "occupancy query");
  if (*bps < 1) return fail(ctx, PAWAN_ERR_INVALID, "pair kernel does not fit on an SM");
  return PAWAN_OK;
}

static bool tile_supported(int precision, const PairConfig &pc, int kernel) {
  if (precision == PAWAN_PREC_F32) return pairs_f32_supported(pc, kernel);
  if (precision == PAWAN_PREC_F64) return pairs_f64_supported(pc, kernel);
  return pairs_plain_supported(pc, kernel);
}

static_assert(PAWAN_KERNEL_HIGHORDER == KERNEL_HIGHORDER && PAWAN_KERNEL_GAUSSIAN == KERNEL_GAUSSIAN,
              "public and device smoothing-kernel codes agree");

// Process blocks of a sharded system start at multiples of kShardAlign
// particles: whole stage blocks and whole target tiles of every tiling.
constexpr size_t kShardAlign = 512;

static size_t shard_first(const pawan_system *y) { return (size_t)y->shard.rank * y->shard.size; }

static size_t shard_count(const pawan_system *y) {
  const size_t f = shard_first(y);
  return f >= y->n ? 0 : std::min(y->shard.size, y->n - f);
}

// Work decomposition.  Target tiles of tb/p particles; sources in chunks of
// whole tb-tiles sized so that the launch holds about `items_per_slot` items
// per resident block (or of `fixed_chunk_sources` when > 0, which makes a
// system's arithmetic independent of the other systems in the plan).  Items are ordered largest first, so the dynamic
// counter hands out the long ones early (longest-processing-time order).
int build_plan(pawan_ctx *ctx, const std::vector<pawan_system *> &systems, int precision,
               const TileChoice &tile, std::unique_ptr<Plan> &out, int fixed_chunk_sources,
               bool ordered_alloc) {
  if (systems.empty()) return fail(ctx, PAWAN_ERR_INVALID, "plan over no systems");
  const int kernel = systems[0]->kernel;
  for (auto *s : systems)
    if (s->kernel != kernel)
      return fail(ctx, PAWAN_ERR_INVALID, "systems of one plan must share the smoothing kernel");
  if (!tile_supported(precision, tile.pc, kernel))
    return fail(ctx, PAWAN_ERR_INVALID, "unsupported pair tiling for this precision and kernel");
  std::unique_ptr<Plan> p(new Plan());
  p->systems = systems;
  p->precision = precision;
  p->kernel = kernel;
  p->tile = tile;
  for (auto *s : systems) {
    p->nus.push_back(s->nu);
    p->geometry_versions.push_back(s->geometry_version);
    p->box_versions.push_back(~0ull);
    if (s->nu != 0.0) p->diffusion = true;
    const double targets = s->shard.active ? (double)shard_count(s) : (double)s->n;
    p->interactions += targets * (double)s->n;
  }
  int bps = 0;
  PAWAN_TRY(occupancy(ctx, precision, tile.pc, p->diffusion, kernel, &bps));
  p->grid = ctx->sm_count * bps;
  const int TB = tile.pc.tb;
  const int TPB = targets_per_block(tile.pc);
  const double slots = (double)p->grid;
  const double target_pairs =
      std::max(p->interactions / (slots * std::max(1, tile.items_per_slot)), (double)TPB * TB);

  struct ItemCost {
    WorkItem w;
    double cost;
  };
  std::vector<ItemCost> items;
  size_t partial_total = 0, box_total = 0;
  std::vector<size_t> partial_off(systems.size()), box_off(systems.size());
  p->nchunks.resize(systems.size());
  for (size_t s = 0; s < systems.size(); ++s) {
    const int n = (int)systems[s]->n;
    const int src_tiles = (n + TB - 1) / TB;
    int tiles_per_chunk = fixed_chunk_sources > 0
                              ? (fixed_chunk_sources + TB - 1) / TB
                              : (int)std::ceil(target_pairs / ((double)TPB * TB));
    tiles_per_chunk = std::max(1, std::min(tiles_per_chunk, src_tiles));
    const int nch = (src_tiles + tiles_per_chunk - 1) / tiles_per_chunk;
    p->nchunks[s] = nch;
    partial_off[s] = partial_total;
    partial_total += (size_t)nch * 6 * (size_t)n;
    box_off[s] = box_total;
    box_total += 2 * (size_t)src_tiles;
    // targets: all particles, or this process's block of a sharded system
    // (block starts are multiples of kShardAlign, so of every TPB and TB)
    const pawan_system *y = systems[s];
    const int t_lo = y->shard.active ? (int)shard_first(y) : 0;
    const int t_hi = y->shard.active ? t_lo + (int)shard_count(y) : n;
    for (int c = 0; c < nch; ++c) {
      const int s0 = c * tiles_per_chunk * TB;
      const int s1 = std::min(n, (c + 1) * tiles_per_chunk * TB);
      for (int t0 = t_lo; t0 < t_hi; t0 += TPB) {
        const int nt = std::min(TPB, t_hi - t0);
        items.push_back({WorkItem{(int)s, t0, c, s0, s1}, (double)nt * (double)(s1 - s0)});
      }
    }
  }
  std::stable_sort(items.begin(), items.end(),
                   [](const ItemCost &a, const ItemCost &b) { return a.cost > b.cost; });
  if (items.size() > (size_t)INT32_MAX) return fail(ctx, PAWAN_ERR_INVALID, "too many work items");
  p->n_items = (int)items.size();

  if (ordered_alloc) {
    p->partial.ordered_on(ctx->stream);
    p->boxes.ordered_on(ctx->stream);
    p->items.ordered_on(ctx->stream);
    p->segs.ordered_on(ctx->stream);
    p->stage_items.ordered_on(ctx->stream);
    p->shard_items.ordered_on(ctx->stream);
    p->stage_descs.ordered_on(ctx->stream);
  }
  PAWAN_CUDA(ctx, p->partial.alloc(partial_total));
  PAWAN_CUDA(ctx, p->boxes.alloc(box_total));
  std::vector<WorkItem> wh(items.size());
  p->item_costs.resize(items.size());
  for (size_t k = 0; k < items.size(); ++k) {
    wh[k] = items[k].w;
    p->item_costs[k] = items[k].cost;  // target x source pairs of the item
  }
  std::vector<SegDesc> sh(systems.size());
  std::vector<StageItem> sih, shh;
  p->stage_host.resize(systems.size());
  for (size_t s = 0; s < systems.size(); ++s) {
    pawan_system *y = systems[s];
    SegDesc &d = sh[s];
    d.pos32 = y->pos32.p;
    d.vor32 = y->vor32.p;
    d.poslo = y->poslo.p;
    d.vorlo = y->vorlo.p;
    d.pos64 = y->pos64.p;
    d.vor64 = y->vor64.p;
    d.boxes = p->boxes.p + box_off[s];
    d.partial = p->partial.p + partial_off[s];
    d.n = (int)y->n;
    d.nchunks = p->nchunks[s];
    d.nu = y->nu;
    d.near2 = (float)(y->r_near * y->r_near);
    StageDesc &g = p->stage_host[s];
    g.partial = d.partial;
    g.nchunks = d.nchunks;
    g.n = d.n;
    g.X = y->X.p;
    g.Xs = y->Xs.p;
    g.K1 = y->K1.p;
    g.K2 = y->K2.p;
    g.R = y->R.p;
    g.rad = y->rad.p;
    g.vol = y->vol.p;
    g.pos32 = y->pos32.p;
    g.vor32 = y->vor32.p;
    g.poslo = y->poslo.p;
    g.vorlo = y->vorlo.p;
    g.pos64 = y->pos64.p;
    g.vor64 = y->vor64.p;
    g.boxes = p->boxes.p + box_off[s];
    g.box_tile = TB;
    g.ox = y->ox;
    g.oy = y->oy;
    g.oz = y->oz;
    g.dt = 0.0;
    g.xchg_out = y->shard.active ? y->shard.send : nullptr;
    g.xchg_in = y->shard.active ? y->shard.recv : nullptr;
    g.shard = y->shard.active ? (int)y->shard.size : 0;
    g.shard_first = y->shard.active ? (int)shard_first(y) : 0;
    for (int l0 = 0; l0 < d.n; l0 += kStageThreads) sih.push_back(StageItem{(int)s, l0});
    if (y->shard.active) {
      const int f = (int)shard_first(y), e = f + (int)shard_count(y);
      for (int l0 = f; l0 < e; l0 += kStageThreads) shh.push_back(StageItem{(int)s, l0});
    }
  }
  p->n_stage_blocks = (int)sih.size();
  p->n_shard_blocks = (int)shh.size();
  p->dts.assign(systems.size(), 0.0);
  PAWAN_CUDA(ctx, p->items.alloc(wh.size()));
  PAWAN_CUDA(ctx, p->segs.alloc(sh.size()));
  PAWAN_CUDA(ctx, p->stage_items.alloc(sih.size()));
  PAWAN_CUDA(ctx, p->stage_descs.alloc(sh.size()));
  PAWAN_CUDA(ctx, cudaMemcpyAsync(p->items.p, wh.data(), wh.size() * sizeof(WorkItem),
                                  cudaMemcpyHostToDevice, ctx->stream));
  PAWAN_CUDA(ctx, cudaMemcpyAsync(p->segs.p, sh.data(), sh.size() * sizeof(SegDesc),
                                  cudaMemcpyHostToDevice, ctx->stream));
  PAWAN_CUDA(ctx, cudaMemcpyAsync(p->stage_items.p, sih.data(), sih.size() * sizeof(StageItem),
                                  cudaMemcpyHostToDevice, ctx->stream));
  if (!shh.empty()) {
    PAWAN_CUDA(ctx, p->shard_items.alloc(shh.size()));
    PAWAN_CUDA(ctx, cudaMemcpyAsync(p->shard_items.p, shh.data(), shh.size() * sizeof(StageItem),
                                    cudaMemcpyHostToDevice, ctx->stream));
  }
  PAWAN_CUDA(ctx, cudaMemcpyAsync(p->stage_descs.p, p->stage_host.data(),
                                  p->stage_host.size() * sizeof(StageDesc), cudaMemcpyHostToDevice,
                                  ctx->stream));
  out = std::move(p);
  // the plan's tile boxes: repack the current states (idempotent for the
  // packed arrays, which already hold pack(X) between API calls)
  PAWAN_TRY(launch_stage_mode(ctx, *out, STAGE_PACK));
  // (the host tables were staged by the copies above; an ordered plan is used
  // on the same stream, so only the others wait here)
  if (!ordered_alloc) PAWAN_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return PAWAN_OK;
}

// Puts each system's dt into the device stage table (only when it changed).
int set_plan_dt(pawan_ctx *ctx, Plan &p, const double *dt, double dt0) {
  bool changed = false;
  for (size_t s = 0; s < p.systems.size(); ++s) {
    const double v = dt ? dt[s] : dt0;
    if (!(v > 0.0) || !std::isfinite(v)) return fail(ctx, PAWAN_ERR_INVALID, "dt must be positive");
    if (p.dts[s] != v) {
      p.dts[s] = v;
      p.stage_host[s].dt = v;
      changed = true;
    }
  }
  if (changed) {
    PAWAN_CUDA(ctx, cudaMemcpyAsync(p.stage_descs.p, p.stage_host.data(),
                                    p.stage_host.size() * sizeof(StageDesc),
                                    cudaMemcpyHostToDevice, ctx->stream));
  }
  return PAWAN_OK;
}

static cudaEvent_t take_event(pawan_ctx *ctx) {
  if (!ctx->event_pool.empty()) {
    cudaEvent_t e = ctx->event_pool.back();
    ctx->event_pool.pop_back();
    return e;
  }
  cudaEvent_t e = nullptr;
  if (cudaEventCreate(&e) != cudaSuccess) return nullptr;
  return e;
}

int launch_pairs(pawan_ctx *ctx, Plan &p, bool allow_events) {
  return launch_pairs_range(ctx, p, 0, p.n_items, allow_events);
}

int launch_pairs_range(pawan_ctx *ctx, Plan &p, int first, int count, bool allow_events) {
  if (first < 0 || count < 0 || first + count > p.n_items)
    return fail(ctx, PAWAN_ERR_INVALID, "work-item range outside the plan");
  const WorkItem *items = p.items.p + first;
  for (size_t s = 0; s < p.systems.size(); ++s)
    if (p.box_versions[s] != p.systems[s]->pack_version) {
      // another plan repacked these systems since this plan's boxes were made
      PAWAN_TRY(launch_stage_mode(ctx, p, STAGE_PACK));
      break;
    }
  PAWAN_CUDA(ctx, cudaMemsetAsync(ctx->d_counter, 0, sizeof(int), ctx->stream));
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (ctx->profile && allow_events) {
    e0 = take_event(ctx);
    e1 = take_event(ctx);
    if (!e0 || !e1) return fail(ctx, PAWAN_ERR_CUDA, "cannot create profiling events");
    PAWAN_CUDA(ctx, cudaEventRecord(e0, ctx->stream));
  }
  cudaError_t e;
  if (p.precision == PAWAN_PREC_F32)
    e = launch_pairs_f32(p.tile.pc, p.diffusion, p.kernel, p.grid, items, count, p.segs.p,
                         ctx->d_counter, ctx->stream);
  else if (p.precision == PAWAN_PREC_F64)
    e = launch_pairs_f64(p.tile.pc, p.diffusion, p.kernel, p.grid, items, count, p.segs.p,
                         ctx->d_counter, ctx->stream);
  else
    e = launch_pairs_plain(p.tile.pc, p.kernel, p.grid, items, count, p.segs.p, ctx->d_counter,
                           ctx->stream);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "pair kernel launch");
  ctx->launches++;
  if (e0) {
    PAWAN_CUDA(ctx, cudaEventRecord(e1, ctx->stream));
    ctx->pending.push_back({e0, e1});
    ctx->pair_launches++;
    double work = 0.0;
    for (int i = first; i < first + count; ++i) work += p.item_costs[i];
    ctx->pair_interactions += work;
  }
  return PAWAN_OK;
}

static void note_repack(Plan &p) {
  for (size_t s = 0; s < p.systems.size(); ++s) {
    p.systems[s]->pack_version++;
    p.box_versions[s] = p.systems[s]->pack_version;
  }
}

// Algorithmic HBM bytes of one stage launch: per particle the chunk partials
// (or the gathered rates of a sharded system), the FP64 state vectors the mode
// reads and writes, radius and volume, and the 128 bytes of packed FP32 / FP64
// tile data; 32 bytes of bounding box per tile.
static double stage_bytes(const Plan &p, int mode) {
  double total = 0.0;
  for (size_t s = 0; s < p.systems.size(); ++s) {
    const pawan_system *y = p.systems[s];
    const double n = (double)y->n;
    const double rates = y->shard.active ? 48.0 : 48.0 * (double)p.nchunks[s];
    const double pack = 16.0 + 128.0 + 32.0 / (double)p.tile.pc.tb;
    double per = 0.0;
    switch (mode) {
      case STAGE_RATES: per = rates + 48.0; break;
      case STAGE_K1: case STAGE_K2: per = rates + 48.0 + 96.0 + pack; break;
      case STAGE_K3: per = rates + 96.0 + 96.0 + pack; break;
      case STAGE_FINAL: per = rates + 144.0 + 48.0 + pack; break;
      case STAGE_EULER: per = rates + 48.0 + 48.0 + pack; break;
      case STAGE_PACK: per = 48.0 + pack; break;
      default: per = 0.0;
    }
    total += n * per;
  }
  return total;
}

int launch_stage_mode(pawan_ctx *ctx, Plan &p, int mode) {
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (ctx->profile) {
    e0 = take_event(ctx);
    e1 = take_event(ctx);
    if (!e0 || !e1) return fail(ctx, PAWAN_ERR_CUDA, "cannot create profiling events");
    PAWAN_CUDA(ctx, cudaEventRecord(e0, ctx->stream));
  }
  cudaError_t e = launch_stage(mode, p.n_stage_blocks, p.stage_items.p, p.stage_descs.p, ctx->stream);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "stage kernel launch");
  ctx->launches++;
  if (e0) {
    PAWAN_CUDA(ctx, cudaEventRecord(e1, ctx->stream));
    ctx->stage_pending.push_back({e0, e1});
    ctx->stage_launches++;
    ctx->stage_bytes += stage_bytes(p, mode);
  }
  if (mode != STAGE_RATES) note_repack(p);
  return PAWAN_OK;
}

// NVTX range over a scope (header-only NVTX; a no-op unless a profiler is
// attached): one per RK4 step and one per stage, so a timeline shows the
// reference's stage structure (rk4.cpp:24-66).
struct NvtxRange {
  explicit NvtxRange(const char *name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
};

static int rk4_one_step(pawan_ctx *ctx, Plan &p, bool allow_events) {
  static const int modes[4] = {STAGE_K1, STAGE_K2, STAGE_K3, STAGE_FINAL};
  static const char *names[4] = {"pawan rk4 k1", "pawan rk4 k2", "pawan rk4 k3", "pawan rk4 k4+update"};
  NvtxRange step("pawan rk4 step");
  for (int s = 0; s < 4; ++s) {
    NvtxRange stage(names[s]);
    PAWAN_TRY(launch_pairs(ctx, p, allow_events));
    PAWAN_TRY(launch_stage_mode(ctx, p, modes[s]));
  }
  return PAWAN_OK;
}

int rk4_steps(pawan_ctx *ctx, Plan &p, size_t nsteps, bool use_graph) {
  if (!use_graph) {
    for (size_t k = 0; k < nsteps; ++k) PAWAN_TRY(rk4_one_step(ctx, p, true));
    return PAWAN_OK;
  }
  if (!p.graph_exec) {
    for (size_t s = 0; s < p.systems.size(); ++s)
      if (p.box_versions[s] != p.systems[s]->pack_version) {
        PAWAN_TRY(launch_stage_mode(ctx, p, STAGE_PACK));
        break;
      }
    PAWAN_CUDA(ctx, cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
    const unsigned long long before = ctx->launches.load();
    int st = rk4_one_step(ctx, p, false);
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(ctx->stream, &g);
    ctx->launches = before;  // capture enqueues nothing; replays count below
    if (st != PAWAN_OK) {
      if (g) cudaGraphDestroy(g);
      return st;
    }
    if (e != cudaSuccess) return cuda_fail(ctx, e, "graph capture");
    p.graph = g;
    PAWAN_CUDA(ctx, cudaGraphInstantiate(&p.graph_exec, g, 0));
  }
  for (size_t k = 0; k < nsteps; ++k) {
    for (size_t s = 0; s < p.systems.size(); ++s)
      if (p.box_versions[s] != p.systems[s]->pack_version) {
        PAWAN_TRY(launch_stage_mode(ctx, p, STAGE_PACK));
        break;
      }
    PAWAN_CUDA(ctx, cudaGraphLaunch(p.graph_exec, ctx->stream));
    ctx->launches += 8;
    for (int st = 0; st < 4; ++st) note_repack(p);
  }
  return PAWAN_OK;
}

int autotune_plan(pawan_ctx *ctx, const std::vector<pawan_system *> &systems, int precision,
                  TileChoice *best) {
  cudaEvent_t e0, e1;
  PAWAN_CUDA(ctx, cudaEventCreate(&e0));
  PAWAN_CUDA(ctx, cudaEventCreate(&e1));
  double best_ms = 1e300;
  TileChoice best_t = default_tile(precision);
  int status = PAWAN_OK;
  auto time_tile = [&](const TileChoice &t, double *ms) -> int {
    std::unique_ptr<Plan> p;
    PAWAN_TRY(build_plan(ctx, systems, precision, t, p));
    PAWAN_TRY(launch_pairs(ctx, *p, false));  // warm-up
    PAWAN_CUDA(ctx, cudaEventRecord(e0, ctx->stream));
    const int reps = 2;
    for (int r = 0; r < reps; ++r) PAWAN_TRY(launch_pairs(ctx, *p, false));
    PAWAN_CUDA(ctx, cudaEventRecord(e1, ctx->stream));
    PAWAN_CUDA(ctx, cudaEventSynchronize(e1));
    float f = 0.f;
    PAWAN_CUDA(ctx, cudaEventElapsedTime(&f, e0, e1));
    *ms = f / reps;
    return PAWAN_OK;
  };
  // 1) tile shape at the default chunking, 2) chunking for the best shape.
  for (const TileChoice &t : tile_candidates(precision, systems[0]->kernel)) {
    double ms = 0;
    status = time_tile(t, &ms);
    if (status != PAWAN_OK) break;
    if (ms < best_ms) {
      best_ms = ms;
      best_t = t;
    }
  }
  if (status == PAWAN_OK) {
    for (int ips : {4, 8, 32, 64, 128}) {
      TileChoice t = best_t;
      t.items_per_slot = ips;
      double ms = 0;
      status = time_tile(t, &ms);
      if (status != PAWAN_OK) break;
      if (ms < best_ms) {
        best_ms = ms;
        best_t = t;
      }
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (status == PAWAN_OK) *best = best_t;
  return status;
}

int system_alloc(pawan_system *sys) {
  pawan_ctx *ctx = sys->ctx;
  const size_t n = sys->n;
  if (sys->ordered_alloc) {
    for (auto *b : {&sys->X, &sys->Xs, &sys->K1, &sys->K2, &sys->R, &sys->rad, &sys->vol,
                    &sys->diag_scratch, &sys->diag_out, &sys->Xc, &sys->field})
      b->ordered_on(ctx->stream);
    sys->wake_id.ordered_on(ctx->stream);
    for (auto *b : {&sys->pos32, &sys->vor32, &sys->poslo, &sys->vorlo}) b->ordered_on(ctx->stream);
    sys->pos64.ordered_on(ctx->stream);
    sys->vor64.ordered_on(ctx->stream);
  }
  PAWAN_CUDA(ctx, sys->X.alloc(6 * n));
  PAWAN_CUDA(ctx, sys->Xs.alloc(6 * n));
  PAWAN_CUDA(ctx, sys->K1.alloc(6 * n));
  PAWAN_CUDA(ctx, sys->K2.alloc(6 * n));
  PAWAN_CUDA(ctx, sys->R.alloc(6 * n));
  PAWAN_CUDA(ctx, sys->rad.alloc(n));
  PAWAN_CUDA(ctx, sys->vol.alloc(n));
  PAWAN_CUDA(ctx, sys->wake_id.alloc(n));
  PAWAN_CUDA(ctx, sys->pos32.alloc(n));
  PAWAN_CUDA(ctx, sys->vor32.alloc(n));
  PAWAN_CUDA(ctx, sys->poslo.alloc(n));
  PAWAN_CUDA(ctx, sys->vorlo.alloc(n));
  PAWAN_CUDA(ctx, sys->pos64.alloc(n));
  PAWAN_CUDA(ctx, sys->vor64.alloc(n));
  PAWAN_CUDA(ctx, sys->diag_scratch.alloc(diag_scratch_doubles((int)n)));
  PAWAN_CUDA(ctx, sys->diag_out.alloc(12));
  std::vector<int> wid(n);
  for (size_t w = 0; w < sys->counts.size(); ++w)
    for (size_t i = 0; i < sys->counts[w]; ++i) wid[sys->offsets[w] + i] = (int)w;
  // on the context's (non-blocking) stream, so later copies on it are ordered after these
  PAWAN_CUDA(ctx, cudaMemcpyAsync(sys->wake_id.p, wid.data(), n * sizeof(int),
                                  cudaMemcpyHostToDevice, ctx->stream));
  PAWAN_CUDA(ctx, cudaMemsetAsync(sys->X.p, 0, 6 * n * sizeof(double), ctx->stream));
  // (the pageable wake ids were staged by the copy; ordered systems are only
  // used on this stream)
  if (!sys->ordered_alloc) PAWAN_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return PAWAN_OK;
}

int system_ensure_plan(pawan_system *sys) {
  if (!sys->has_particles)
    return fail(sys->ctx, PAWAN_ERR_STATE, "particles not set (pawan_system_set_particles)");
  if (sys->plan && !sys->plan->stale() && sys->plan->tile == sys->tile &&
      sys->plan->precision == sys->precision)
    return PAWAN_OK;
  sys->plan.reset();
  return build_plan(sys->ctx, {sys}, sys->precision, sys->tile, sys->plan);
}

// Reference layout (per wake [x | alpha]) -> device union layout [x | alpha].
int state_to_device(pawan_system *sys, const double *state) {
  pawan_ctx *ctx = sys->ctx;
  const size_t N = sys->n;
  for (size_t w = 0; w < sys->counts.size(); ++w) {
    const size_t o = sys->offsets[w], c = sys->counts[w];
    const double *src = state + 6 * o;
    PAWAN_CUDA(ctx, cudaMemcpyAsync(sys->X.p + 3 * o, src, 3 * c * sizeof(double),
                                    cudaMemcpyHostToDevice, ctx->stream));
    PAWAN_CUDA(ctx, cudaMemcpyAsync(sys->X.p + 3 * N + 3 * o, src + 3 * c, 3 * c * sizeof(double),
                                    cudaMemcpyHostToDevice, ctx->stream));
  }
  return PAWAN_OK;
}

// Device union layout -> reference layout; synchronous.
int state_from_device(pawan_system *sys, const double *dev_union, double *state) {
  pawan_ctx *ctx = sys->ctx;
  const size_t N = sys->n;
  for (size_t w = 0; w < sys->counts.size(); ++w) {
    const size_t o = sys->offsets[w], c = sys->counts[w];
    double *dst = state + 6 * o;
    PAWAN_CUDA(ctx, cudaMemcpyAsync(dst, dev_union + 3 * o, 3 * c * sizeof(double),
                                    cudaMemcpyDeviceToHost, ctx->stream));
    PAWAN_CUDA(ctx, cudaMemcpyAsync(dst + 3 * c, dev_union + 3 * N + 3 * o, 3 * c * sizeof(double),
                                    cudaMemcpyDeviceToHost, ctx->stream));
  }
  PAWAN_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return PAWAN_OK;
}

}  // namespace pawan

size_t pawan_system::device_bytes() const {
  return X.bytes() + Xs.bytes() + K1.bytes() + K2.bytes() + R.bytes() + rad.bytes() +
         vol.bytes() + wake_id.bytes() + pos32.bytes() + vor32.bytes() + poslo.bytes() +
         vorlo.bytes() + pos64.bytes() +
         vor64.bytes() + diag_scratch.bytes() + diag_out.bytes() + Xc.bytes() + field.bytes() +
         (plan ? plan->partial.bytes() : 0);
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
  if (cudaMalloc(&ctx->d_counter, sizeof(int)) != cudaSuccess) {
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
                    t->blocks_per_sm, t->packed};
  c.items_per_slot = t->items_per_slot;
  if (t->items_per_slot < 1 || t->targets_per_thread < 1 || t->blocks_per_sm < 0 || t->packed < 0 ||
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
  tiling->items_per_slot = sys->tile.items_per_slot;
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

// Host engine of the pawan B200 library: tile choices, execution plans over
// one or many systems (the reference's __interaction with its wakes), pair and
// stage launches, RK4 driving with CUDA graphs, autotuning internals, and a
// system's device buffers and state conversions.  The C ABI over it is in
// abi.cpp.
#include "runtime.h"

#include <nvtx3/nvToolsExt.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdint>
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
    // the packed unroll-4 shapes again with a separate near pass, scalar (1) or
    // packed (2) (ahead where near tile pairs are many: ragged batches of small
    // rings, scrambled states)
    for (int split : {1, 2})
      for (int tb : {128, 256})
        for (int pk : {1, 2}) {
          TileChoice t;
          t.pc = PairConfig{tb, 1, 4, 1, 0, pk, split};
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

bool tile_supported(int precision, const PairConfig &pc, int kernel) {
  if (precision == PAWAN_PREC_F32) return pairs_f32_supported(pc, kernel);
  if (precision == PAWAN_PREC_F64) return pairs_f64_supported(pc, kernel);
  return pairs_plain_supported(pc, kernel);
}

static_assert(PAWAN_KERNEL_HIGHORDER == KERNEL_HIGHORDER && PAWAN_KERNEL_GAUSSIAN == KERNEL_GAUSSIAN,
              "public and device smoothing-kernel codes agree");

static size_t shard_first(const pawan_system *y) { return (size_t)y->shard.rank * y->shard.size; }

static size_t shard_count(const pawan_system *y) {
  const size_t f = shard_first(y);
  return f >= y->n ? 0 : std::min(y->shard.size, y->n - f);
}

// Work decomposition.  Target tiles of tb/p particles; sources in chunks of
// whole tb-tiles sized so that the launch holds about `items_per_slot` items
// per resident block (or of `fixed_chunk_sources` when > 0, which makes a
// system's arithmetic independent of the other systems in the plan).  The
// systems with the largest items come first, so the dynamic counter hands out
// the long items early (longest-processing-time order), and within a system a
// target tile's chunks are consecutive.
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
  // per system: partial slots [target tiles][chunks][6][TPB] (none with one
  // chunk), rates [6][n], one counter per target tile
  if (TPB % 8 != 0) return fail(ctx, PAWAN_ERR_INVALID, "targets per block must be a multiple of 8");
  size_t partial_total = 0, box_total = 0, rates_total = 0, count_total = 0, slot_total = 0;
  std::vector<size_t> partial_off(systems.size()), box_off(systems.size()), slot_off(systems.size());
  std::vector<size_t> rates_off(systems.size()), count_off(systems.size());
  std::vector<double> sys_cost(systems.size(), 0.0);
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
    const size_t target_tiles = ((size_t)n + TPB - 1) / TPB;
    partial_off[s] = partial_total;
    if (nch > 1) partial_total += target_tiles * (size_t)nch * 6 * (size_t)TPB;
    slot_off[s] = slot_total;  // item slots (target tile, chunk), for the near pass
    slot_total += target_tiles * (size_t)nch;
    rates_off[s] = rates_total;
    rates_total += 6 * (size_t)n;
    count_off[s] = count_total;
    count_total += target_tiles;
    box_off[s] = box_total;
    box_total += 2 * (size_t)src_tiles;
    // targets: all particles, or this process's block of a sharded system
    // (block starts are multiples of kShardAlign, so of every TPB and TB)
    const pawan_system *y = systems[s];
    const int t_lo = y->shard.active ? (int)shard_first(y) : 0;
    const int t_hi = y->shard.active ? t_lo + (int)shard_count(y) : n;
    // target-major: a target tile's chunks are consecutive, so they run at
    // about the same time and the block completing the tile finds their
    // partial slots still in L2
    for (int t0 = t_lo; t0 < t_hi; t0 += TPB) {
      const int nt = std::min(TPB, t_hi - t0);
      for (int c = 0; c < nch; ++c) {
        const int s0 = c * tiles_per_chunk * TB;
        const int s1 = std::min(n, (c + 1) * tiles_per_chunk * TB);
        const double cost = (double)nt * (double)(s1 - s0);
        sys_cost[s] = std::max(sys_cost[s], cost);
        items.push_back({WorkItem{(int)s, t0, c, s0, s1}, cost});
      }
    }
  }
  // Systems whose items are largest go first (longest-processing-time order
  // across the systems of a batch); each system's items keep their order.
  std::stable_sort(items.begin(), items.end(), [&](const ItemCost &a, const ItemCost &b) {
    return sys_cost[a.w.seg] > sys_cost[b.w.seg];
  });
  if (items.size() > (size_t)INT32_MAX) return fail(ctx, PAWAN_ERR_INVALID, "too many work items");
  p->n_items = (int)items.size();

  if (ordered_alloc) {
    p->partial.ordered_on(ctx->stream);
    p->rates.ordered_on(ctx->stream);
    p->tile_count.ordered_on(ctx->stream);
    p->near_partial.ordered_on(ctx->stream);
    p->near_flag.ordered_on(ctx->stream);
    p->boxes.ordered_on(ctx->stream);
    p->items.ordered_on(ctx->stream);
    p->segs.ordered_on(ctx->stream);
    p->stage_items.ordered_on(ctx->stream);
    p->shard_items.ordered_on(ctx->stream);
    p->stage_descs.ordered_on(ctx->stream);
  }
  PAWAN_CUDA(ctx, p->partial.alloc(partial_total));
  // the pair kernels discard the slots' L2 lines after summing them: every
  // slot must start on a 128-byte line (slot sizes are multiples of 128 bytes)
  if (reinterpret_cast<uintptr_t>(p->partial.p) % 128 != 0)
    return fail(ctx, PAWAN_ERR_CUDA, "partial-sum buffer not 128-byte aligned");
  PAWAN_CUDA(ctx, p->rates.alloc(rates_total));
  PAWAN_CUDA(ctx, p->tile_count.alloc(count_total));
  PAWAN_CUDA(ctx, cudaMemsetAsync(p->tile_count.p, 0, p->tile_count.bytes(), ctx->stream));
  if (tile.pc.split > 0) {
    PAWAN_CUDA(ctx, p->near_partial.alloc(slot_total * 6 * (size_t)TPB));
    PAWAN_CUDA(ctx, p->near_flag.alloc(slot_total));
  }
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
    d.partial = p->nchunks[s] > 1 ? p->partial.p + partial_off[s] : nullptr;
    d.rates = p->rates.p + rates_off[s];
    d.tile_count = p->tile_count.p + count_off[s];
    d.near_partial = tile.pc.split > 0 ? p->near_partial.p + slot_off[s] * 6 * (size_t)TPB : nullptr;
    d.near_flag = tile.pc.split > 0 ? p->near_flag.p + slot_off[s] : nullptr;
    d.n = (int)y->n;
    d.nchunks = p->nchunks[s];
    d.nu = y->nu;
    d.near2 = (float)(y->r_near * y->r_near);
    StageDesc &g = p->stage_host[s];
    g.rates = d.rates;
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
  PAWAN_CUDA(ctx, cudaMemsetAsync(ctx->d_counter, 0, 2 * sizeof(int), ctx->stream));
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

// Algorithmic HBM bytes of one stage launch: per particle the rates (48
// bytes: the pair kernel's summed chunks, or the gathered rates of a sharded
// system), the FP64 state vectors the mode reads and writes, radius and
// volume, and the 128 bytes of packed FP32 / FP64 tile data; 32 bytes of
// bounding box per tile.  An RK4 stage is 336-384 bytes per particle.
static double stage_bytes(const Plan &p, int mode) {
  double total = 0.0;
  for (size_t s = 0; s < p.systems.size(); ++s) {
    const pawan_system *y = p.systems[s];
    const double n = (double)y->n;
    const double rates = 48.0;
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
  // One right-hand side as an RK4 stage runs it: the pair launch and the
  // reduction of its chunk partials (STAGE_RATES writes only the rates
  // buffer), so that finer chunking pays for the partials it adds.
  auto rhs = [&](Plan &p) -> int {
    PAWAN_TRY(launch_pairs(ctx, p, false));
    return launch_stage_mode(ctx, p, STAGE_RATES);
  };
  auto time_tile = [&](const TileChoice &t, double *ms) -> int {
    std::unique_ptr<Plan> p;
    PAWAN_TRY(build_plan(ctx, systems, precision, t, p));
    PAWAN_TRY(rhs(*p));  // warm-up
    PAWAN_CUDA(ctx, cudaEventRecord(e0, ctx->stream));
    const int reps = 2;
    for (int r = 0; r < reps; ++r) PAWAN_TRY(rhs(*p));
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
    for (int ips : kTuneItemsPerSlot) {
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

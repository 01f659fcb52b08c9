// Internal host-side runtime of the pawan B200 library: context, systems,
// execution plans.  Shared by the C-ABI (runtime.cpp) and the serving engine
// (serve.cpp); not part of the public interface.
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <map>
#include <memory>
#include <string>
#include <tuple>
#include <vector>

#include "../../include/pawan_b200.h"
#include "kernels.h"

namespace pawan {

// A device allocation that frees itself.  By default cudaMalloc / cudaFree
// (the free waits for the device); after ordered_on(stream) the buffer is
// taken from and returned to the device's memory pool in the order of
// `stream` (cudaMallocAsync / cudaFreeAsync, no device-wide synchronisation),
// so every use must be ordered on that stream before the buffer is released.
template <class T>
struct DBuf {
  T *p = nullptr;
  size_t n = 0;
  cudaStream_t stream = nullptr;
  bool ordered = false;
  DBuf() = default;
  DBuf(const DBuf &) = delete;
  DBuf &operator=(const DBuf &) = delete;
  ~DBuf() { reset(); }
  void ordered_on(cudaStream_t s) {
    stream = s;
    ordered = true;
  }
  cudaError_t alloc(size_t count) {
    reset();
    if (count == 0) return cudaSuccess;
    cudaError_t e = ordered ? cudaMallocAsync(reinterpret_cast<void **>(&p), count * sizeof(T), stream)
                            : cudaMalloc(reinterpret_cast<void **>(&p), count * sizeof(T));
    if (e != cudaSuccess) {
      p = nullptr;
      return e;
    }
    n = count;
    return cudaSuccess;
  }
  void reset() {
    if (p) {
      if (ordered)
        cudaFreeAsync(p, stream);
      else
        cudaFree(p);
    }
    p = nullptr;
    n = 0;
  }
  size_t bytes() const { return n * sizeof(T); }
};

// Tiling of the pair kernel plus how finely sources are chunked.
struct TileChoice {
  PairConfig pc{128, 1, 4};
  int items_per_slot = 16;
  bool operator==(const TileChoice &o) const {
    return pc.tb == o.pc.tb && pc.p == o.pc.p && pc.r == o.pc.r && pc.unroll == o.pc.unroll &&
           pc.minb == o.pc.minb && pc.packed == o.pc.packed && pc.split == o.pc.split &&
           items_per_slot == o.items_per_slot;
  }
};

TileChoice default_tile(int precision);
// Tilings the autotuner times (at the default chunking), and the chunkings
// (work items per resident block) it then times for the fastest of them.
std::vector<TileChoice> tile_candidates(int precision, int kernel);
const std::vector<int> kTuneItemsPerSlot = {4, 8, 32, 64, 128};

struct Plan;

}  // namespace pawan

struct pawan_ctx {
  int device = 0;
  int sm_count = 0;
  int cc_major = 0, cc_minor = 0;
  size_t total_mem = 0;
  cudaStream_t stream = nullptr;
  std::string err;
  std::atomic<unsigned long long> launches{0};
  int *d_counter = nullptr;  // work-item counter of the persistent pair kernels
  // profiling of pair launches
  bool profile = false;
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> pending;
  std::vector<cudaEvent_t> event_pool;
  double pair_ms = 0.0;
  unsigned long long pair_launches = 0;
  double pair_interactions = 0.0;
  // the same for the per-particle stage kernel, with its algorithmic bytes
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> stage_pending;
  double stage_ms = 0.0;
  unsigned long long stage_launches = 0;
  double stage_bytes = 0.0;
  cudaEvent_t marks[16] = {};
  void *flush_buf = nullptr;
  size_t flush_bytes = 0;
  // autotune results: (precision, diffusion, log2 sum n^2, log2 segments) -> tile
  std::map<std::tuple<int, int, int, int>, pawan::TileChoice> tune_cache;
};

struct pawan_system {
  pawan_ctx *ctx = nullptr;
  std::vector<size_t> counts;   // particles per wake
  std::vector<size_t> offsets;  // first particle of each wake
  size_t n = 0;
  double nu = 0.0;
  int precision = PAWAN_PREC_F32;
  int kernel = PAWAN_KERNEL_HIGHORDER;  // smoothing kernel (SmoothingKernel)
  bool has_particles = false;
  bool fixed_tile = false;
  pawan::TileChoice tile;
  pawan::DBuf<double> X, Xs, K1, K2, R, rad, vol, diag_scratch, diag_out, Xc;
  pawan::DBuf<double> field;  // vorticity field (N x 3), allocated on first use
  pawan::DBuf<int> wake_id;
  pawan::DBuf<float4> pos32, vor32, poslo, vorlo;
  pawan::DBuf<double4> pos64, vor64;
  std::unique_ptr<pawan::Plan> plan;  // single-system plan for `tile`
  // origin of the FP32 positions and near-tile radius, fixed by set_particles
  double ox = 0, oy = 0, oz = 0;
  double r_near = 0;
  unsigned long long geometry_version = 0;  // bumps when origin / r_near change
  unsigned long long pack_version = 0;      // bumps whenever the packed arrays change
  // device buffers from the memory pool in the order of ctx->stream (systems
  // owned by the serving engine); the context must outlive the system
  bool ordered_alloc = false;
  // target sharding over processes (pawan_system_set_shard): this process
  // computes the rates of particles [rank * size, min(n, (rank + 1) * size))
  struct Shard {
    bool active = false;
    int rank = 0, world = 1;
    size_t size = 0;         // particles per process block
    double *send = nullptr;  // device, 6 * size: this process's block
    double *recv = nullptr;  // device, 6 * size * world: every block, gathered
  } shard;
  size_t device_bytes() const;
};

namespace pawan {

// Everything one persistent pair launch plus its stage launch need for a set
// of systems.  Owns the partial buffers and the device-side tables.
struct Plan {
  std::vector<pawan_system *> systems;
  std::vector<double> nus;  // nu of each system when the plan was built
  std::vector<unsigned long long> geometry_versions;
  std::vector<unsigned long long> box_versions;  // pack_version the boxes were made at
  int precision = PAWAN_PREC_F32;
  int kernel = PAWAN_KERNEL_HIGHORDER;
  TileChoice tile;
  bool diffusion = false;
  int grid = 0;
  int n_items = 0;
  std::vector<double> item_costs;  // interactions of each work item, in launch order
  int n_stage_blocks = 0;
  double interactions = 0.0;  // sum n^2
  std::vector<int> nchunks;
  DBuf<double> partial;   // per system [target tiles][chunks][6][tpb] (chunks > 1)
  DBuf<double> rates;     // per system [6][n]: the summed chunks
  DBuf<int> tile_count;   // per system and target tile; 0 between launches
  DBuf<double> near_partial;        // split tilings: near sums per item slot (as partial)
  DBuf<unsigned char> near_flag;    // split tilings: per item slot, whether it had near tiles
  DBuf<float4> boxes;
  DBuf<WorkItem> items;
  DBuf<SegDesc> segs;
  DBuf<StageItem> stage_items;
  DBuf<StageItem> shard_items;  // the stage blocks of this process's targets
  int n_shard_blocks = 0;
  DBuf<StageDesc> stage_descs;
  std::vector<StageDesc> stage_host;
  std::vector<double> dts;  // dt in the device stage table
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t graph_exec = nullptr;
  ~Plan();
  bool stale() const;
};

// Status helpers: record the message on the context and return the code.
int fail(pawan_ctx *ctx, int code, const std::string &msg);
int cuda_fail(pawan_ctx *ctx, cudaError_t e, const char *where);

// Return the status of a failed CUDA call (recorded on ctx) or of a failed
// library call, from the enclosing function.
#define PAWAN_CUDA(ctx, expr)                                           \
  do {                                                                  \
    cudaError_t e_ = (expr);                                            \
    if (e_ != cudaSuccess) return ::pawan::cuda_fail((ctx), e_, #expr); \
  } while (0)

#define PAWAN_TRY(expr)            \
  do {                             \
    int s_ = (expr);               \
    if (s_ != PAWAN_OK) return s_; \
  } while (0)

// Process blocks of a sharded system start at multiples of kShardAlign
// particles: whole stage blocks and whole target tiles of every tiling.
constexpr size_t kShardAlign = 512;

// Whether a precision's kernels are compiled for a tiling and smoothing kernel.
bool tile_supported(int precision, const PairConfig &pc, int kernel);

int build_plan(pawan_ctx *ctx, const std::vector<pawan_system *> &systems, int precision,
               const TileChoice &tile, std::unique_ptr<Plan> &out, int fixed_chunk_sources = 0,
               bool ordered_alloc = false);
int set_plan_dt(pawan_ctx *ctx, Plan &p, const double *dt, double dt0);
int launch_pairs(pawan_ctx *ctx, Plan &p, bool allow_events = true);
// The pair kernel over the plan's work items [first, first + count) only (the
// items write disjoint partial slots, so a stage may be split over launches).
int launch_pairs_range(pawan_ctx *ctx, Plan &p, int first, int count, bool allow_events = true);
int launch_stage_mode(pawan_ctx *ctx, Plan &p, int mode);
int rk4_steps(pawan_ctx *ctx, Plan &p, size_t nsteps, bool use_graph);
int autotune_plan(pawan_ctx *ctx, const std::vector<pawan_system *> &systems, int precision,
                  TileChoice *best);
int system_alloc(pawan_system *sys);
// A system without device-side plan (the serving engine plans over many):
// creation with buffers from the memory pool (ordered on ctx->stream), and
// the particle upload (validation, geometry, copies; packing is left to the
// next plan built over the system).  Neither waits for the device.
int system_create_ordered(pawan_ctx *ctx, size_t n_wakes, const size_t *num_particles, double nu,
                          int precision, pawan_system **out);
int system_upload(pawan_system *sys, const double *position, const double *vorticity,
                  const double *radius, const double *volume);
int system_ensure_plan(pawan_system *sys);
int state_to_device(pawan_system *sys, const double *state);
int state_from_device(pawan_system *sys, const double *dev_union, double *state);

}  // namespace pawan

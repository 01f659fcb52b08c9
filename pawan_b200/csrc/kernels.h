// Host-side launchers of the pawan B200 kernels (implemented in the .cu files).
#pragma once

#include <cuda_runtime.h>

#include "device.cuh"

namespace pawan {

// Tiling of the all-pairs kernels: `tb` threads per block (= sources per
// shared-memory tile), `p` threads per target, `r` targets per thread
// (targets per block = tb / p * r), `unroll` = unroll depth of the source loop,
// `minb` = blocks per SM the registers are bounded for (0: the default),
// `packed` = far tiles computed two sources per FP32x2 instruction (1: 1/rho^2
// from the MUFU reciprocal on uniform-radius tiles, 2: from rsqrt squared;
// 0: one source per instruction).
// `split` = 1: near tile pairs are computed by a pass of their own before the
// far pass (which then skips them), each kernel with its own register
// allocation, the near pass forming alpha_i x alpha_j by the projection form
// (19 operations instead of the one pass's 27); `split` = 2: the same with the
// near pass two sources per FP32x2 instruction.
struct PairConfig {
  int tb;
  int p;
  int unroll;
  int r = 1;
  int minb = 0;
  int packed = 0;
  int split = 0;
};

inline int targets_per_block(const PairConfig &c) { return c.tb / c.p * c.r; }

// `kernel` below is a SmoothingKernel (device.cuh).

// FP32 pair math, FP64 accumulation of per-tile partial sums.
bool pairs_f32_supported(const PairConfig &c, int kernel);
cudaError_t pairs_f32_occupancy(const PairConfig &c, bool diffusion, int kernel, int *blocks_per_sm);
// next_item: two counters (the far pass's and the near pass's), zero at launch.
cudaError_t launch_pairs_f32(const PairConfig &c, bool diffusion, int kernel, int grid,
                             const WorkItem *items, int n_items, const SegDesc *segs,
                             int *next_item, cudaStream_t s);

// FP64 with the same algebra as the FP32 kernel ("tuned FP64").
bool pairs_f64_supported(const PairConfig &c, int kernel);
cudaError_t pairs_f64_occupancy(const PairConfig &c, bool diffusion, int kernel, int *blocks_per_sm);
cudaError_t launch_pairs_f64(const PairConfig &c, bool diffusion, int kernel, int grid,
                             const WorkItem *items, int n_items, const SegDesc *segs,
                             int *next_item, cudaStream_t s);

// FP64, the reference's formula term by term (pow, divisions): the plain
// FP64 comparator.
bool pairs_plain_supported(const PairConfig &c, int kernel);
cudaError_t pairs_plain_occupancy(const PairConfig &c, int kernel, int *blocks_per_sm);
cudaError_t launch_pairs_plain(const PairConfig &c, int kernel, int grid, const WorkItem *items,
                               int n_items, const SegDesc *segs, int *next_item, cudaStream_t s);

// Per-particle stage kernel (RK4 stage update from the summed rates, pack).
cudaError_t launch_stage(int mode, int n_blocks, const StageItem *items, const StageDesc *descs,
                         cudaStream_t s);

// Diagnostics of one system.  `scratch` holds at least diag_scratch_doubles(n)
// doubles; out[0..10] = total vorticity (3), linear impulse (3), angular
// impulse (3), enstrophy, helicity; out[11] = kinetic energy.
size_t diag_scratch_doubles(int n);
cudaError_t launch_diagnostics(int n, int kernel, const double4 *pos64, const double4 *vor64,
                               const int *wake_id, double *scratch, double *out, bool quadratic,
                               cudaStream_t s);

// Vorticity field (FP64) of one system: field[3i..3i+2] = sum_j Z_ij alpha_j.
cudaError_t launch_influence(int n, int kernel, const double4 *pos64, const double4 *vor64,
                             double *field, cudaStream_t s);
// Columns per block of the columns kernel; a launch covers at most
// 65,535 x kInfluenceColumnGroup columns (the grid's y extent).
constexpr int kInfluenceColumnGroup = 8;
// The same for ncols strength vectors over one set of positions and radii:
// cols and field are ncols blocks of N x 3 doubles; column c of field is
// bit-identical to launch_influence with vor64 = column c of cols.
cudaError_t launch_influence_columns(int n, int ncols, int kernel, const double4 *pos64,
                                     const double *cols, double *field, cudaStream_t s);

// Throughput probes: FP32 FFMA and FP64 DFMA chains.  flops = launched FMAs * 2.
cudaError_t launch_ffma_peak(int blocks, int threads, int iters, float *sink, cudaStream_t s);
cudaError_t launch_dfma_peak(int blocks, int threads, int iters, double *sink, cudaStream_t s);
// FMAs launched: as above (kPeakChains FMAs per thread and repetition, in pairs).
cudaError_t launch_ffma2_peak(int blocks, int threads, int iters, float *sink, cudaStream_t s);
constexpr int kPeakChains = 8;

}  // namespace pawan

// Shared device-side types of the pawan B200 library.
//
// HBM layout of one system (the reference's __interaction over its wakes,
// src/interaction/interaction.h:21-235), all particles of all wakes in wake
// order, N in total:
//   X      double[6N]  state [x (N x 3) | alpha (N x 3)]  (the reference keeps
//                      this per wake, wake.cpp:87-120; the host API converts)
//   rad    double[N]   smoothing radius s          (wake.h:39)
//   vol    double[N]   particle volume v           (wake.h:40)
//   pos32  float4[N]   (x-c, y-c, z-c, s^2/2)  packed FP32 tile data: position
//                      relative to the system's origin c, rounded to FP32 (hi)
//   poslo  float4[N]   (x-c - hi, ..., 0)  what the FP32 rounding dropped (lo)
//   vor32  float4[N]   (ax, ay, az, v)    strength (hi) and volume
//   vorlo  float4[N]   (ax - hi, ..., 0)  strength (lo)
//                      -> 64 bytes per particle; hi + lo carries ~48 bits
//   pos64  double4[N]  (x, y, z, s)       packed FP64 data (FP64 kernels,
//   vor64  double4[N]  (ax, ay, az, v)     diagnostics)
//   boxes  float4[2 per source tile]  bounding box of each tile's hi positions
//   partial double[T][C][6][tpb]  per (target tile, source chunk) sums (u,
//                      dalpha) of the pair kernel: T target tiles of tpb
//                      particles, C source chunks
//   rates  double[6][N]  the chunks summed in chunk order (u, dalpha), written
//                      by the pair kernel's block that completes a target tile
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace pawan {

// One solve as the pair kernels see it.
struct SegDesc {
  const float4 *pos32;
  const float4 *vor32;
  const float4 *poslo;
  const float4 *vorlo;
  const double4 *pos64;
  const double4 *vor64;
  const float4 *boxes;  // [2 * ceil(n / tile)] (lo, hi) per source tile
  double *partial;      // [ceil(n / tpb)][nchunks][6][tpb] (unused when nchunks == 1)
  double *rates;        // [6][n]
  int *tile_count;      // [ceil(n / tpb)] items of the tile done in this launch (0 between launches)
  // with a separate near pass (split tilings): each item's sums over its near
  // tile pairs, [ceil(n / tpb)][nchunks][6][tpb], and whether it had any
  double *near_partial;
  unsigned char *near_flag;  // [ceil(n / tpb)][nchunks]
  int n;
  int nchunks;
  double nu;
  float near2;          // squared box distance below which a tile pair is "near"
};

// One unit of pair work: targets [t0, t0 + targets_per_block) of segment `seg`
// against its sources [s0, s1), written to partial chunk `chunk`.
struct WorkItem {
  int seg;
  int t0;
  int chunk;
  int s0;
  int s1;
};

// One block of the per-particle stage kernel: particles [l0, l0 + 256) of
// segment `seg`.
struct StageItem {
  int seg;
  int l0;
};

// What the stage kernel needs of one segment.
struct StageDesc {
  const double *rates;  // [6][n], the pair kernel's summed chunks
  int n;
  double *X;   // state x
  double *Xs;  // stage state x_s
  double *K1;  // k1
  double *K2;  // k2, then k2 + k3
  double *R;   // rates of a plain solve
  const double *rad;
  const double *vol;
  float4 *pos32;
  float4 *vor32;
  float4 *poslo;
  float4 *vorlo;
  double4 *pos64;
  double4 *vor64;
  float4 *boxes;     // per box_tile particles: (lo, hi)
  int box_tile;      // 128 or 256 (divides kStageThreads)
  double ox, oy, oz; // origin the FP32 positions are relative to
  double dt;
  // Target sharding over processes (null / 0 otherwise).  Process blocks of
  // `shard` particles; this process's block starts at shard_first.  The
  // exchange layout is [process][6][shard]: STAGE_SHARD writes this
  // process's block to xchg_out, and when xchg_in is set (the all-gathered
  // blocks of every process) the other modes read their rates from it
  // instead of the partial chunks.
  double *xchg_out;
  const double *xchg_in;
  int shard;
  int shard_first;
};

enum StageMode : int {
  STAGE_RATES = 0,   // R = the rates
  STAGE_K1 = 1,      // k1 = r; x_s = k1*(dt/2) + x; pack x_s
  STAGE_K2 = 2,      // k2 = r; x_s = k2*(dt/2) + x; pack x_s
  STAGE_K3 = 3,      // k2 = k2 + r; x_s = r*dt + x; pack x_s
  STAGE_FINAL = 4,   // x = x + ((k1 + r)*(dt/6) + (k2+k3)*(dt/3)); pack x
  STAGE_EULER = 5,   // x = x + r*dt; pack x   (integration.cpp:37-45)
  STAGE_PACK = 6,    // pack x only
  STAGE_SHARD = 7,   // this process's block of rates -> xchg_out (no state change)
};

// Smoothing kernel of a system: the reference's high-order algebraic kernel
// (src/interaction/highorder.h, its default) or its Gaussian one
// (src/interaction/gaussian.h, selected there by #define GAUSSIAN).
enum SmoothingKernel : int {
  KERNEL_HIGHORDER = 0,
  KERNEL_GAUSSIAN = 1,
};

// 1/(4 pi) and friends.
constexpr double kInv4Pi = 0.07957747154594766788;
constexpr double kInvPi = 0.31830988618379067154;
constexpr double kPi = 3.14159265358979323846;
constexpr double kSqrt2OverPi = 0.79788456080286535588;  // sqrt(2/pi)
constexpr double kSqrtHalf = 0.70710678118654752440;     // 1/sqrt(2)

// Block sizes.  Source tiles (and so bounding boxes) are 128 or 256
// particles; stage blocks cover whole tiles.
constexpr int kStageThreads = 256;


#ifdef __CUDACC__
// ---- per-item partial sums and their in-launch reduction -------------------
//
// A work item (target tile x source chunk) of a segment with nchunks > 1
// stores its sums in its own slot, partial_slot(); when nchunks == 1 it
// writes the rates directly.  After storing, every thread of the block calls
// finish_item(): the item is counted for its target tile, and the block whose
// item completes the tile sums the tile's slots in chunk order
// (r = c0, r += c1, ...: the same order whichever block is last, so results
// do not depend on scheduling) into rates[6][n], drops the slots' L2 lines
// without writing them back to DRAM (discard.global.L2: they are never read
// again; the next launch writes them afresh), and re-arms the tile's counter
// to 0 for the next launch.  Slots are multiples of 128 bytes (tpb is a
// multiple of 8) and the partial buffer is 128-byte aligned, so no line is
// shared between tiles.
__device__ __forceinline__ double *partial_slot(const SegDesc &sg, int t0, int chunk, int tpb) {
  const size_t tile = (size_t)(t0 / tpb);
  return sg.partial + ((tile * (size_t)sg.nchunks + (size_t)chunk) * 6) * (size_t)tpb;
}

__device__ __forceinline__ void discard_l2_line(const void *p) {
  asm volatile("discard.global.L2 [%0], 128;" ::"l"(p) : "memory");
}

template <int NT>
__device__ __forceinline__ void finish_item(const SegDesc &sg, int t0, int tpb, int *s_flag) {
  __threadfence();  // this thread's slot stores, before the count below
  __syncthreads();
  const int tile = t0 / tpb;
  if (threadIdx.x == 0) *s_flag = (atomicAdd(sg.tile_count + tile, 1) == sg.nchunks - 1);
  __syncthreads();
  if (!*s_flag) return;  // block-uniform
  __threadfence();
  const double *base = sg.partial + (size_t)tile * (size_t)sg.nchunks * 6 * (size_t)tpb;
  const int nt = min(tpb, sg.n - t0);
  const size_t n = (size_t)sg.n;
  const size_t cstride = 6 * (size_t)tpb;
  for (int u = threadIdx.x; u < 6 * tpb; u += NT) {
    const int k = u / tpb, q = u - k * tpb;
    if (q >= nt) continue;
    const double *p = base + (size_t)k * tpb + q;
    double r = __ldcg(p);
    int c = 1;
    // four chunks' loads in flight, summed in chunk order
    for (; c + 4 <= sg.nchunks; c += 4) {
      const double a = __ldcg(p + c * cstride), b = __ldcg(p + (c + 1) * cstride);
      const double d = __ldcg(p + (c + 2) * cstride), e = __ldcg(p + (c + 3) * cstride);
      r = __dadd_rn(__dadd_rn(__dadd_rn(__dadd_rn(r, a), b), d), e);
    }
    for (; c < sg.nchunks; ++c) r = __dadd_rn(r, __ldcg(p + c * cstride));
    sg.rates[(size_t)k * n + (size_t)t0 + q] = r;
  }
  __syncthreads();  // every read of the slots is done
  const size_t lines = (size_t)sg.nchunks * cstride * sizeof(double) / 128;
  for (size_t l = threadIdx.x; l < lines; l += NT)
    discard_l2_line(reinterpret_cast<const char *>(base) + 128 * l);
  if (threadIdx.x == 0) sg.tile_count[tile] = 0;
}

// Where an item's six sums go: its slot (row stride tpb) or, for a segment of
// one chunk, the rates themselves (row stride n); index by target - t0.
struct ItemOut {
  double *base;
  size_t stride;
};

__device__ __forceinline__ ItemOut item_out(const SegDesc &sg, int t0, int chunk, int tpb) {
  if (sg.nchunks == 1) return ItemOut{sg.rates + t0, (size_t)sg.n};
  return ItemOut{partial_slot(sg, t0, chunk, tpb), (size_t)tpb};
}
#endif  // __CUDACC__

}  // namespace pawan

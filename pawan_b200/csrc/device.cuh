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
//   partial double[C][6][N]  per source-chunk sums (u, dalpha) of the pair
//                      kernel, reduced in fixed chunk order by the stage kernel
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
  double *partial;      // [nchunks][6][n]
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
  const double *partial;
  int nchunks;
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
  STAGE_RATES = 0,   // R = sum of partials
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

}  // namespace pawan

// Per-particle stage kernel: reads the rates (u | dalpha) the pair kernel
// summed, applies the RK4 stage update in FP64 with the reference's operation
// order, packs the new state into the FP32 hi/lo and FP64 tile arrays the next
// pair launch reads, and writes the bounding box of each source tile.  One
// thread per particle, HBM-bound.
//
// Reference: __rk4::step (src/integration/rk4.cpp:12-76):
//   x1 = k1*(0.5 dt) + x        (:29-31)      STAGE_K1
//   x2 = k2*(0.5 dt) + x        (:39-41)      STAGE_K2
//   x3 = k3*dt + x              (:49-51)      STAGE_K3 (also forms k2 + k3, :61)
//   x += (k1 + k4)*(dt/6) + (k2 + k3)*(dt/3)   (:58-66)   STAGE_FINAL
// and __integration::step (src/integration/integration.cpp:37-45): x += r*dt.
// For a system sharded over processes, STAGE_SHARD writes this process's
// block of reduced rates to the exchange buffer, and after the all-gather the
// stage modes read every particle's rates from the gathered buffer.
// Products and sums use __dmul_rn/__dadd_rn so no multiply-add is contracted,
// keeping the update bit-identical to the reference's for equal rates.
#include "device.cuh"
#include "kernels.h"

namespace pawan {
namespace {

// Blocks per SM the register budget is held to: a segment of 131,072
// particles is 512 blocks of 256, one wave at four blocks per SM on 148 SMs.
// The descriptor is read through a reference (uniform, L1-cached) rather than
// copied, which is what frees the registers.
constexpr int kStageMinBlocks = 4;

// Packs one particle: FP32 hi/lo pairs of the position relative to the
// system's origin and of the strength, plus the FP64 copies.  Returns the hi
// position and h = s^2/2 for the tile's bounding box.
__device__ __forceinline__ float4 pack(const StageDesc &d, int l, const double x[6]) {
  const double s = d.rad[l];
  const double v = d.vol[l];
  const double rx = x[0] - d.ox, ry = x[1] - d.oy, rz = x[2] - d.oz;
  const float hx = (float)rx, hy = (float)ry, hz = (float)rz;
  const float ax = (float)x[3], ay = (float)x[4], az = (float)x[5];
  const float hw = (float)(0.5 * s * s);
  d.pos32[l] = make_float4(hx, hy, hz, hw);
  d.poslo[l] = make_float4((float)(rx - (double)hx), (float)(ry - (double)hy),
                           (float)(rz - (double)hz), 0.f);
  d.vor32[l] = make_float4(ax, ay, az, (float)v);
  d.vorlo[l] = make_float4((float)(x[3] - (double)ax), (float)(x[4] - (double)ay),
                           (float)(x[5] - (double)az), 0.f);
  d.pos64[l] = make_double4(x[0], x[1], x[2], s);
  d.vor64[l] = make_double4(x[3], x[4], x[5], v);
  return make_float4(hx, hy, hz, hw);
}

// Bounding boxes of the block's tiles (box_tile particles each, aligned to
// the segment); particles beyond n contribute nothing.  The box's w components
// carry the tile's smallest (lo) and largest (hi) h = s^2/2, so the pair
// kernel can tell tile pairs of one smoothing radius.  Each warp reduces its
// 32 particles by shuffles, then one thread per tile combines the tile's
// warps (4 or 8) from shared memory: one barrier.
__device__ __forceinline__ void tile_boxes(const StageDesc &d, int l0, float4 p, bool has) {
  constexpr int kWarps = kStageThreads / 32;
  __shared__ float wv[8][kWarps];
  float v[8] = {has ? p.x : INFINITY,  has ? p.y : INFINITY,  has ? p.z : INFINITY,
                has ? p.w : INFINITY,  has ? p.x : -INFINITY, has ? p.y : -INFINITY,
                has ? p.z : -INFINITY, has ? p.w : -INFINITY};
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      v[k] = fminf(v[k], __shfl_xor_sync(0xffffffffu, v[k], o));
      v[4 + k] = fmaxf(v[4 + k], __shfl_xor_sync(0xffffffffu, v[4 + k], o));
    }
  }
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  if (lane == 0) {
#pragma unroll
    for (int k = 0; k < 8; ++k) wv[k][warp] = v[k];
  }
  __syncthreads();
  const int wpt = d.box_tile / 32;
  if (t < kStageThreads / d.box_tile && l0 + t * d.box_tile < d.n) {
    float lo[4], hi[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      lo[k] = wv[k][t * wpt];
      hi[k] = wv[4 + k][t * wpt];
    }
    for (int w = 1; w < wpt; ++w) {
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        lo[k] = fminf(lo[k], wv[k][t * wpt + w]);
        hi[k] = fmaxf(hi[k], wv[4 + k][t * wpt + w]);
      }
    }
    const int b = (l0 + t * d.box_tile) / d.box_tile;
    d.boxes[2 * b] = make_float4(lo[0], lo[1], lo[2], lo[3]);
    d.boxes[2 * b + 1] = make_float4(hi[0], hi[1], hi[2], hi[3]);
  }
}

template <int MODE>
__global__ void __launch_bounds__(kStageThreads, kStageMinBlocks)
    stage_kernel(const StageItem *__restrict__ items, const StageDesc *__restrict__ descs) {
  const StageItem it = items[blockIdx.x];
  const StageDesc &d = descs[it.seg];
  const int l = it.l0 + threadIdx.x;
  const bool has = l < d.n;
  const size_t n = (size_t)d.n;
  size_t idx[6];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    idx[k] = 3 * (size_t)l + k;
    idx[3 + k] = 3 * n + 3 * (size_t)l + k;
  }

  double r[6] = {0, 0, 0, 0, 0, 0};
  if (MODE != STAGE_PACK && has) {
    if (MODE != STAGE_SHARD && d.xchg_in) {
      const size_t S = (size_t)d.shard;
      const double *g = d.xchg_in + ((size_t)l / S) * 6 * S + (size_t)l % S;
#pragma unroll
      for (int k = 0; k < 6; ++k) r[k] = g[(size_t)k * S];
    } else {
      // the pair kernel's rates (its chunks already summed); read once, so
      // streaming loads keep them from evicting the state from L2
#pragma unroll
      for (int k = 0; k < 6; ++k) r[k] = __ldcs(d.rates + (size_t)k * n + l);
    }
  }
  if (MODE == STAGE_SHARD) {
    if (has) {
      double *o = d.xchg_out + (l - d.shard_first);
#pragma unroll
      for (int k = 0; k < 6; ++k) o[(size_t)k * d.shard] = r[k];
    }
    return;
  }

  // Per-segment step size; the coefficients are formed as the reference forms
  // them (0.5*dt, dt/6., dt/3.), and device division is correctly rounded.
  const double dt = d.dt;
  const double half = 0.5 * dt;
  const double full = dt;
  const double sixth = dt / 6.;
  const double third = dt / 3.;

  if (MODE == STAGE_RATES) {
    if (has) {
#pragma unroll
      for (int k = 0; k < 6; ++k) d.R[idx[k]] = r[k];
    }
    return;  // uniform across the block: no pack, no boxes
  }
  double x[6] = {0, 0, 0, 0, 0, 0};
  if (has) {
    if (MODE == STAGE_K1 || MODE == STAGE_K2) {
      double *K = (MODE == STAGE_K1) ? d.K1 : d.K2;
#pragma unroll
      for (int k = 0; k < 6; ++k) {
        K[idx[k]] = r[k];
        x[k] = __dadd_rn(__dmul_rn(r[k], half), d.X[idx[k]]);
        d.Xs[idx[k]] = x[k];
      }
    } else if (MODE == STAGE_K3) {
#pragma unroll
      for (int k = 0; k < 6; ++k) {
        d.K2[idx[k]] = __dadd_rn(d.K2[idx[k]], r[k]);
        x[k] = __dadd_rn(__dmul_rn(r[k], full), d.X[idx[k]]);
        d.Xs[idx[k]] = x[k];
      }
    } else if (MODE == STAGE_FINAL) {
#pragma unroll
      for (int k = 0; k < 6; ++k) {
        const double a = __dmul_rn(__dadd_rn(d.K1[idx[k]], r[k]), sixth);
        const double b = __dmul_rn(d.K2[idx[k]], third);
        x[k] = __dadd_rn(d.X[idx[k]], __dadd_rn(a, b));
        d.X[idx[k]] = x[k];
      }
    } else if (MODE == STAGE_EULER) {
#pragma unroll
      for (int k = 0; k < 6; ++k) {
        x[k] = __dadd_rn(d.X[idx[k]], __dmul_rn(r[k], full));
        d.X[idx[k]] = x[k];
      }
    } else {  // STAGE_PACK
#pragma unroll
      for (int k = 0; k < 6; ++k) x[k] = d.X[idx[k]];
    }
  }
  float4 p = make_float4(0.f, 0.f, 0.f, 0.f);
  if (has) p = pack(d, l, x);
  tile_boxes(d, it.l0, p, has);
}

}  // namespace

cudaError_t launch_stage(int mode, int n_blocks, const StageItem *items, const StageDesc *descs,
                         cudaStream_t s) {
  if (n_blocks <= 0) return cudaSuccess;
  dim3 grid(n_blocks), block(kStageThreads);
  switch (mode) {
    case STAGE_RATES:
      stage_kernel<STAGE_RATES><<<grid, block, 0, s>>>(items, descs);
      break;
    case STAGE_K1:
      stage_kernel<STAGE_K1><<<grid, block, 0, s>>>(items, descs);
      break;
    case STAGE_K2:
      stage_kernel<STAGE_K2><<<grid, block, 0, s>>>(items, descs);
      break;
    case STAGE_K3:
      stage_kernel<STAGE_K3><<<grid, block, 0, s>>>(items, descs);
      break;
    case STAGE_FINAL:
      stage_kernel<STAGE_FINAL><<<grid, block, 0, s>>>(items, descs);
      break;
    case STAGE_EULER:
      stage_kernel<STAGE_EULER><<<grid, block, 0, s>>>(items, descs);
      break;
    case STAGE_PACK:
      stage_kernel<STAGE_PACK><<<grid, block, 0, s>>>(items, descs);
      break;
    case STAGE_SHARD:
      stage_kernel<STAGE_SHARD><<<grid, block, 0, s>>>(items, descs);
      break;
    default:
      return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

}  // namespace pawan

// All-pairs vortex-particle interaction, FP32 pair math with FP64
// accumulation of per-tile partial sums (the hot kernel).
//
// Reference: the pair physics of INTERACT (src/interaction/interaction_utils.h:363-407)
// with KERNEL (src/interaction/highorder.h:48-60), summed over all pairs of a
// system by __interaction::interact (src/interaction/interaction.cpp:95-108).
//
// Gather form.  For target i and source j != i, d = x_i - x_j,
// sigma^2 = (s_i^2 + s_j^2)/2 = h_i + h_j with h = s^2/2, rho^2 = |d|^2:
//   u_i     += q (alpha_j x d)
//   dalpha_i += q (alpha_i x alpha_j) + F [d.(alpha_i x alpha_j)] d
//             + (2 nu Z / sigma^2)(v_i alpha_j - v_j alpha_i)
// with (A = 1/(4 pi), w = (rho^2 + sigma^2)^(-1/2))
//   Z = 7.5 A sigma^12 w^15            ((15/8pi) sigma^-3 (rho_bar^2+1)^-7.5)
//   phi/rho_bar = A (rho^2 + 1.5 sigma^2) w^4 / rho
//   q = (phi/rho_bar - Z) sigma^2 / rho^2,   F = (Z - 3q) / rho^2.
// The kernel keeps per target, summed over sources:
//   U = sum qh (alpha_j x d)            (q = A qh)
//   Q = sum qh alpha_j                  -> alpha_i x (A Q) is the q-stretching term
//   G = sum fh [alpha_i.(alpha_j x d)] d   (F = 3A fh, and d.(a_i x a_j) = a_i.(a_j x d))
//   E = sum Dp alpha_j,  V = sum Dp v_j    (2 nu Z/sigma^2 = 15 nu A Dp)
// with Dp = sigma^10 w^15 = (sigma^2 w^2)^5 w^5 and Zc = sigma^12 w^15 = Dp sigma^2:
//   qh = (phi_hat - 7.5 Zc) sigma^2 / rho^2,  fh = (2.5 Zc - qh) / rho^2.
// Two MUFU rsqrt and 49 FP32 instructions per pair (45 without diffusion).
//
// Layout: one persistent block per SM slot takes work items (target tile x
// source chunk) from a counter; sources stream through a two-stage shared-memory
// ring, each thread loading one source (two float4) for the next tile while the
// block computes the current one.  Per tile the FP32 sums are added into FP64
// accumulators; the result of an item (u and dalpha, FP64) goes to the item's
// chunk of the partial buffer, which the stage kernel reduces in chunk order.
#include "device.cuh"
#include "kernels.h"

namespace pawan {
namespace {

struct Acc32 {
  float ux, uy, uz;
  float qx, qy, qz;
  float gx, gy, gz;
  float ex, ey, ez, ev;
};

// A source that contributes exactly zero: far away (all kernel factors
// underflow to 0, still finite) and with zero strength and volume.
__device__ __forceinline__ void load_source_f32(const SegDesc &sg, int j, int s1, float4 &p,
                                                float4 &v) {
  if (j < s1) {
    p = __ldg(sg.pos32 + j);
    v = __ldg(sg.vor32 + j);
  } else {
    p = make_float4(1e18f, 1e18f, 1e18f, 1.0f);
    v = make_float4(0.f, 0.f, 0.f, 0.f);
  }
}

template <bool DIFF, bool CHECK, int P, int NSRC, int U>
__device__ __forceinline__ void tile_f32(const float4 *__restrict__ sp,
                                         const float4 *__restrict__ sv, int g, int skip, float xi,
                                         float yi, float zi, float hi, float axi, float ayi,
                                         float azi, Acc32 &a) {
#pragma unroll U
  for (int k = 0; k < NSRC / P; ++k) {
    const int jj = g + P * k;
    const float4 p = sp[jj];
    const float4 s = sv[jj];
    const float dx = xi - p.x, dy = yi - p.y, dz = zi - p.z;
    const float r2 = fmaf(dz, dz, fmaf(dy, dy, dx * dx));
    const float sig2 = hi + p.w;
    const float w = rsqrtf(r2 + sig2);
    const float ri = rsqrtf(r2);
    const float ri2 = ri * ri;
    const float w2 = w * w;
    const float w4 = w2 * w2;
    const float uu = sig2 * w2;
    const float u2 = uu * uu;
    const float u4 = u2 * u2;
    const float u5 = u4 * uu;
    float dp = u5 * (w4 * w);
    const float zc = dp * sig2;
    const float ph = fmaf(1.5f, sig2, r2) * w4 * ri;
    float qh = fmaf(-7.5f, zc, ph) * sig2 * ri2;
    const float fh = fmaf(2.5f, zc, -qh) * ri2;
    const float cx = fmaf(s.y, dz, -s.z * dy);
    const float cy = fmaf(s.z, dx, -s.x * dz);
    const float cz = fmaf(s.x, dy, -s.y * dx);
    const float t = fmaf(azi, cz, fmaf(ayi, cy, axi * cx));
    float ft = fh * t;
    if (CHECK) {
      const bool self = (jj == skip);
      qh = self ? 0.f : qh;
      ft = self ? 0.f : ft;
      dp = self ? 0.f : dp;
    }
    a.ux = fmaf(qh, cx, a.ux);
    a.uy = fmaf(qh, cy, a.uy);
    a.uz = fmaf(qh, cz, a.uz);
    a.qx = fmaf(qh, s.x, a.qx);
    a.qy = fmaf(qh, s.y, a.qy);
    a.qz = fmaf(qh, s.z, a.qz);
    a.gx = fmaf(ft, dx, a.gx);
    a.gy = fmaf(ft, dy, a.gy);
    a.gz = fmaf(ft, dz, a.gz);
    if (DIFF) {
      a.ex = fmaf(dp, s.x, a.ex);
      a.ey = fmaf(dp, s.y, a.ey);
      a.ez = fmaf(dp, s.z, a.ez);
      a.ev = fmaf(dp, s.w, a.ev);
    }
  }
}

template <int TB, int P, int U, bool DIFF>
__global__ void __launch_bounds__(TB, (TB <= 128 ? 4 : 2))
    pairs_f32_kernel(const WorkItem *__restrict__ items, int n_items,
                     const SegDesc *__restrict__ segs, int *__restrict__ next_item) {
  constexpr int TPB = TB / P;
  __shared__ float4 sp[2][TB];
  __shared__ float4 sv[2][TB];
  __shared__ int s_item;
  const int tid = threadIdx.x;
  const int g = tid % P;
  const int lt = tid / P;

  for (;;) {
    if (tid == 0) s_item = atomicAdd(next_item, 1);
    __syncthreads();
    const int it = s_item;
    __syncthreads();
    if (it >= n_items) break;

    const WorkItem w = items[it];
    const SegDesc sg = segs[w.seg];
    const int i = w.t0 + lt;
    const bool valid = i < sg.n;
    float4 pi = make_float4(0.f, 0.f, 0.f, 1.f);
    float4 vi = make_float4(0.f, 0.f, 0.f, 0.f);
    if (valid) {
      pi = __ldg(sg.pos32 + i);
      vi = __ldg(sg.vor32 + i);
    }
    double ux = 0, uy = 0, uz = 0, qx = 0, qy = 0, qz = 0, gx = 0, gy = 0, gz = 0;
    double ex = 0, ey = 0, ez = 0, ev = 0;

    const int ntiles = (w.s1 - w.s0 + TB - 1) / TB;
    float4 rp, rv;
    load_source_f32(sg, w.s0 + tid, w.s1, rp, rv);
    for (int t = 0; t < ntiles; ++t) {
      const int buf = t & 1;
      sp[buf][tid] = rp;
      sv[buf][tid] = rv;
      __syncthreads();
      const int ts = w.s0 + t * TB;
      if (t + 1 < ntiles) load_source_f32(sg, ts + TB + tid, w.s1, rp, rv);
      Acc32 a = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
      const bool diag = (ts < w.t0 + TPB) && (w.t0 < ts + TB);
      if (diag)
        tile_f32<DIFF, true, P, TB, U>(sp[buf], sv[buf], g, i - ts, pi.x, pi.y, pi.z, pi.w, vi.x,
                                       vi.y, vi.z, a);
      else
        tile_f32<DIFF, false, P, TB, U>(sp[buf], sv[buf], g, -1, pi.x, pi.y, pi.z, pi.w, vi.x,
                                        vi.y, vi.z, a);
      ux += a.ux; uy += a.uy; uz += a.uz;
      qx += a.qx; qy += a.qy; qz += a.qz;
      gx += a.gx; gy += a.gy; gz += a.gz;
      if (DIFF) { ex += a.ex; ey += a.ey; ez += a.ez; ev += a.ev; }
    }

    if (P > 1) {
#pragma unroll
      for (int off = 1; off < P; off <<= 1) {
        ux += __shfl_xor_sync(0xffffffffu, ux, off);
        uy += __shfl_xor_sync(0xffffffffu, uy, off);
        uz += __shfl_xor_sync(0xffffffffu, uz, off);
        qx += __shfl_xor_sync(0xffffffffu, qx, off);
        qy += __shfl_xor_sync(0xffffffffu, qy, off);
        qz += __shfl_xor_sync(0xffffffffu, qz, off);
        gx += __shfl_xor_sync(0xffffffffu, gx, off);
        gy += __shfl_xor_sync(0xffffffffu, gy, off);
        gz += __shfl_xor_sync(0xffffffffu, gz, off);
        if (DIFF) {
          ex += __shfl_xor_sync(0xffffffffu, ex, off);
          ey += __shfl_xor_sync(0xffffffffu, ey, off);
          ez += __shfl_xor_sync(0xffffffffu, ez, off);
          ev += __shfl_xor_sync(0xffffffffu, ev, off);
        }
      }
    }

    if (valid && g == 0) {
      const double A = kInv4Pi;
      const double ax = vi.x, ay = vi.y, az = vi.z;
      const double Qx = A * qx, Qy = A * qy, Qz = A * qz;
      double dax = (ay * Qz - az * Qy) + 3.0 * A * gx;
      double day = (az * Qx - ax * Qz) + 3.0 * A * gy;
      double daz = (ax * Qy - ay * Qx) + 3.0 * A * gz;
      if (DIFF) {
        const double c = 15.0 * sg.nu * A;
        const double v = vi.w;
        dax += c * (v * ex - ev * ax);
        day += c * (v * ey - ev * ay);
        daz += c * (v * ez - ev * az);
      }
      const size_t n = (size_t)sg.n;
      double *out = sg.partial + (size_t)w.chunk * 6 * n + i;
      out[0] = A * ux;
      out[n] = A * uy;
      out[2 * n] = A * uz;
      out[3 * n] = dax;
      out[4 * n] = day;
      out[5 * n] = daz;
    }
  }
}

using KernelFn = void (*)(const WorkItem *, int, const SegDesc *, int *);

template <bool DIFF>
KernelFn select(const PairConfig &c) {
#define PAWAN_F32_CASE(TB_, P_, U_) \
  if (c.tb == TB_ && c.p == P_ && c.unroll == U_) return &pairs_f32_kernel<TB_, P_, U_, DIFF>;
  PAWAN_F32_CASE(128, 1, 2)
  PAWAN_F32_CASE(128, 1, 4)
  PAWAN_F32_CASE(128, 2, 2)
  PAWAN_F32_CASE(128, 2, 4)
  PAWAN_F32_CASE(128, 4, 2)
  PAWAN_F32_CASE(128, 4, 4)
  PAWAN_F32_CASE(256, 1, 2)
  PAWAN_F32_CASE(256, 1, 4)
  PAWAN_F32_CASE(256, 2, 2)
  PAWAN_F32_CASE(256, 2, 4)
  PAWAN_F32_CASE(256, 4, 2)
  PAWAN_F32_CASE(256, 4, 4)
#undef PAWAN_F32_CASE
  return nullptr;
}

KernelFn select(const PairConfig &c, bool diffusion) {
  return diffusion ? select<true>(c) : select<false>(c);
}

}  // namespace

bool pairs_f32_supported(const PairConfig &c) { return select(c, true) != nullptr; }

cudaError_t pairs_f32_occupancy(const PairConfig &c, bool diffusion, int *blocks_per_sm) {
  KernelFn f = select(c, diffusion);
  if (!f) return cudaErrorInvalidValue;
  return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, f, c.tb, 0);
}

cudaError_t launch_pairs_f32(const PairConfig &c, bool diffusion, int grid, const WorkItem *items,
                             int n_items, const SegDesc *segs, int *next_item, cudaStream_t s) {
  KernelFn f = select(c, diffusion);
  if (!f) return cudaErrorInvalidValue;
  f<<<grid, c.tb, 0, s>>>(items, n_items, segs, next_item);
  return cudaGetLastError();
}

}  // namespace pawan

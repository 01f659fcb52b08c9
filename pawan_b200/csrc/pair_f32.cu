// All-pairs vortex-particle interaction, FP32 pair math with FP64
// accumulation of per-tile partial sums (the hot kernel).
//
// Reference: the pair physics of INTERACT (src/interaction/interaction_utils.h:363-407)
// with KERNEL (src/interaction/highorder.h:48-60), summed over all pairs of a
// system by __interaction::interact (src/interaction/interaction.cpp:95-108).
//
// Gather form.  For target i and source j != i, d = x_i - x_j,
// sigma^2 = (s_i^2 + s_j^2)/2 = h_i + h_j with h = s^2/2, rho^2 = |d|^2:
//   u_i      += q (alpha_j x d)
//   dalpha_i += q (alpha_i x alpha_j) + F [d.(alpha_i x alpha_j)] d
//             + (2 nu Z / sigma^2)(v_i alpha_j - v_j alpha_i)
// with A = 1/(4 pi), w = (rho^2 + sigma^2)^(-1/2):
//   Z = 7.5 A sigma^12 w^15            (= (15/8pi) sigma^-3 (rho_bar^2+1)^-7.5)
//   phi/rho_bar = A (rho^2 + 1.5 sigma^2) w^4 / rho
//   q = (phi/rho_bar - Z) sigma^2 / rho^2,   F = (Z - 3q) / rho^2.
// In units of A: qh = q/A = (ph - 7.5 Zc) sigma^2/rho^2 with ph = (rho^2 +
// 1.5 sigma^2) w^4/rho, Zc = sigma^12 w^15 = Dp sigma^2, Dp = (sigma^2 w^2)^5 w^5;
// F = 3A fh with fh = (2.5 Zc - qh)/rho^2; 2 nu Z/sigma^2 = 15 nu A Dp.
// Two MUFU rsqrt per pair, no division, no pow.
//
// Precision.  The pair kernel is singular like 1/rho^3 inside the smoothing
// radius, and in a finely resolved tube neighbouring particles sit much closer
// than the coordinates' magnitude, with nearly parallel strengths.  Two
// formulations, chosen per (target tile, source tile) from the tiles'
// bounding boxes (a block-uniform branch):
//  * near tiles (box distance below a few smoothing radii, and the tile
//    holding the target itself): positions and strengths in hi+lo FP32 pairs,
//    d = (x_hi,i - x_hi,j) + (x_lo,i - x_lo,j) and delta = alpha_j - alpha_i the
//    same way, so the differences are accurate to the FP64 inputs; alpha_i x
//    alpha_j per pair from the hi/lo strengths with FMA-exact 2x2 determinants
//    (accurate for nearly parallel and antiparallel strengths alike), and
//    diffusion as v_i delta + (v_i - v_j) alpha_i (= v_i alpha_j - v_j alpha_i).
//    ~94 FP32 instructions per pair.
//  * far tiles: hi positions only, and the per-target sums
//      U = sum qh (alpha_j x d), Q = sum qh alpha_j, G = sum fh [alpha_i.(alpha_j x d)] d,
//      E = sum Dp alpha_j, V = sum Dp v_j
//    from which dalpha = alpha_i x (A Q) + 3A G + 15 nu A (v_i E - V alpha_i):
//    49 FP32 instructions per pair (45 without diffusion).
// After each tile both are folded into six FP64 sums (u, dalpha) with the
// target's strength in FP64 (hi + lo).
//
// Layout: one persistent block per SM slot takes work items (target tile x
// source chunk) from a counter; sources stream through a two-stage shared-memory
// ring, each thread loading one source (four float4) for the next tile while
// the block computes the current one.  The result of an item (u, dalpha in
// FP64) goes to its chunk of the partial buffer, which the stage kernel
// reduces in chunk order.
#include "device.cuh"
#include "kernels.h"

namespace pawan {
namespace {

struct Acc32 {
  float ux, uy, uz;
  float qx, qy, qz;  // far: sum qh alpha_j        near: sum qh (alpha_i x delta)
  float gx, gy, gz;
  float ex, ey, ez;  // far: sum Dp alpha_j        near: sum Dp delta
  float ev;          // far: sum Dp v_j            near: sum Dp (v_i - v_j)
};

struct Target {
  float xh, yh, zh, h;
  float xl, yl, zl;
  float ah, bh, ch, v;  // strength hi (x, y, z) and volume
  float al, bl, cl;     // strength lo
};

// A source that contributes exactly zero: far away (every kernel factor
// underflows to 0 and stays finite) with zero strength and volume.
__device__ __forceinline__ void load_source(const SegDesc &sg, int j, int s1, float4 (&r)[4]) {
  if (j < s1) {
    r[0] = __ldg(sg.pos32 + j);
    r[1] = __ldg(sg.vor32 + j);
    r[2] = __ldg(sg.poslo + j);
    r[3] = __ldg(sg.vorlo + j);
  } else {
    r[0] = make_float4(1e18f, 1e18f, 1e18f, 1.0f);
    r[1] = make_float4(0.f, 0.f, 0.f, 0.f);
    r[2] = make_float4(0.f, 0.f, 0.f, 0.f);
    r[3] = make_float4(0.f, 0.f, 0.f, 0.f);
  }
}

template <bool DIFF, int P, int NSRC, int U>
__device__ __forceinline__ void tile_far(const float4 *__restrict__ sp,
                                         const float4 *__restrict__ sv, int g, const Target &T,
                                         Acc32 &a) {
#pragma unroll U
  for (int k = 0; k < NSRC / P; ++k) {
    const int jj = g + P * k;
    const float4 p = sp[jj];
    const float4 s = sv[jj];
    const float dx = T.xh - p.x, dy = T.yh - p.y, dz = T.zh - p.z;
    const float r2 = fmaf(dz, dz, fmaf(dy, dy, dx * dx));
    const float sig2 = T.h + p.w;
    const float w = rsqrtf(r2 + sig2);
    const float ri = rsqrtf(r2);
    const float ri2 = ri * ri;
    const float w2 = w * w;
    const float w4 = w2 * w2;
    const float uu = sig2 * w2;
    const float u2 = uu * uu;
    const float u4 = u2 * u2;
    const float u5 = u4 * uu;
    const float dp = u5 * (w4 * w);
    const float zc = dp * sig2;
    const float ph = fmaf(1.5f, sig2, r2) * w4 * ri;
    const float qh = fmaf(-7.5f, zc, ph) * sig2 * ri2;
    const float fh = fmaf(2.5f, zc, -qh) * ri2;
    const float cx = fmaf(s.y, dz, -s.z * dy);
    const float cy = fmaf(s.z, dx, -s.x * dz);
    const float cz = fmaf(s.x, dy, -s.y * dx);
    const float t = fmaf(T.ch, cz, fmaf(T.bh, cy, T.ah * cx));
    const float ft = fh * t;
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

// a*d - b*c to within 1.5 ulp of the result (Kahan's FMA algorithm): the
// rounding error of b*c is recovered exactly by the second FMA.
__device__ __forceinline__ float det2(float a, float b, float c, float d) {
  const float w = b * c;
  const float e = fmaf(-b, c, w);
  const float f = fmaf(a, d, -w);
  return f + e;
}

// (ah + al) x (bh + bl) with error ~ 1 ulp of the result plus ~eps^2 |a||b|,
// i.e. accurate also for nearly parallel or antiparallel strengths.
__device__ __forceinline__ void cross_accurate(float ax, float ay, float az, float lx, float ly,
                                               float lz, float bx, float by, float bz, float mx,
                                               float my, float mz, float &wx, float &wy,
                                               float &wz) {
  wx = det2(ay, az, by, bz) + fmaf(ay, mz, fmaf(-az, my, fmaf(ly, bz, -lz * by)));
  wy = det2(az, ax, bz, bx) + fmaf(az, mx, fmaf(-ax, mz, fmaf(lz, bx, -lx * bz)));
  wz = det2(ax, ay, bx, by) + fmaf(ax, my, fmaf(-ay, mx, fmaf(lx, by, -ly * bx)));
}

template <bool DIFF, bool CHECK, int P, int NSRC, int U>
__device__ __forceinline__ void tile_near(const float4 *__restrict__ sp,
                                          const float4 *__restrict__ sv,
                                          const float4 *__restrict__ spl,
                                          const float4 *__restrict__ svl, int g, int skip,
                                          const Target &T, Acc32 &a) {
  // near tiles are a few percent of the work: a shallow unroll keeps the
  // register budget of the far loop
#pragma unroll(U < 2 ? U : 2)
  for (int k = 0; k < NSRC / P; ++k) {
    const int jj = g + P * k;
    const float4 p = sp[jj];
    const float4 s = sv[jj];
    const float4 pl = spl[jj];
    const float4 sl = svl[jj];
    const float dx = (T.xh - p.x) + (T.xl - pl.x);
    const float dy = (T.yh - p.y) + (T.yl - pl.y);
    const float dz = (T.zh - p.z) + (T.zl - pl.z);
    const float r2 = fmaf(dz, dz, fmaf(dy, dy, dx * dx));
    const float sig2 = T.h + p.w;
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
    // velocity: alpha_j x d
    const float cx = fmaf(s.y, dz, -s.z * dy);
    const float cy = fmaf(s.z, dx, -s.x * dz);
    const float cz = fmaf(s.x, dy, -s.y * dx);
    // stretching: alpha_i x alpha_j from the hi/lo strengths
    float wx, wy, wz;
    cross_accurate(T.ah, T.bh, T.ch, T.al, T.bl, T.cl, s.x, s.y, s.z, sl.x, sl.y, sl.z, wx, wy, wz);
    const float t = fmaf(dz, wz, fmaf(dy, wy, dx * wx));
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
    a.qx = fmaf(qh, wx, a.qx);
    a.qy = fmaf(qh, wy, a.qy);
    a.qz = fmaf(qh, wz, a.qz);
    a.gx = fmaf(ft, dx, a.gx);
    a.gy = fmaf(ft, dy, a.gy);
    a.gz = fmaf(ft, dz, a.gz);
    if (DIFF) {
      // delta = alpha_j - alpha_i from the hi/lo strengths
      const float ex = (s.x - T.ah) + (sl.x - T.al);
      const float ey = (s.y - T.bh) + (sl.y - T.bl);
      const float ez = (s.z - T.ch) + (sl.z - T.cl);
      a.ex = fmaf(dp, ex, a.ex);
      a.ey = fmaf(dp, ey, a.ey);
      a.ez = fmaf(dp, ez, a.ez);
      a.ev = fmaf(dp, T.v - s.w, a.ev);
    }
  }
}

__device__ __forceinline__ float box_gap2(float4 alo, float4 ahi, float4 blo, float4 bhi) {
  const float gx = fmaxf(0.f, fmaxf(alo.x - bhi.x, blo.x - ahi.x));
  const float gy = fmaxf(0.f, fmaxf(alo.y - bhi.y, blo.y - ahi.y));
  const float gz = fmaxf(0.f, fmaxf(alo.z - bhi.z, blo.z - ahi.z));
  return gx * gx + gy * gy + gz * gz;
}

template <int TB, int P, int U, bool DIFF>
__global__ void __launch_bounds__(TB, (TB <= 128 ? 4 : 2))
    pairs_f32_kernel(const WorkItem *__restrict__ items, int n_items,
                     const SegDesc *__restrict__ segs, int *__restrict__ next_item) {
  constexpr int TPB = TB / P;
  __shared__ float4 sp[2][TB];
  __shared__ float4 sv[2][TB];
  __shared__ float4 spl[2][TB];
  __shared__ float4 svl[2][TB];
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
    Target T;
    {
      float4 a = make_float4(0.f, 0.f, 0.f, 1.f), b = make_float4(0.f, 0.f, 0.f, 0.f);
      float4 c = b, d = b;
      if (valid) {
        a = __ldg(sg.pos32 + i);
        b = __ldg(sg.vor32 + i);
        c = __ldg(sg.poslo + i);
        d = __ldg(sg.vorlo + i);
      }
      T.xh = a.x; T.yh = a.y; T.zh = a.z; T.h = a.w;
      T.ah = b.x; T.bh = b.y; T.ch = b.z; T.v = b.w;
      T.xl = c.x; T.yl = c.y; T.zl = c.z;
      T.al = d.x; T.bl = d.y; T.cl = d.z;
    }
    // target strength in FP64 (hi + lo) for the per-tile folds
    const double ax = (double)T.ah + (double)T.al;
    const double ay = (double)T.bh + (double)T.bl;
    const double az = (double)T.ch + (double)T.cl;
    const double A = kInv4Pi;
    const double cnu = 15.0 * sg.nu * A;
    double ou0 = 0, ou1 = 0, ou2 = 0, oa0 = 0, oa1 = 0, oa2 = 0;

    // the target tile lies inside source tile t0 / TB (TPB divides TB)
    const float4 tlo = __ldg(sg.boxes + 2 * (w.t0 / TB));
    const float4 thi = __ldg(sg.boxes + 2 * (w.t0 / TB) + 1);

    const int ntiles = (w.s1 - w.s0 + TB - 1) / TB;
    float4 r[4];
    load_source(sg, w.s0 + tid, w.s1, r);
    for (int t = 0; t < ntiles; ++t) {
      const int buf = t & 1;
      sp[buf][tid] = r[0];
      sv[buf][tid] = r[1];
      spl[buf][tid] = r[2];
      svl[buf][tid] = r[3];
      __syncthreads();
      const int ts = w.s0 + t * TB;
      if (t + 1 < ntiles) load_source(sg, ts + TB + tid, w.s1, r);
      Acc32 a = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
      const bool diag = (ts < w.t0 + TPB) && (w.t0 < ts + TB);
      const float4 slo = __ldg(sg.boxes + 2 * (ts / TB));
      const float4 shi = __ldg(sg.boxes + 2 * (ts / TB) + 1);
      const bool near = diag || box_gap2(tlo, thi, slo, shi) < sg.near2;
      if (!near) {
        tile_far<DIFF, P, TB, U>(sp[buf], sv[buf], g, T, a);
        const double Qx = A * a.qx, Qy = A * a.qy, Qz = A * a.qz;
        oa0 += (ay * Qz - az * Qy) + 3.0 * A * a.gx;
        oa1 += (az * Qx - ax * Qz) + 3.0 * A * a.gy;
        oa2 += (ax * Qy - ay * Qx) + 3.0 * A * a.gz;
        if (DIFF) {
          oa0 += cnu * ((double)T.v * a.ex - (double)a.ev * ax);
          oa1 += cnu * ((double)T.v * a.ey - (double)a.ev * ay);
          oa2 += cnu * ((double)T.v * a.ez - (double)a.ev * az);
        }
      } else {
        if (diag)
          tile_near<DIFF, true, P, TB, U>(sp[buf], sv[buf], spl[buf], svl[buf], g, i - ts, T, a);
        else
          tile_near<DIFF, false, P, TB, U>(sp[buf], sv[buf], spl[buf], svl[buf], g, -1, T, a);
        oa0 += A * a.qx + 3.0 * A * a.gx;
        oa1 += A * a.qy + 3.0 * A * a.gy;
        oa2 += A * a.qz + 3.0 * A * a.gz;
        if (DIFF) {
          oa0 += cnu * ((double)T.v * a.ex + (double)a.ev * ax);
          oa1 += cnu * ((double)T.v * a.ey + (double)a.ev * ay);
          oa2 += cnu * ((double)T.v * a.ez + (double)a.ev * az);
        }
      }
      ou0 += A * a.ux;
      ou1 += A * a.uy;
      ou2 += A * a.uz;
    }

    if (P > 1) {
#pragma unroll
      for (int off = 1; off < P; off <<= 1) {
        ou0 += __shfl_xor_sync(0xffffffffu, ou0, off);
        ou1 += __shfl_xor_sync(0xffffffffu, ou1, off);
        ou2 += __shfl_xor_sync(0xffffffffu, ou2, off);
        oa0 += __shfl_xor_sync(0xffffffffu, oa0, off);
        oa1 += __shfl_xor_sync(0xffffffffu, oa1, off);
        oa2 += __shfl_xor_sync(0xffffffffu, oa2, off);
      }
    }

    if (valid && g == 0) {
      const size_t n = (size_t)sg.n;
      double *out = sg.partial + (size_t)w.chunk * 6 * n + i;
      out[0] = ou0;
      out[n] = ou1;
      out[2 * n] = ou2;
      out[3 * n] = oa0;
      out[4 * n] = oa1;
      out[5 * n] = oa2;
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

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
//  * far tiles: hi positions relative to the centre c of the source tile's
//    box, x' = x - c, and two crosses formed once per particle and tile
//    instead of once per pair, beta_j = alpha_j x x'_j (when the tile is
//    staged) and gamma_i = x'_i x alpha_i (per target), so that
//      alpha_j x d = alpha_j x x'_i - beta_j,
//      alpha_i.(alpha_j x d) = alpha_j.gamma_i - alpha_i.beta_j.
//    Per target the sums
//      W = sum qh beta_j, Q = sum qh alpha_j, G = sum fh [alpha_i.(alpha_j x d)] d,
//      E = sum Dp alpha_j, V = sum Dp v_j
//    give u = A (Q x x'_i - W) and
//    dalpha = alpha_i x (A Q) + 3A G + 15 nu A (v_i E - V alpha_i).
//    The split costs accuracy where |x'| >> |d|; a tile pair is far only when
//    its box gap is at least the source box's half-diagonal, which bounds
//    |x'_i| + |x'_j| by 3 |d|.  When both tiles hold one smoothing radius
//    (sigma^2 = 2h for every pair) the factor sigma^2 and the constants leave
//    the pair loop for the per-tile fold (kernel_scalars_uniform).
//    39 FP32 instructions per pair with one radius (43 with several; 4 fewer
//    without diffusion).
//  * far tiles whose every pair is at least 6 smoothing radii apart (box gap
//    >= 6 sigma_max): the far formulation without the Z terms, which are below
//    3e-9 of the terms they are added to there (kernel_scalars_nz); 29 FP32
//    instructions per pair with one radius, no diffusion sums.
//  * far tiles whose every pair is at least 16 smoothing radii apart: the
//    Z-free field with its smoothing factor by a two-term series exact to
//    3e-8 there (kernel_scalars_series); one MUFU rsqrt per pair instead of
//    an rsqrt and a reciprocal.
// After each tile both are folded into six FP64 sums (u, dalpha) with the
// target's strength in FP64 (hi + lo).
//
// Layout: one persistent block per SM slot takes work items (target tile x
// source chunk) from a counter; sources stream through a two-stage shared-memory
// ring, each thread starting asynchronous copies (cp.async, no registers held)
// of one source (four float4) for the next tile while the block computes the
// current one.  The result of an item (u, dalpha in FP64) goes to its slot of
// the partial buffer; the block that completes a target tile sums the tile's
// slots in chunk order into the rates (finish_item, device.cuh).
#include <mutex>
#include <set>
#include <utility>

#include "device.cuh"
#include "kernels.h"

namespace pawan {
namespace {

struct Acc32 {
  float ux, uy, uz;  // far: sum qh beta_j         near: sum qh (alpha_j x d)
  float qx, qy, qz;  // far: sum qh alpha_j        near: sum qh (alpha_i x delta)
  float gx, gy, gz;
  float ex, ey, ez;  // far: sum Dp alpha_j        near: sum Dp delta
  float ev;          // far: sum Dp v_j            near: sum Dp (v_i - v_j)
};

// A target's hi parts (registers for the whole work item); the lo parts are
// read from global memory only for near tiles.
struct Target {
  float xh, yh, zh, h;
  float ah, bh, ch, v;  // strength hi (x, y, z) and volume
};

// A target relative to the current far source tile.
struct FarTarget {
  float x, y, z;     // x'_i = x_i - c
  float gx, gy, gz;  // gamma_i = x'_i x alpha_i
};

__device__ __forceinline__ float rcp_approx(float x) {
  float r;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}

__device__ __forceinline__ void cp_async16(float4 *smem, const float4 *gmem) {
  const unsigned a = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(a), "l"(gmem) : "memory");
}

// Starts the copy of source j into one shared-memory slot (pos32, vor32,
// poslo, vorlo), or writes a source that contributes exactly zero when j is
// past the chunk: far away (every kernel factor underflows to 0 and stays
// finite) with zero strength and volume.
__device__ __forceinline__ void stage_source(const SegDesc &sg, int j, int s1, float4 *p,
                                             float4 *v, float4 *pl, float4 *vl) {
  if (j < s1) {
    cp_async16(p, sg.pos32 + j);
    cp_async16(v, sg.vor32 + j);
    cp_async16(pl, sg.poslo + j);
    cp_async16(vl, sg.vorlo + j);
  } else {
    *p = make_float4(1e18f, 1e18f, 1e18f, 1.0f);
    *v = make_float4(0.f, 0.f, 0.f, 0.f);
    *pl = make_float4(0.f, 0.f, 0.f, 0.f);
    *vl = make_float4(0.f, 0.f, 0.f, 0.f);
  }
  asm volatile("cp.async.commit_group;" ::: "memory");
}

__device__ __forceinline__ void wait_staged() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

// q, F and the diffusion factor of one pair in units of A = 1/(4 pi), from
// sigma^2, w = (rho^2 + sigma^2)^-1/2 and ri = 1/rho (u = sigma^2 w^2):
//   Dp = (u w)^5 = sigma^10 w^15,  Zc = Dp sigma^2,
//   ph = (rho^2 + 1.5 sigma^2) w^4 / rho = (1 + u/2) w^2 / rho,
//   qh = (ph - 7.5 Zc) sigma^2 / rho^2,   fh = (2.5 Zc - qh) / rho^2.
// 16 FP32 instructions.
__device__ __forceinline__ void kernel_scalars(float sig2, float w, float ri, float &qh, float &fh,
                                               float &dp) {
  const float w2 = w * w;
  const float uu = sig2 * w2;
  const float v = uu * w;
  const float v2 = v * v;
  const float v4 = v2 * v2;
  dp = v4 * v;
  const float zc = dp * sig2;
  const float ph = fmaf(0.5f, uu, 1.0f) * w2 * ri;
  const float ri2 = ri * ri;
  qh = fmaf(-7.5f, zc, ph) * sig2 * ri2;
  fh = fmaf(2.5f, zc, -qh) * ri2;
}

// kernel_scalars for sigma^2 = 2h the same for every pair of the tile, with
// the factors that do not vary per pair left to the per-tile fold: returns
//   qs = qh / sigma^2,  fs = fh / sigma^2,  ds = Dp / 32,
// from u' = h w^2 = u/2 and v' = u' w = v/2 (so ds = v'^5):
//   ph = (1 + u') w^2 / rho,  qs = (ph - 240 sigma^2 ds) / rho^2,
//   fs = (80 ds - qs) / rho^2.
// 1/rho^2 comes from the MUFU reciprocal; 12 FP32 instructions.
__device__ __forceinline__ void kernel_scalars_uniform(float h, float c240, float w, float ri,
                                                       float r2, float &qs, float &fs, float &ds) {
  const float y = w * w;
  const float u = h * y;
  const float v = u * w;
  const float v2 = v * v;
  ds = v2 * v2 * v;
  const float ph = fmaf(u, y, y) * ri;
  const float ri2 = rcp_approx(r2);
  qs = fmaf(c240, ds, ph) * ri2;
  fs = fmaf(80.f, ds, -qs) * ri2;
}

// Far field without the Z terms.  Where every pair of a tile pair has
// rho >= 6 sigma (checked on the tiles' boxes), Z = (15/8pi) sigma^-3
// (rho_bar^2 + 1)^-7.5 is below 3e-9 of phi/rho_bar in q = (phi/rho_bar - Z)
// / rho_bar^2 and of 3q in F = (Z - 3q)/rho^2, i.e. twenty times below FP32
// rounding, and the diffusion rate 2 nu Z / sigma^2 (v_i alpha_j - v_j alpha_i)
// of those pairs is as small against the near-field diffusion: the terms are
// zero at FP32 resolution and are not formed.  What remains, with
// y = 1/(rho^2 + sigma^2) and (rho^2 + 1.5 sigma^2) w^4 = y (1 + y sigma^2/2):
//   qh = y (1 + y sigma^2/2) sigma^2 / rho^3,   fh = -qh / rho^2.
// kernel_scalars_nz returns them for one sigma^2 per pair (12 FP32
// instructions with the MUFU reciprocal and rsqrt); the uniform-radius form
// returns qs = qh / sigma^2, -fs = qh / (sigma^2 rho^2) (8 instructions).
__device__ __forceinline__ void kernel_scalars_nz(float sig2, float r2, float &qh, float &nfh) {
  const float y = rcp_approx(r2 + sig2);
  const float ri = rsqrtf(r2);
  const float ri2 = ri * ri;
  const float hy = 0.5f * sig2 * y;
  const float ph = fmaf(hy, y, y);
  qh = ph * sig2 * ri * ri2;
  nfh = qh * ri2;
}

// Far field without the Z terms, and a series for the smoothing factor.
// With eps = sigma^2 / rho^2,
//   rho^2 y (1 + y sigma^2/2) = 1/(1 + eps) + (eps/2)/(1 + eps)^2
//                             = 1 - eps/2 + 0 eps^2 + eps^3/2 - ...,
// so where every pair of a tile pair has rho >= 16 sigma (eps <= 1/256, checked
// on the tiles' boxes) the two-term form 1 - sigma^2/(2 rho^2) is exact to
// 3.0e-8 relative, below FP32's unit roundoff (6e-8):
//   qh = sigma^2 rho^-5 (1 - sigma^2 rho^-2 / 2),   fh = -qh / rho^2,
// one MUFU rsqrt per pair instead of an rsqrt and a reciprocal (the
// uniform-radius form returns qs = qh / sigma^2 = rho^-5 (1 - h rho^-2)).
__device__ __forceinline__ void kernel_scalars_series(float sig2, float r2, float &qh, float &nfh) {
  const float ri = rsqrtf(r2);
  const float ri2 = ri * ri;
  const float e = sig2 * ri2;
  const float c = fmaf(-0.5f, e, 1.0f);
  qh = e * ri * ri2 * c;
  nfh = qh * ri2;
}

// The Gaussian kernel (gaussian.h:20-59) in the units of kernel_scalars: with
// x2 = rho^2/sigma^2, e = exp(-x2/2) and K = sqrt(2/pi),
//   qh = gq / sigma^3,        gq = (erf(x/sqrt 2)/x - K e) / x2,
//   fh = gf / (3 sigma^5),    gf = (K e - 3 gq) / x2,
//   dp = (2/15) K e / sigma^5.
// Below x2 = 1 the closed forms lose digits to cancellation; there gq and gf
// come from their power series in y = -x2/2,
//   gq = K sum_m y^m / (m! (2m+3)),   gf = -K sum_m y^m / (m! (2m+5)),
// nine terms (relative truncation error < 1e-8 at x2 = 1).
// Far field of the Gaussian kernel (gauss_far): where every pair of a tile pair
// has x = rho/sigma >= 7 (checked on the tiles' boxes), e = exp(-x2/2) <=
// 2.3e-11 and erf(x/sqrt 2) = 1 - 2.6e-12, so gq = 1/x^3 to 1.3e-10 relative
// (K e x against 1), gf = -3/x^5 to 2.1e-9 (K e x^3/3 against 1) and dp is 0
// at FP32 resolution:
//   qh = rho^-3,   fh = -rho^-5 = -qh / rho^2,   dp = 0,
// the singular field, one MUFU rsqrt and three multiplies per pair in place of
// an exp and an erf (the far loops' series branches with KERN = Gaussian).
__device__ __forceinline__ void gauss_scalars(float sig2, float r2, float ri, float &qh, float &fh,
                                              float &dp) {
  const float K = 0.797884561f;
  const float is = rsqrtf(sig2);
  const float is2 = is * is;
  const float is3 = is2 * is;
  const float x2 = r2 * is2;
  const float e = expf(-0.5f * x2);
  float gq, gf;
  if (x2 < 1.0f) {
    const float y = -0.5f * x2;
    float sq = 1.0f / (40320.0f * 19.0f), sf = 1.0f / (40320.0f * 21.0f);
    sq = fmaf(sq, y, 1.0f / (5040.0f * 17.0f));
    sf = fmaf(sf, y, 1.0f / (5040.0f * 19.0f));
    sq = fmaf(sq, y, 1.0f / (720.0f * 15.0f));
    sf = fmaf(sf, y, 1.0f / (720.0f * 17.0f));
    sq = fmaf(sq, y, 1.0f / (120.0f * 13.0f));
    sf = fmaf(sf, y, 1.0f / (120.0f * 15.0f));
    sq = fmaf(sq, y, 1.0f / (24.0f * 11.0f));
    sf = fmaf(sf, y, 1.0f / (24.0f * 13.0f));
    sq = fmaf(sq, y, 1.0f / (6.0f * 9.0f));
    sf = fmaf(sf, y, 1.0f / (6.0f * 11.0f));
    sq = fmaf(sq, y, 1.0f / (2.0f * 7.0f));
    sf = fmaf(sf, y, 1.0f / (2.0f * 9.0f));
    sq = fmaf(sq, y, 1.0f / 5.0f);
    sf = fmaf(sf, y, 1.0f / 7.0f);
    sq = fmaf(sq, y, 1.0f / 3.0f);
    sf = fmaf(sf, y, 1.0f / 5.0f);
    gq = K * sq;
    gf = -K * sf;
  } else {
    const float x = r2 * ri * is;  // rho / sigma
    const float ix = rcp_approx(x);
    const float ix2 = ix * ix;
    gq = fmaf(erff(0.707106781f * x), ix, -K * e) * ix2;
    gf = fmaf(-3.0f, gq, K * e) * ix2;
  }
  const float is5 = is3 * is2;
  qh = gq * is3;
  fh = gf * is5 * (1.0f / 3.0f);
  dp = (2.0f / 15.0f) * K * e * is5;
}

// Far tile, shared-memory format (written when the tile is staged):
//   sa[j] = (x'_j, h_j),  sb[j] = (alpha_j, v_j),  sc[j] = (beta_j, 0).
// UNI: every pair has sigma^2 = 2 hu (sums in the units of
// kernel_scalars_uniform).  NZ: the Z-free far field; SER (with NZ): its
// two-term series (kernel_scalars_series).
template <bool DIFF, bool UNI, int P, int R, int NSRC, int U, int KERN, bool NZ, bool SER = false>
__device__ __forceinline__ void tile_far(const float4 *__restrict__ sa,
                                         const float4 *__restrict__ sb,
                                         const float4 *__restrict__ sc, int g,
                                         const Target (&T)[R], const FarTarget (&F)[R], float hu,
                                         Acc32 (&a)[R]) {
  const float s2u = 2.f * hu;
  const float c240 = -480.f * hu;
#pragma unroll U
  for (int k = 0; k < NSRC / P; ++k) {
    const int jj = g + P * k;
    const float4 p = sa[jj];
    const float4 s = sb[jj];
    const float4 b = sc[jj];
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const float dx = F[r].x - p.x, dy = F[r].y - p.y, dz = F[r].z - p.z;
      const float r2 = fmaf(dz, dz, fmaf(dy, dy, dx * dx));
      float qh, fh, dp;
      if (NZ && SER) {
        // Z-free far field by the series (kernel_scalars_series), or the
        // Gaussian kernel's far field (gauss_far)
        float nfh;
        if (KERN == KERNEL_GAUSSIAN) {
          const float ri = rsqrtf(r2);
          const float ri2 = ri * ri;
          qh = ri * ri2;
          nfh = qh * ri2;
        } else if (UNI) {
          const float ri = rsqrtf(r2);
          const float ri2 = ri * ri;
          qh = ri * ri2 * fmaf(-hu, ri2, 1.0f) * ri2;
          nfh = qh * ri2;
        } else {
          kernel_scalars_series(T[r].h + p.w, r2, qh, nfh);
        }
        fh = -nfh;
        dp = 0.f;
      } else if (NZ) {
        // Z-free far field (kernel_scalars_nz); the diffusion sums stay 0
        float nfh;
        if (UNI) {
          const float y = rcp_approx(r2 + s2u);
          const float ri = rsqrtf(r2);
          const float ri2 = ri * ri;
          qh = fmaf(hu * y, y, y) * ri * ri2;
          nfh = qh * ri2;
        } else {
          kernel_scalars_nz(T[r].h + p.w, r2, qh, nfh);
        }
        fh = -nfh;
        dp = 0.f;
      } else if (UNI) {
        const float w = rsqrtf(r2 + s2u);
        const float ri = rsqrtf(r2);
        kernel_scalars_uniform(hu, c240, w, ri, r2, qh, fh, dp);
      } else if (KERN == KERNEL_GAUSSIAN) {
        gauss_scalars(T[r].h + p.w, r2, rsqrtf(r2), qh, fh, dp);
      } else {
        const float sig2 = T[r].h + p.w;
        const float w = rsqrtf(r2 + sig2);
        const float ri = rsqrtf(r2);
        kernel_scalars(sig2, w, ri, qh, fh, dp);
      }
      // alpha_i.(alpha_j x d) = alpha_j.gamma_i - alpha_i.beta_j
      const float t = fmaf(-T[r].ch, b.z, fmaf(-T[r].bh, b.y, fmaf(-T[r].ah, b.x,
                      fmaf(s.z, F[r].gz, fmaf(s.y, F[r].gy, s.x * F[r].gx)))));
      const float ft = fh * t;
      a[r].ux = fmaf(qh, b.x, a[r].ux);
      a[r].uy = fmaf(qh, b.y, a[r].uy);
      a[r].uz = fmaf(qh, b.z, a[r].uz);
      a[r].qx = fmaf(qh, s.x, a[r].qx);
      a[r].qy = fmaf(qh, s.y, a[r].qy);
      a[r].qz = fmaf(qh, s.z, a[r].qz);
      a[r].gx = fmaf(ft, dx, a[r].gx);
      a[r].gy = fmaf(ft, dy, a[r].gy);
      a[r].gz = fmaf(ft, dz, a[r].gz);
      if (DIFF && !NZ) {
        a[r].ex = fmaf(dp, s.x, a[r].ex);
        a[r].ey = fmaf(dp, s.y, a[r].ey);
        a[r].ez = fmaf(dp, s.z, a[r].ez);
        a[r].ev = fmaf(dp, s.w, a[r].ev);
      }
    }
  }
}

// ---- packed far path: two sources per FP32x2 instruction -----------------
// The far formulation above with every FP32 operation on a pair of sources
// (FFMA2/FMUL2/FADD2 issue once for two lanes' worth of work, halving the
// issue slots the FMA pipe needs).  Shared-memory layout of a far tile, per
// source pair k = (a, b) = (2k, 2k+1):
//   f0[k] = (-x'_a, -x'_b, -y'_a, -y'_b)   f1[k] = (-z'_a, -z'_b, h_a, h_b)
//   f2[k] = (ax_a, ax_b, ay_a, ay_b)       f3[k] = (az_a, az_b, v_a, v_b)
//   f4[k] = (bx_a, bx_b, by_a, by_b)       f5[k] = (bz_a, bz_b)   (beta = alpha x x')
// so every load yields operand pairs and the target enters each instruction
// as a broadcast pair held in registers.  Signs are arranged so that no
// operand needs negating in the loop (a negated pair costs two scalar
// instructions): positions are stored negated, the target's strength is held
// negated, and the loop accumulates -fh.

struct Acc2 {
  float2 wx, wy, wz;  // sum qh beta_j
  float2 qx, qy, qz;  // sum qh alpha_j
  float2 gx, gy, gz;  // sum -fh t d
  float2 ex, ey, ez;  // sum Dp alpha_j
  float2 ev;          // sum Dp v_j
};

struct Target2 {
  float2 x, y, z;     // x'_i, broadcast
  float2 h;           // h_i, broadcast
  float2 na, nb, nc;  // -alpha_i (hi), broadcast
  float2 gx, gy, gz;  // gamma_i = x'_i x alpha_i, broadcast
};

__device__ __forceinline__ float2 bc2(float v) { return make_float2(v, v); }

// 1/rho^2 of a source pair on a uniform-radius tile, given ri = rho^-1:
// RM = 1 from the MUFU reciprocal (two XU operations), RM = 2 as ri * ri (one
// FMA-pipe FMUL2).  (One of each per pair was measured too: slower than both
// on the ring pair, the helical wake and the ragged batch.)
template <int RM>
__device__ __forceinline__ float2 inv_r2(float2 r2, float2 ri) {
  if (RM == 1) return make_float2(rcp_approx(r2.x), rcp_approx(r2.y));
  return __fmul2_rn(ri, ri);
}

template <bool DIFF, bool UNI, int RM, int NSRC, int U, int KERN, bool NZ, bool SER = false>
__device__ __forceinline__ void tile_far_packed(const float4 *__restrict__ f0,
                                                const float4 *__restrict__ f1,
                                                const float4 *__restrict__ f2,
                                                const float4 *__restrict__ f3,
                                                const float4 *__restrict__ f4,
                                                const float2 *__restrict__ f5, const Target2 &T,
                                                float hu, Acc2 &a) {
  const float2 s2u = bc2(2.f * hu), h2 = bc2(hu), c240 = bc2(-480.f * hu);
  const float2 nh2 = bc2(-hu), one2 = bc2(1.0f), nhalf2 = bc2(-0.5f);
#pragma unroll U
  for (int k = 0; k < NSRC / 2; ++k) {
    const float4 A0 = f0[k], A1 = f1[k], A2 = f2[k], A3 = f3[k], A4 = f4[k];
    const float2 bz = f5[k];
    const float2 npx = make_float2(A0.x, A0.y), npy = make_float2(A0.z, A0.w);
    const float2 npz = make_float2(A1.x, A1.y), hj = make_float2(A1.z, A1.w);
    const float2 sx = make_float2(A2.x, A2.y), sy = make_float2(A2.z, A2.w);
    const float2 sz = make_float2(A3.x, A3.y), sv = make_float2(A3.z, A3.w);
    const float2 bx = make_float2(A4.x, A4.y), by = make_float2(A4.z, A4.w);
    const float2 dx = __fadd2_rn(T.x, npx);
    const float2 dy = __fadd2_rn(T.y, npy);
    const float2 dz = __fadd2_rn(T.z, npz);
    const float2 r2 = __ffma2_rn(dz, dz, __ffma2_rn(dy, dy, __fmul2_rn(dx, dx)));
    float2 qh, nfh, dp;
    if (NZ && SER) {
      // Z-free far field by the series in pairs (kernel_scalars_series):
      // one MUFU rsqrt per source (and a reciprocal for 1/rho^2 when RM =
      // 1), 5 FP32x2 operations with one radius (6 when RM = 2)
      const float2 ri = make_float2(rsqrtf(r2.x), rsqrtf(r2.y));
      const float2 ri2 = inv_r2<RM>(r2, ri);
      if (KERN == KERNEL_GAUSSIAN) {
        // the Gaussian kernel's far field (gauss_far): qh = rho^-3
        qh = __fmul2_rn(ri, ri2);
      } else if (UNI) {
        qh = __fmul2_rn(__fmul2_rn(__fmul2_rn(ri, ri2), __ffma2_rn(nh2, ri2, one2)), ri2);
      } else {
        const float2 e = __fmul2_rn(__fadd2_rn(T.h, hj), ri2);
        qh = __fmul2_rn(__fmul2_rn(__fmul2_rn(e, ri), ri2), __ffma2_rn(nhalf2, e, one2));
      }
      nfh = __fmul2_rn(qh, ri2);
      dp = make_float2(0.f, 0.f);
    } else if (NZ) {
      // Z-free far field in pairs (kernel_scalars_nz), no diffusion sums
      if (UNI) {
        const float2 sr = __fadd2_rn(r2, s2u);
        const float2 y = make_float2(rcp_approx(sr.x), rcp_approx(sr.y));
        const float2 ri = make_float2(rsqrtf(r2.x), rsqrtf(r2.y));
        const float2 ri2 = inv_r2<RM>(r2, ri);
        const float2 ph = __ffma2_rn(__fmul2_rn(h2, y), y, y);
        qh = __fmul2_rn(__fmul2_rn(ph, ri), ri2);
        nfh = __fmul2_rn(qh, ri2);
      } else {
        const float2 sig2 = __fadd2_rn(T.h, hj);
        float qa, fa, qb, fb;
        kernel_scalars_nz(sig2.x, r2.x, qa, fa);
        kernel_scalars_nz(sig2.y, r2.y, qb, fb);
        qh = make_float2(qa, qb);
        nfh = make_float2(fa, fb);
      }
      dp = make_float2(0.f, 0.f);
    } else if (UNI) {
      // kernel_scalars_uniform in pairs, returning -fs
      const float2 sr = __fadd2_rn(r2, s2u);
      const float2 w = make_float2(rsqrtf(sr.x), rsqrtf(sr.y));
      const float2 ri = make_float2(rsqrtf(r2.x), rsqrtf(r2.y));
      // which pipe has room for 1/rho^2 depends on the instruction mix
      const float2 ri2 = inv_r2<RM>(r2, ri);
      const float2 y = __fmul2_rn(w, w);
      const float2 u = __fmul2_rn(h2, y);
      const float2 v = __fmul2_rn(u, w);
      const float2 v2 = __fmul2_rn(v, v);
      dp = __fmul2_rn(__fmul2_rn(v2, v2), v);
      const float2 ph = __fmul2_rn(__ffma2_rn(u, y, y), ri);
      qh = __fmul2_rn(__ffma2_rn(c240, dp, ph), ri2);
      nfh = __fmul2_rn(__ffma2_rn(bc2(-80.f), dp, qh), ri2);
    } else if (KERN == KERNEL_GAUSSIAN) {
      // one source at a time (exp and erf do not pair), returning -fh
      const float2 sig2 = __fadd2_rn(T.h, hj);
      float qa, fa, da, qb, fb, db;
      gauss_scalars(sig2.x, r2.x, rsqrtf(r2.x), qa, fa, da);
      gauss_scalars(sig2.y, r2.y, rsqrtf(r2.y), qb, fb, db);
      qh = make_float2(qa, qb);
      nfh = make_float2(-fa, -fb);
      dp = make_float2(da, db);
    } else {
      // kernel_scalars in pairs, returning -fh
      const float2 sig2 = __fadd2_rn(T.h, hj);
      const float2 sr = __fadd2_rn(r2, sig2);
      const float2 w = make_float2(rsqrtf(sr.x), rsqrtf(sr.y));
      const float2 ri = make_float2(rsqrtf(r2.x), rsqrtf(r2.y));
      const float2 w2 = __fmul2_rn(w, w);
      const float2 uu = __fmul2_rn(sig2, w2);
      const float2 v = __fmul2_rn(uu, w);
      const float2 v2 = __fmul2_rn(v, v);
      dp = __fmul2_rn(__fmul2_rn(v2, v2), v);
      const float2 zc = __fmul2_rn(dp, sig2);
      const float2 ph = __fmul2_rn(__fmul2_rn(__ffma2_rn(bc2(0.5f), uu, bc2(1.0f)), w2), ri);
      const float2 ri2 = __fmul2_rn(ri, ri);
      qh = __fmul2_rn(__fmul2_rn(__ffma2_rn(bc2(-7.5f), zc, ph), sig2), ri2);
      nfh = __fmul2_rn(__ffma2_rn(bc2(-2.5f), zc, qh), ri2);
    }
    // alpha_i.(alpha_j x d) = alpha_j.gamma_i - alpha_i.beta_j
    const float2 t = __ffma2_rn(T.nc, bz, __ffma2_rn(T.nb, by, __ffma2_rn(T.na, bx,
                     __ffma2_rn(sz, T.gz, __ffma2_rn(sy, T.gy, __fmul2_rn(sx, T.gx))))));
    const float2 nft = __fmul2_rn(nfh, t);
    a.wx = __ffma2_rn(qh, bx, a.wx);
    a.wy = __ffma2_rn(qh, by, a.wy);
    a.wz = __ffma2_rn(qh, bz, a.wz);
    a.qx = __ffma2_rn(qh, sx, a.qx);
    a.qy = __ffma2_rn(qh, sy, a.qy);
    a.qz = __ffma2_rn(qh, sz, a.qz);
    a.gx = __ffma2_rn(nft, dx, a.gx);
    a.gy = __ffma2_rn(nft, dy, a.gy);
    a.gz = __ffma2_rn(nft, dz, a.gz);
    if (DIFF && !NZ) {
      a.ex = __ffma2_rn(dp, sx, a.ex);
      a.ey = __ffma2_rn(dp, sy, a.ey);
      a.ez = __ffma2_rn(dp, sz, a.ez);
      a.ev = __ffma2_rn(dp, sv, a.ev);
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

// (a + a_lo) x (b + b_lo) for a target strength a + a_lo and a source strength
// b + b_lo (FP32 hi + lo), accurate to a few ulp of the result also for nearly
// parallel or antiparallel strengths, in 19 operations (cross_accurate: 27).
// With mu = (a.b)/|a|^2, v = b - mu a is formed by one FMA per component, so
// exactly up to its own rounding, and a x v = a x b whatever mu's rounding
// (its error only moves v along a).  v is (nearly) perpendicular to a, so
// a x (v + b_lo) has no cancellation; and a_lo x b = mu (a_lo x a) + a_lo x v,
// the last term eps |a||v| relative to |a x v| = |a||v|.  iaa = 1/|a|^2 (0
// for a = 0) and (lx, ly, lz) = a_lo x a are per target.
__device__ __forceinline__ void projection_cross(float ax, float ay, float az, float iaa, float lx,
                                                 float ly, float lz, float bx, float by, float bz,
                                                 float mx, float my, float mz, float &wx, float &wy,
                                                 float &wz) {
  const float mu = fmaf(az, bz, fmaf(ay, by, ax * bx)) * iaa;
  const float vx = fmaf(-mu, ax, bx) + mx;
  const float vy = fmaf(-mu, ay, by) + my;
  const float vz = fmaf(-mu, az, bz) + mz;
  wx = fmaf(mu, lx, fmaf(ay, vz, -az * vy));
  wy = fmaf(mu, ly, fmaf(az, vx, -ax * vz));
  wz = fmaf(mu, lz, fmaf(ax, vy, -ay * vx));
}

// Near tile, shared-memory format: sp, sv, spl, svl = pos32, vor32, poslo,
// vorlo of the sources; tpl, tvl = poslo, vorlo of the targets.
// NX: alpha_i x alpha_j by cross_accurate (0) or projection_cross (1).
// UNI: every pair has sigma^2 = 2 hu; the sums are then in the units of
// kernel_scalars_uniform (qh, fh over sigma^2, Dp over 32).
template <bool DIFF, bool CHECK, int P, int R, int NSRC, int KERN, int NX = 0, int NU = 1,
          bool UNI = false>
__device__ __forceinline__ void tile_near(const float4 *__restrict__ sp,
                                          const float4 *__restrict__ sv,
                                          const float4 *__restrict__ spl,
                                          const float4 *__restrict__ svl, int g,
                                          const int (&skip)[R], const Target (&T)[R],
                                          const float4 (&tpl)[R], const float4 (&tvl)[R],
                                          Acc32 (&a)[R], float hu = 0.f) {
  const float s2u = 2.f * hu, c240 = -480.f * hu;
  float iaa[R], lcx[R], lcy[R], lcz[R];  // per target, for projection_cross
  if (NX) {
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const float aa = fmaf(T[r].ch, T[r].ch, fmaf(T[r].bh, T[r].bh, T[r].ah * T[r].ah));
      iaa[r] = aa > 0.f ? 1.0f / aa : 0.f;
      lcx[r] = fmaf(tvl[r].y, T[r].ch, -tvl[r].z * T[r].bh);
      lcy[r] = fmaf(tvl[r].z, T[r].ah, -tvl[r].x * T[r].ch);
      lcz[r] = fmaf(tvl[r].x, T[r].bh, -tvl[r].y * T[r].ah);
    }
  }
  // near tiles are a few percent of the work: inside the pair kernel no
  // unrolling (NU = 1) keeps the register budget of the far loop; the separate
  // near pass has its own and unrolls
#pragma unroll NU
  for (int k = 0; k < NSRC / P; ++k) {
    const int jj = g + P * k;
    const float4 p = sp[jj];
    const float4 s = sv[jj];
    const float4 pl = spl[jj];
    const float4 sl = svl[jj];
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const float dx = (T[r].xh - p.x) + (tpl[r].x - pl.x);
      const float dy = (T[r].yh - p.y) + (tpl[r].y - pl.y);
      const float dz = (T[r].zh - p.z) + (tpl[r].z - pl.z);
      const float r2 = fmaf(dz, dz, fmaf(dy, dy, dx * dx));
      const float sig2 = T[r].h + p.w;
      const float ri = rsqrtf(r2);
      float qh, fh, dp;
      if (KERN == KERNEL_GAUSSIAN) {
        gauss_scalars(sig2, r2, ri, qh, fh, dp);
      } else if (UNI) {
        const float w = rsqrtf(r2 + s2u);
        kernel_scalars_uniform(hu, c240, w, ri, r2, qh, fh, dp);
      } else {
        const float w = rsqrtf(r2 + sig2);
        kernel_scalars(sig2, w, ri, qh, fh, dp);
      }
      // velocity: alpha_j x d
      const float cx = fmaf(s.y, dz, -s.z * dy);
      const float cy = fmaf(s.z, dx, -s.x * dz);
      const float cz = fmaf(s.x, dy, -s.y * dx);
      // stretching: alpha_i x alpha_j from the hi/lo strengths
      float wx, wy, wz;
      if (NX)
        projection_cross(T[r].ah, T[r].bh, T[r].ch, iaa[r], lcx[r], lcy[r], lcz[r], s.x, s.y, s.z,
                         sl.x, sl.y, sl.z, wx, wy, wz);
      else
        cross_accurate(T[r].ah, T[r].bh, T[r].ch, tvl[r].x, tvl[r].y, tvl[r].z, s.x, s.y, s.z, sl.x,
                       sl.y, sl.z, wx, wy, wz);
      const float t = fmaf(dz, wz, fmaf(dy, wy, dx * wx));
      float ft = fh * t;
      if (CHECK) {
        const bool self = (jj == skip[r]);
        qh = self ? 0.f : qh;
        ft = self ? 0.f : ft;
        dp = self ? 0.f : dp;
      }
      a[r].ux = fmaf(qh, cx, a[r].ux);
      a[r].uy = fmaf(qh, cy, a[r].uy);
      a[r].uz = fmaf(qh, cz, a[r].uz);
      a[r].qx = fmaf(qh, wx, a[r].qx);
      a[r].qy = fmaf(qh, wy, a[r].qy);
      a[r].qz = fmaf(qh, wz, a[r].qz);
      a[r].gx = fmaf(ft, dx, a[r].gx);
      a[r].gy = fmaf(ft, dy, a[r].gy);
      a[r].gz = fmaf(ft, dz, a[r].gz);
      if (DIFF) {
        // delta = alpha_j - alpha_i from the hi/lo strengths
        const float ex = (s.x - T[r].ah) + (sl.x - tvl[r].x);
        const float ey = (s.y - T[r].bh) + (sl.y - tvl[r].y);
        const float ez = (s.z - T[r].ch) + (sl.z - tvl[r].z);
        a[r].ex = fmaf(dp, ex, a[r].ex);
        a[r].ey = fmaf(dp, ey, a[r].ey);
        a[r].ez = fmaf(dp, ez, a[r].ez);
        a[r].ev = fmaf(dp, T[r].v - s.w, a[r].ev);
      }
    }
  }
}

// ---- packed near tiles: two sources per FP32x2 instruction ----------------
// tile_near's arithmetic (hi/lo differences, the projection cross product)
// on a pair of sources per instruction, for the separate near pass, whose
// scalar loop is bound by instruction issue.  Shared-memory layout of a near
// tile, per source pair k = (a, b) = (2k, 2k+1):
//   n0[k] = (-xh_a, -xh_b, -yh_a, -yh_b)   n1[k] = (-zh_a, -zh_b, h_a, h_b)
//   n2[k] = (-xl_a, -xl_b, -yl_a, -yl_b)   n3[k] = (-zl_a, -zl_b, -v_a, -v_b)
//   n4[k] = (ax_a, ax_b, ay_a, ay_b)       n5[k] = (az_a, az_b, axl_a, axl_b)
//   n6[k] = (ayl_a, ayl_b, azl_a, azl_b)   n7[k] = (-ax_a, -ax_b, -ay_a, -ay_b)
//   n8[k] = (-az_a, -az_b)
// (h = s/2 squared, x hi/lo, alpha hi/lo, v the volume).  Positions, the
// volume and a second copy of the strength are stored negated so that no
// operand is negated in the loop; the target's quantities enter as broadcast
// pairs.  The loop accumulates -fh (as the packed far loop does).
struct NearT2 {
  float2 xh, yh, zh, xl, yl, zl;  // position hi, lo
  float2 h;                       // h_i
  float2 ax, ay, az;              // strength hi
  float2 nax, nay, naz;           // -strength hi
  float2 nlx, nly, nlz;           // -(alpha_lo x alpha_hi) of the target
  float2 iaa;                     // 1 / |alpha_hi|^2 (0 for alpha = 0)
  float2 nalx, naly, nalz;        // -strength lo
  float2 v;                       // volume
};

struct NearAcc2 {
  float2 ux, uy, uz;  // sum qh (alpha_j x d)
  float2 qx, qy, qz;  // sum qh (alpha_i x alpha_j)
  float2 gx, gy, gz;  // sum -fh t d
  float2 ex, ey, ez;  // sum Dp delta
  float2 ev;          // sum Dp (v_i - v_j)
};

// CHECK: the tile holds the target (skip = its index in the tile, whose pair
// contributes nothing).  UNI: every pair has sigma^2 = 2 hu (the sums in the
// units of kernel_scalars_uniform).
template <bool DIFF, bool CHECK, bool UNI, int RM, int NSRC>
__device__ __forceinline__ void tile_near_packed(const float4 *__restrict__ n0,
                                                 const float4 *__restrict__ n1,
                                                 const float4 *__restrict__ n2,
                                                 const float4 *__restrict__ n3,
                                                 const float4 *__restrict__ n4,
                                                 const float4 *__restrict__ n5,
                                                 const float4 *__restrict__ n6,
                                                 const float4 *__restrict__ n7,
                                                 const float2 *__restrict__ n8, int skip,
                                                 const NearT2 &T, float hu, NearAcc2 &a) {
  const float2 s2u = bc2(2.f * hu), h2 = bc2(hu), c240 = bc2(-480.f * hu);
#pragma unroll 1
  for (int k = 0; k < NSRC / 2; ++k) {
    const float4 A0 = n0[k], A1 = n1[k], A2 = n2[k], A3 = n3[k];
    const float2 dx = __fadd2_rn(__fadd2_rn(T.xh, make_float2(A0.x, A0.y)),
                                 __fadd2_rn(T.xl, make_float2(A2.x, A2.y)));
    const float2 dy = __fadd2_rn(__fadd2_rn(T.yh, make_float2(A0.z, A0.w)),
                                 __fadd2_rn(T.yl, make_float2(A2.z, A2.w)));
    const float2 dz = __fadd2_rn(__fadd2_rn(T.zh, make_float2(A1.x, A1.y)),
                                 __fadd2_rn(T.zl, make_float2(A3.x, A3.y)));
    const float2 r2 = __ffma2_rn(dz, dz, __ffma2_rn(dy, dy, __fmul2_rn(dx, dx)));
    const float2 ri = make_float2(rsqrtf(r2.x), rsqrtf(r2.y));
    float2 qh, nfh, dp;
    if (UNI) {
      // kernel_scalars_uniform in pairs, returning -fs
      const float2 sr = __fadd2_rn(r2, s2u);
      const float2 w = make_float2(rsqrtf(sr.x), rsqrtf(sr.y));
      const float2 ri2 = inv_r2<RM>(r2, ri);
      const float2 y = __fmul2_rn(w, w);
      const float2 u = __fmul2_rn(h2, y);
      const float2 v = __fmul2_rn(u, w);
      const float2 v2 = __fmul2_rn(v, v);
      dp = __fmul2_rn(__fmul2_rn(v2, v2), v);
      const float2 ph = __fmul2_rn(__ffma2_rn(u, y, y), ri);
      qh = __fmul2_rn(__ffma2_rn(c240, dp, ph), ri2);
      nfh = __fmul2_rn(__ffma2_rn(bc2(-80.f), dp, qh), ri2);
    } else {
      // kernel_scalars in pairs, returning -fh
      const float2 sig2 = __fadd2_rn(T.h, make_float2(A1.z, A1.w));
      const float2 sr = __fadd2_rn(r2, sig2);
      const float2 w = make_float2(rsqrtf(sr.x), rsqrtf(sr.y));
      const float2 w2 = __fmul2_rn(w, w);
      const float2 uu = __fmul2_rn(sig2, w2);
      const float2 v = __fmul2_rn(uu, w);
      const float2 v2 = __fmul2_rn(v, v);
      dp = __fmul2_rn(__fmul2_rn(v2, v2), v);
      const float2 zc = __fmul2_rn(dp, sig2);
      const float2 ph = __fmul2_rn(__fmul2_rn(__ffma2_rn(bc2(0.5f), uu, bc2(1.0f)), w2), ri);
      const float2 ri2 = __fmul2_rn(ri, ri);
      qh = __fmul2_rn(__fmul2_rn(__ffma2_rn(bc2(-7.5f), zc, ph), sig2), ri2);
      nfh = __fmul2_rn(__ffma2_rn(bc2(-2.5f), zc, qh), ri2);
    }
    const float4 A4 = n4[k], A5 = n5[k], A6 = n6[k], A7 = n7[k];
    const float2 B8 = n8[k];
    const float2 bx = make_float2(A4.x, A4.y), by = make_float2(A4.z, A4.w);
    const float2 bz = make_float2(A5.x, A5.y), mx = make_float2(A5.z, A5.w);
    const float2 my = make_float2(A6.x, A6.y), mz = make_float2(A6.z, A6.w);
    const float2 nbx = make_float2(A7.x, A7.y), nby = make_float2(A7.z, A7.w);
    // velocity: alpha_j x d
    const float2 cx = __ffma2_rn(by, dz, __fmul2_rn(B8, dy));
    const float2 cy = __ffma2_rn(bz, dx, __fmul2_rn(nbx, dz));
    const float2 cz = __ffma2_rn(bx, dy, __fmul2_rn(nby, dx));
    // stretching: alpha_i x alpha_j by projection_cross, with nmu = -mu
    const float2 nmu = __fmul2_rn(
        __ffma2_rn(T.naz, bz, __ffma2_rn(T.nay, by, __fmul2_rn(T.nax, bx))), T.iaa);
    const float2 vx = __fadd2_rn(__ffma2_rn(nmu, T.ax, bx), mx);
    const float2 vy = __fadd2_rn(__ffma2_rn(nmu, T.ay, by), my);
    const float2 vz = __fadd2_rn(__ffma2_rn(nmu, T.az, bz), mz);
    const float2 wx = __ffma2_rn(nmu, T.nlx, __ffma2_rn(T.ay, vz, __fmul2_rn(T.naz, vy)));
    const float2 wy = __ffma2_rn(nmu, T.nly, __ffma2_rn(T.az, vx, __fmul2_rn(T.nax, vz)));
    const float2 wz = __ffma2_rn(nmu, T.nlz, __ffma2_rn(T.ax, vy, __fmul2_rn(T.nay, vx)));
    const float2 t = __ffma2_rn(dz, wz, __ffma2_rn(dy, wy, __fmul2_rn(dx, wx)));
    float2 nft = __fmul2_rn(nfh, t);
    if (CHECK) {
      // the target's own pair contributes nothing
      if (2 * k == skip) qh.x = nft.x = dp.x = 0.f;
      if (2 * k + 1 == skip) qh.y = nft.y = dp.y = 0.f;
    }
    a.ux = __ffma2_rn(qh, cx, a.ux);
    a.uy = __ffma2_rn(qh, cy, a.uy);
    a.uz = __ffma2_rn(qh, cz, a.uz);
    a.qx = __ffma2_rn(qh, wx, a.qx);
    a.qy = __ffma2_rn(qh, wy, a.qy);
    a.qz = __ffma2_rn(qh, wz, a.qz);
    a.gx = __ffma2_rn(nft, dx, a.gx);
    a.gy = __ffma2_rn(nft, dy, a.gy);
    a.gz = __ffma2_rn(nft, dz, a.gz);
    if (DIFF) {
      // delta = alpha_j - alpha_i from the hi/lo strengths
      const float2 ex = __fadd2_rn(__fadd2_rn(bx, T.nax), __fadd2_rn(mx, T.nalx));
      const float2 ey = __fadd2_rn(__fadd2_rn(by, T.nay), __fadd2_rn(my, T.naly));
      const float2 ez = __fadd2_rn(__fadd2_rn(bz, T.naz), __fadd2_rn(mz, T.nalz));
      a.ex = __ffma2_rn(dp, ex, a.ex);
      a.ey = __ffma2_rn(dp, ey, a.ey);
      a.ez = __ffma2_rn(dp, ez, a.ez);
      a.ev = __ffma2_rn(dp, __fadd2_rn(T.v, make_float2(A3.z, A3.w)), a.ev);
    }
  }
}

__device__ __forceinline__ float box_gap2(float4 alo, float4 ahi, float4 blo, float4 bhi) {
  const float gx = fmaxf(0.f, fmaxf(alo.x - bhi.x, blo.x - ahi.x));
  const float gy = fmaxf(0.f, fmaxf(alo.y - bhi.y, blo.y - ahi.y));
  const float gz = fmaxf(0.f, fmaxf(alo.z - bhi.z, blo.z - ahi.z));
  return gx * gx + gy * gy + gz * gz;
}

// Far formulation allowed: box gap positive and at least max(near radius,
// half-diagonal of the source box).
__device__ __forceinline__ bool far_tiles(float gap2, float4 slo, float4 shi, float near2) {
  const float ex = shi.x - slo.x, ey = shi.y - slo.y, ez = shi.z - slo.z;
  const float half_diag2 = 0.25f * (ex * ex + ey * ey + ez * ez);
  return gap2 > 0.f && gap2 >= near2 && gap2 >= half_diag2;
}

// Threads per target P > 1 split a tile's sources (R = 1); targets per thread
// R > 1 reuse each source loaded from shared memory for R targets (P = 1);
// PK > 0: the far path processes two sources per FP32x2 instruction (P = R =
// 1), taking 1/rho^2 on uniform-radius tiles from the MUFU reciprocal (PK = 1)
// or from rsqrt squared (PK = 2).
// MINB: blocks per SM the register allocation is bounded for (occupancy).
// KERN: the smoothing kernel (SmoothingKernel); the uniform-radius
// specialisation exists for the high-order kernel only.
// SPLIT: near tile pairs were computed by pairs_f32_near_kernel before this
// launch; they are skipped here and each item adds its near sums (if any).
template <int TB, int P, int R, int U, bool DIFF, int MINB, int PK, int KERN, bool SPLIT = false>
__global__ void __launch_bounds__(TB, MINB)
    pairs_f32_kernel(const WorkItem *__restrict__ items, int n_items,
                     const SegDesc *__restrict__ segs, int *__restrict__ next_item) {
  static_assert(PK == 0 || (P == 1 && R == 1), "the packed far path has one target per thread");
  constexpr int TG = TB / P;   // targets per block and per target row r
  constexpr int TPB = TG * R;  // targets per block
  constexpr int FQ = PK ? TB / 2 : 1;
  // two-stage tile ring in dynamic shared memory (pair_f32_smem_bytes):
  // sp, sv, spl, svl [2][TB] (pos32, vor32, poslo, vorlo as staged), then
  // the packed far format fq [5][2][FQ] float4 and fz [2][FQ] float2
  extern __shared__ float4 smem_f32[];
  float4 *const sp = smem_f32;
  float4 *const sv = sp + 2 * TB;
  float4 *const spl = sv + 2 * TB;
  float4 *const svl = spl + 2 * TB;
  float4 *const fq = svl + 2 * TB;
  float2 *const fz = reinterpret_cast<float2 *>(fq + 10 * FQ);
  __shared__ int s_item, s_last;
  const int tid = threadIdx.x;
  const int g = tid % P;
  const int lt = tid / P;
  const double A = kInv4Pi;

  for (;;) {
    if (tid == 0) s_item = atomicAdd(next_item, 1);
    __syncthreads();
    const int it = s_item;
    __syncthreads();
    if (it >= n_items) break;

    const WorkItem w = items[it];
    const SegDesc sg = segs[w.seg];
    const double cnu = 15.0 * sg.nu * A;
    int ti[R];
    bool valid[R];
    Target T[R];
    float al[R], bl[R], cl[R];  // strength lo: the folds use alpha_i = hi + lo in FP64
    double ou[R][3], oa[R][3];
#pragma unroll
    for (int r = 0; r < R; ++r) {
      ti[r] = w.t0 + lt + r * TG;
      valid[r] = ti[r] < sg.n;
      float4 a = make_float4(0.f, 0.f, 0.f, 1.f), b = make_float4(0.f, 0.f, 0.f, 0.f), d = b;
      if (valid[r]) {
        a = __ldg(sg.pos32 + ti[r]);
        b = __ldg(sg.vor32 + ti[r]);
        d = __ldg(sg.vorlo + ti[r]);
      }
      T[r].xh = a.x; T[r].yh = a.y; T[r].zh = a.z; T[r].h = a.w;
      T[r].ah = b.x; T[r].bh = b.y; T[r].ch = b.z; T[r].v = b.w;
      al[r] = d.x; bl[r] = d.y; cl[r] = d.z;
#pragma unroll
      for (int k = 0; k < 3; ++k) ou[r][k] = oa[r][k] = 0.0;
    }

    // box of the target tile: union of the source-tile boxes it covers (w:
    // range of h)
    float4 tlo = __ldg(sg.boxes + 2 * (w.t0 / TB));
    float4 thi = __ldg(sg.boxes + 2 * (w.t0 / TB) + 1);
#pragma unroll
    for (int q = 1; q < (TPB + TB - 1) / TB; ++q) {
      if (w.t0 + q * TB < sg.n) {
        const float4 l2 = __ldg(sg.boxes + 2 * (w.t0 / TB + q));
        const float4 h2 = __ldg(sg.boxes + 2 * (w.t0 / TB + q) + 1);
        tlo = make_float4(fminf(tlo.x, l2.x), fminf(tlo.y, l2.y), fminf(tlo.z, l2.z),
                          fminf(tlo.w, l2.w));
        thi = make_float4(fmaxf(thi.x, h2.x), fmaxf(thi.y, h2.y), fmaxf(thi.z, h2.z),
                          fmaxf(thi.w, h2.w));
      }
    }

    const int ntiles = (w.s1 - w.s0 + TB - 1) / TB;
    stage_source(sg, w.s0 + tid, w.s1, sp + tid, sv + tid, spl + tid, svl + tid);
    for (int t = 0; t < ntiles; ++t) {
      const int buf = t & 1;
      const int ts = w.s0 + t * TB;
      const float4 slo = __ldg(sg.boxes + 2 * (ts / TB));
      const float4 shi = __ldg(sg.boxes + 2 * (ts / TB) + 1);
      const bool diag = (ts < w.t0 + TPB) && (w.t0 < ts + TB);
      const float gap2 = box_gap2(tlo, thi, slo, shi);
      const bool near = diag || !far_tiles(gap2, slo, shi, sg.near2);
      // every pair at rho >= 6 sigma: the Z-free far field (w of a box = the
      // range of h = s^2/2, so thi.w + shi.w is the largest sigma^2)
      // Gaussian kernel, every pair at rho >= 7 sigma: its far field (gauss_far),
      // taken by the series branches of the far loops
      const bool gfar = KERN == KERNEL_GAUSSIAN && !near && gap2 >= 49.f * (thi.w + shi.w);
      const bool nz = (KERN == KERNEL_HIGHORDER && !near && gap2 >= 36.f * (thi.w + shi.w)) || gfar;
      // every pair at rho >= 16 sigma: the Z-free field by its series
      const bool ser = (nz && gap2 >= 256.f * (thi.w + shi.w)) || gfar;
      // one smoothing radius over both tiles
      const bool uni = KERN == KERNEL_HIGHORDER && tlo.w == thi.w && slo.w == shi.w && tlo.w == slo.w;
      const float cx = 0.5f * (slo.x + shi.x), cy = 0.5f * (slo.y + shi.y),
                  cz = 0.5f * (slo.z + shi.z);
      // this thread's own slot of the tile: wait for its copies, then rewrite
      // it in the far format (or the packed one); the barrier publishes the
      // tile and retires the previous one, whose buffer the next copies reuse
      wait_staged();
      if (!near) {
        const float4 p0 = sp[buf * TB + tid], p1 = sv[buf * TB + tid];
        const float px = p0.x - cx, py = p0.y - cy, pz = p0.z - cz;
        const float bx = fmaf(p1.y, pz, -p1.z * py), by = fmaf(p1.z, px, -p1.x * pz),
                    bz = fmaf(p1.x, py, -p1.y * px);
        if (PK) {
          const int k = tid >> 1, hf = tid & 1;
          float *q0 = reinterpret_cast<float *>(fq + (0 * 2 + buf) * FQ + k);
          float *q1 = reinterpret_cast<float *>(fq + (1 * 2 + buf) * FQ + k);
          float *q2 = reinterpret_cast<float *>(fq + (2 * 2 + buf) * FQ + k);
          float *q3 = reinterpret_cast<float *>(fq + (3 * 2 + buf) * FQ + k);
          float *q4 = reinterpret_cast<float *>(fq + (4 * 2 + buf) * FQ + k);
          float *q5 = reinterpret_cast<float *>(fz + buf * FQ + k);
          q0[hf] = -px;
          q0[2 + hf] = -py;
          q1[hf] = -pz;
          q1[2 + hf] = p0.w;
          q2[hf] = p1.x;
          q2[2 + hf] = p1.y;
          q3[hf] = p1.z;
          q3[2 + hf] = p1.w;
          q4[hf] = bx;
          q4[2 + hf] = by;
          q5[hf] = bz;
        } else {
          sp[buf * TB + tid] = make_float4(px, py, pz, p0.w);
          spl[buf * TB + tid] = make_float4(bx, by, bz, 0.f);
        }
      }
      __syncthreads();
      if (t + 1 < ntiles)
        stage_source(sg, ts + TB + tid, w.s1, sp + (buf ^ 1) * TB + tid, sv + (buf ^ 1) * TB + tid,
                     spl + (buf ^ 1) * TB + tid, svl + (buf ^ 1) * TB + tid);
      Acc32 a[R];
#pragma unroll
      for (int r = 0; r < R; ++r) a[r] = Acc32{0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
      double ax[R], ay[R], az[R];
#pragma unroll
      for (int r = 0; r < R; ++r) {
        ax[r] = (double)T[r].ah + (double)al[r];
        ay[r] = (double)T[r].bh + (double)bl[r];
        az[r] = (double)T[r].ch + (double)cl[r];
      }
      if (!near && PK) {
        Target2 T2;
        const float fx = T[0].xh - cx, fy = T[0].yh - cy, fzz = T[0].zh - cz;
        T2.x = bc2(fx);
        T2.y = bc2(fy);
        T2.z = bc2(fzz);
        T2.h = bc2(T[0].h);
        T2.na = bc2(-T[0].ah);
        T2.nb = bc2(-T[0].bh);
        T2.nc = bc2(-T[0].ch);
        T2.gx = bc2(fmaf(fy, T[0].ch, -fzz * T[0].bh));
        T2.gy = bc2(fmaf(fzz, T[0].ah, -fx * T[0].ch));
        T2.gz = bc2(fmaf(fx, T[0].bh, -fy * T[0].ah));
        Acc2 b;
        b.wx = b.wy = b.wz = b.qx = b.qy = b.qz = b.gx = b.gy = b.gz = make_float2(0.f, 0.f);
        b.ex = b.ey = b.ez = b.ev = make_float2(0.f, 0.f);
        const float4 *f0 = fq + buf * FQ, *f1 = fq + (2 + buf) * FQ, *f2 = fq + (4 + buf) * FQ,
                     *f3 = fq + (6 + buf) * FQ, *f4 = fq + (8 + buf) * FQ;
        const float2 *f5 = fz + buf * FQ;
        if (ser && uni)
          tile_far_packed<DIFF, true, PK, TB, U, KERN, true, true>(f0, f1, f2, f3, f4, f5, T2, slo.w, b);
        else if (ser)
          tile_far_packed<DIFF, false, PK, TB, U, KERN, true, true>(f0, f1, f2, f3, f4, f5, T2, 0.f, b);
        else if (nz && uni)
          tile_far_packed<DIFF, true, PK, TB, U, KERN, true>(f0, f1, f2, f3, f4, f5, T2, slo.w, b);
        else if (nz)
          tile_far_packed<DIFF, false, PK, TB, U, KERN, true>(f0, f1, f2, f3, f4, f5, T2, 0.f, b);
        else if (uni)
          tile_far_packed<DIFF, true, PK, TB, U, KERN, false>(f0, f1, f2, f3, f4, f5, T2, slo.w, b);
        else
          tile_far_packed<DIFF, false, PK, TB, U, KERN, false>(f0, f1, f2, f3, f4, f5, T2, 0.f, b);
        const double s2 = uni ? 2.0 * (double)slo.w : 1.0;
        const double As2 = A * s2;
        const double cd = uni ? 32.0 * cnu : cnu;
        const double Qx = As2 * (b.qx.x + b.qx.y), Qy = As2 * (b.qy.x + b.qy.y),
                     Qz = As2 * (b.qz.x + b.qz.y);
        const double xp = fx, yp = fy, zp = fzz;
        ou[0][0] += (Qy * zp - Qz * yp) - As2 * (b.wx.x + b.wx.y);
        ou[0][1] += (Qz * xp - Qx * zp) - As2 * (b.wy.x + b.wy.y);
        ou[0][2] += (Qx * yp - Qy * xp) - As2 * (b.wz.x + b.wz.y);
        oa[0][0] += (ay[0] * Qz - az[0] * Qy) - 3.0 * As2 * (b.gx.x + b.gx.y);
        oa[0][1] += (az[0] * Qx - ax[0] * Qz) - 3.0 * As2 * (b.gy.x + b.gy.y);
        oa[0][2] += (ax[0] * Qy - ay[0] * Qx) - 3.0 * As2 * (b.gz.x + b.gz.y);
        if (DIFF && !nz) {
          const double v = T[0].v, ev = b.ev.x + b.ev.y;
          oa[0][0] += cd * (v * (b.ex.x + b.ex.y) - ev * ax[0]);
          oa[0][1] += cd * (v * (b.ey.x + b.ey.y) - ev * ay[0]);
          oa[0][2] += cd * (v * (b.ez.x + b.ez.y) - ev * az[0]);
        }
      } else if (!near) {
        FarTarget F[R];
#pragma unroll
        for (int r = 0; r < R; ++r) {
          F[r].x = T[r].xh - cx;
          F[r].y = T[r].yh - cy;
          F[r].z = T[r].zh - cz;
          F[r].gx = fmaf(F[r].y, T[r].ch, -F[r].z * T[r].bh);
          F[r].gy = fmaf(F[r].z, T[r].ah, -F[r].x * T[r].ch);
          F[r].gz = fmaf(F[r].x, T[r].bh, -F[r].y * T[r].ah);
        }
        const float4 *ta = sp + buf * TB, *tb = sv + buf * TB, *tc = spl + buf * TB;
        if (ser && uni)
          tile_far<DIFF, true, P, R, TB, U, KERN, true, true>(ta, tb, tc, g, T, F, slo.w, a);
        else if (ser)
          tile_far<DIFF, false, P, R, TB, U, KERN, true, true>(ta, tb, tc, g, T, F, 0.f, a);
        else if (nz && uni)
          tile_far<DIFF, true, P, R, TB, U, KERN, true>(ta, tb, tc, g, T, F, slo.w, a);
        else if (nz)
          tile_far<DIFF, false, P, R, TB, U, KERN, true>(ta, tb, tc, g, T, F, 0.f, a);
        else if (uni)
          tile_far<DIFF, true, P, R, TB, U, KERN, false>(ta, tb, tc, g, T, F, slo.w, a);
        else
          tile_far<DIFF, false, P, R, TB, U, KERN, false>(ta, tb, tc, g, T, F, 0.f, a);
        // undo the uniform-radius scaling: qh = sigma^2 qs, fh = sigma^2 fs, Dp = 32 ds
        const double s2 = uni ? 2.0 * (double)slo.w : 1.0;
        const double As2 = A * s2;
        const double cd = uni ? 32.0 * cnu : cnu;
#pragma unroll
        for (int r = 0; r < R; ++r) {
          const double Qx = As2 * a[r].qx, Qy = As2 * a[r].qy, Qz = As2 * a[r].qz;
          const double xp = F[r].x, yp = F[r].y, zp = F[r].z;
          // u = A sigma^2 (Q x x' - W)
          ou[r][0] += (Qy * zp - Qz * yp) - As2 * a[r].ux;
          ou[r][1] += (Qz * xp - Qx * zp) - As2 * a[r].uy;
          ou[r][2] += (Qx * yp - Qy * xp) - As2 * a[r].uz;
          oa[r][0] += (ay[r] * Qz - az[r] * Qy) + 3.0 * As2 * a[r].gx;
          oa[r][1] += (az[r] * Qx - ax[r] * Qz) + 3.0 * As2 * a[r].gy;
          oa[r][2] += (ax[r] * Qy - ay[r] * Qx) + 3.0 * As2 * a[r].gz;
          if (DIFF && !nz) {
            const double v = T[r].v;
            oa[r][0] += cd * (v * a[r].ex - (double)a[r].ev * ax[r]);
            oa[r][1] += cd * (v * a[r].ey - (double)a[r].ev * ay[r]);
            oa[r][2] += cd * (v * a[r].ez - (double)a[r].ev * az[r]);
          }
        }
      } else if (!SPLIT) {
        int skip[R];
        float4 tpl[R], tvl[R];
#pragma unroll
        for (int r = 0; r < R; ++r) {
          skip[r] = ti[r] - ts;
          tpl[r] = valid[r] ? __ldg(sg.poslo + ti[r]) : make_float4(0.f, 0.f, 0.f, 0.f);
          tvl[r] = valid[r] ? __ldg(sg.vorlo + ti[r]) : make_float4(0.f, 0.f, 0.f, 0.f);
        }
        if (diag)
          tile_near<DIFF, true, P, R, TB, KERN>(sp + buf * TB, sv + buf * TB, spl + buf * TB,
                                          svl + buf * TB, g, skip, T, tpl, tvl, a);
        else
          tile_near<DIFF, false, P, R, TB, KERN>(sp + buf * TB, sv + buf * TB, spl + buf * TB,
                                           svl + buf * TB, g, skip, T, tpl, tvl, a);
#pragma unroll
        for (int r = 0; r < R; ++r) {
          ou[r][0] += A * a[r].ux;
          ou[r][1] += A * a[r].uy;
          ou[r][2] += A * a[r].uz;
          oa[r][0] += A * a[r].qx + 3.0 * A * a[r].gx;
          oa[r][1] += A * a[r].qy + 3.0 * A * a[r].gy;
          oa[r][2] += A * a[r].qz + 3.0 * A * a[r].gz;
          if (DIFF) {
            const double v = T[r].v;
            oa[r][0] += cnu * (v * a[r].ex + (double)a[r].ev * ax[r]);
            oa[r][1] += cnu * (v * a[r].ey + (double)a[r].ev * ay[r]);
            oa[r][2] += cnu * (v * a[r].ez + (double)a[r].ev * az[r]);
          }
        }
      }
    }

    if (P > 1) {
#pragma unroll
      for (int off = 1; off < P; off <<= 1) {
#pragma unroll
        for (int k = 0; k < 3; ++k) {
          ou[0][k] += __shfl_xor_sync(0xffffffffu, ou[0][k], off);
          oa[0][k] += __shfl_xor_sync(0xffffffffu, oa[0][k], off);
        }
      }
    }

    if (SPLIT) {
      const size_t fi = (size_t)(w.t0 / TPB) * (size_t)sg.nchunks + (size_t)w.chunk;
      if (sg.near_flag[fi] && g == 0) {
        const double *ns = sg.near_partial + fi * 6 * (size_t)TPB;
#pragma unroll
        for (int r = 0; r < R; ++r) {
          const int q = ti[r] - w.t0;
#pragma unroll
          for (int k = 0; k < 3; ++k) {
            ou[r][k] += ns[(size_t)k * TPB + q];
            oa[r][k] += ns[(size_t)(3 + k) * TPB + q];
          }
        }
      }
    }
    const ItemOut o = item_out(sg, w.t0, w.chunk, TPB);
    if (g == 0) {
#pragma unroll
      for (int r = 0; r < R; ++r) {
        if (!valid[r]) continue;
        double *out = o.base + (ti[r] - w.t0);
        out[0] = ou[r][0];
        out[o.stride] = ou[r][1];
        out[2 * o.stride] = ou[r][2];
        out[3 * o.stride] = oa[r][0];
        out[4 * o.stride] = oa[r][1];
        out[5 * o.stride] = oa[r][2];
      }
    }
    if (sg.nchunks > 1) finish_item<TB>(sg, w.t0, TPB, &s_last);
  }
}

// The near pass of a split tiling: the same work items, only their near tile
// pairs (the same box test as pairs_f32_kernel), each staged and computed
// with the accurate near formulation; an item's sums go to its near slot and
// its flag says whether it had any.  It runs before the far pass, which adds
// the flagged slots to its own sums.
// PKN: the near tiles two sources per FP32x2 instruction (tile_near_packed;
// P = R = 1), with 1/rho^2 on uniform-radius tiles as packed mode RM gives it.
template <int TB, int P, int R, bool DIFF, int MINB, int KERN, int NX, int NU = 2, int PKN = 0,
          int RM = 2>
__global__ void __launch_bounds__(TB, MINB)
    pairs_f32_near_kernel(const WorkItem *__restrict__ items, int n_items,
                          const SegDesc *__restrict__ segs, int *__restrict__ next_item) {
  static_assert(PKN == 0 || (P == 1 && R == 1), "the packed near pass has one target per thread");
  constexpr int TG = TB / P;
  constexpr int TPB = TG * R;
  constexpr int NQ = PKN ? TB / 2 : 1;
  __shared__ float4 sp[TB], sv[TB], spl[TB], svl[TB];
  __shared__ float4 nq[8][NQ];  // packed near format n0..n7
  __shared__ float2 n8[NQ];
  __shared__ int s_item;
  const int tid = threadIdx.x;
  const int g = tid % P;
  const int lt = tid / P;
  const double A = kInv4Pi;

  for (;;) {
    if (tid == 0) s_item = atomicAdd(next_item, 1);
    __syncthreads();
    const int it = s_item;
    __syncthreads();
    if (it >= n_items) break;

    const WorkItem w = items[it];
    const SegDesc sg = segs[w.seg];
    const double cnu = 15.0 * sg.nu * A;
    int ti[R];
    bool valid[R];
    Target T[R];
    float4 tpl[R], tvl[R];
    double ou[R][3], oa[R][3], ax[R], ay[R], az[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
      ti[r] = w.t0 + lt + r * TG;
      valid[r] = ti[r] < sg.n;
      float4 a = make_float4(0.f, 0.f, 0.f, 1.f), b = make_float4(0.f, 0.f, 0.f, 0.f);
      tpl[r] = tvl[r] = make_float4(0.f, 0.f, 0.f, 0.f);
      if (valid[r]) {
        a = __ldg(sg.pos32 + ti[r]);
        b = __ldg(sg.vor32 + ti[r]);
        tpl[r] = __ldg(sg.poslo + ti[r]);
        tvl[r] = __ldg(sg.vorlo + ti[r]);
      }
      T[r].xh = a.x; T[r].yh = a.y; T[r].zh = a.z; T[r].h = a.w;
      T[r].ah = b.x; T[r].bh = b.y; T[r].ch = b.z; T[r].v = b.w;
      ax[r] = (double)b.x + (double)tvl[r].x;
      ay[r] = (double)b.y + (double)tvl[r].y;
      az[r] = (double)b.z + (double)tvl[r].z;
#pragma unroll
      for (int k = 0; k < 3; ++k) ou[r][k] = oa[r][k] = 0.0;
    }
    float4 tlo = __ldg(sg.boxes + 2 * (w.t0 / TB));
    float4 thi = __ldg(sg.boxes + 2 * (w.t0 / TB) + 1);
#pragma unroll
    for (int q = 1; q < (TPB + TB - 1) / TB; ++q) {
      if (w.t0 + q * TB < sg.n) {
        const float4 l2 = __ldg(sg.boxes + 2 * (w.t0 / TB + q));
        const float4 h2 = __ldg(sg.boxes + 2 * (w.t0 / TB + q) + 1);
        tlo = make_float4(fminf(tlo.x, l2.x), fminf(tlo.y, l2.y), fminf(tlo.z, l2.z),
                          fminf(tlo.w, l2.w));
        thi = make_float4(fmaxf(thi.x, h2.x), fmaxf(thi.y, h2.y), fmaxf(thi.z, h2.z),
                          fmaxf(thi.w, h2.w));
      }
    }

    // the target as broadcast pairs for the packed loop
    NearT2 T2;
    if (PKN) {
      const float aa = fmaf(T[0].ch, T[0].ch, fmaf(T[0].bh, T[0].bh, T[0].ah * T[0].ah));
      T2.xh = bc2(T[0].xh); T2.yh = bc2(T[0].yh); T2.zh = bc2(T[0].zh);
      T2.xl = bc2(tpl[0].x); T2.yl = bc2(tpl[0].y); T2.zl = bc2(tpl[0].z);
      T2.h = bc2(T[0].h);
      T2.ax = bc2(T[0].ah); T2.ay = bc2(T[0].bh); T2.az = bc2(T[0].ch);
      T2.nax = bc2(-T[0].ah); T2.nay = bc2(-T[0].bh); T2.naz = bc2(-T[0].ch);
      T2.nlx = bc2(-fmaf(tvl[0].y, T[0].ch, -tvl[0].z * T[0].bh));
      T2.nly = bc2(-fmaf(tvl[0].z, T[0].ah, -tvl[0].x * T[0].ch));
      T2.nlz = bc2(-fmaf(tvl[0].x, T[0].bh, -tvl[0].y * T[0].ah));
      T2.iaa = bc2(aa > 0.f ? 1.0f / aa : 0.f);
      T2.nalx = bc2(-tvl[0].x); T2.naly = bc2(-tvl[0].y); T2.nalz = bc2(-tvl[0].z);
      T2.v = bc2(T[0].v);
    }

    bool any = false;
    const int ntiles = (w.s1 - w.s0 + TB - 1) / TB;
    for (int t = 0; t < ntiles; ++t) {
      const int ts = w.s0 + t * TB;
      const float4 slo = __ldg(sg.boxes + 2 * (ts / TB));
      const float4 shi = __ldg(sg.boxes + 2 * (ts / TB) + 1);
      const bool diag = (ts < w.t0 + TPB) && (w.t0 < ts + TB);
      const bool near = diag || !far_tiles(box_gap2(tlo, thi, slo, shi), slo, shi, sg.near2);
      if (!near) continue;  // block-uniform
      any = true;
      __syncthreads();  // the previous near tile is no longer read
      stage_source(sg, ts + tid, w.s1, sp + tid, sv + tid, spl + tid, svl + tid);
      wait_staged();
      if (PKN) {
        // this thread's own slot, rewritten in the packed near format
        const float4 p0 = sp[tid], p1 = sv[tid], p2 = spl[tid], p3 = svl[tid];
        const int k = tid >> 1, hf = tid & 1;
        float *q0 = reinterpret_cast<float *>(&nq[0][k]);
        float *q1 = reinterpret_cast<float *>(&nq[1][k]);
        float *q2 = reinterpret_cast<float *>(&nq[2][k]);
        float *q3 = reinterpret_cast<float *>(&nq[3][k]);
        float *q4 = reinterpret_cast<float *>(&nq[4][k]);
        float *q5 = reinterpret_cast<float *>(&nq[5][k]);
        float *q6 = reinterpret_cast<float *>(&nq[6][k]);
        float *q7 = reinterpret_cast<float *>(&nq[7][k]);
        float *q8 = reinterpret_cast<float *>(&n8[k]);
        q0[hf] = -p0.x; q0[2 + hf] = -p0.y;
        q1[hf] = -p0.z; q1[2 + hf] = p0.w;
        q2[hf] = -p2.x; q2[2 + hf] = -p2.y;
        q3[hf] = -p2.z; q3[2 + hf] = -p1.w;
        q4[hf] = p1.x;  q4[2 + hf] = p1.y;
        q5[hf] = p1.z;  q5[2 + hf] = p3.x;
        q6[hf] = p3.y;  q6[2 + hf] = p3.z;
        q7[hf] = -p1.x; q7[2 + hf] = -p1.y;
        q8[hf] = -p1.z;
      }
      __syncthreads();
      if (PKN) {
        const bool uni =
            KERN == KERNEL_HIGHORDER && tlo.w == thi.w && slo.w == shi.w && tlo.w == slo.w;
        NearAcc2 b;
        b.ux = b.uy = b.uz = b.qx = b.qy = b.qz = b.gx = b.gy = b.gz = make_float2(0.f, 0.f);
        b.ex = b.ey = b.ez = b.ev = make_float2(0.f, 0.f);
        const int skip = ti[0] - ts;
        if (diag && uni)
          tile_near_packed<DIFF, true, true, RM, TB>(nq[0], nq[1], nq[2], nq[3], nq[4], nq[5], nq[6],
                                                     nq[7], n8, skip, T2, slo.w, b);
        else if (diag)
          tile_near_packed<DIFF, true, false, RM, TB>(nq[0], nq[1], nq[2], nq[3], nq[4], nq[5], nq[6],
                                                      nq[7], n8, skip, T2, 0.f, b);
        else if (uni)
          tile_near_packed<DIFF, false, true, RM, TB>(nq[0], nq[1], nq[2], nq[3], nq[4], nq[5], nq[6],
                                                      nq[7], n8, skip, T2, slo.w, b);
        else
          tile_near_packed<DIFF, false, false, RM, TB>(nq[0], nq[1], nq[2], nq[3], nq[4], nq[5],
                                                       nq[6], nq[7], n8, skip, T2, 0.f, b);
        // undo the uniform-radius scaling; b.g holds -fh t d
        const double As2 = uni ? A * 2.0 * (double)slo.w : A;
        const double cd = uni ? 32.0 * cnu : cnu;
        ou[0][0] += As2 * ((double)b.ux.x + (double)b.ux.y);
        ou[0][1] += As2 * ((double)b.uy.x + (double)b.uy.y);
        ou[0][2] += As2 * ((double)b.uz.x + (double)b.uz.y);
        oa[0][0] += As2 * (((double)b.qx.x + (double)b.qx.y) - 3.0 * ((double)b.gx.x + (double)b.gx.y));
        oa[0][1] += As2 * (((double)b.qy.x + (double)b.qy.y) - 3.0 * ((double)b.gy.x + (double)b.gy.y));
        oa[0][2] += As2 * (((double)b.qz.x + (double)b.qz.y) - 3.0 * ((double)b.gz.x + (double)b.gz.y));
        if (DIFF) {
          const double v = T[0].v, ev = (double)b.ev.x + (double)b.ev.y;
          oa[0][0] += cd * (v * ((double)b.ex.x + (double)b.ex.y) + ev * ax[0]);
          oa[0][1] += cd * (v * ((double)b.ey.x + (double)b.ey.y) + ev * ay[0]);
          oa[0][2] += cd * (v * ((double)b.ez.x + (double)b.ez.y) + ev * az[0]);
        }
        continue;
      }
      int skip[R];
      Acc32 a[R];
#pragma unroll
      for (int r = 0; r < R; ++r) {
        skip[r] = ti[r] - ts;
        a[r] = Acc32{0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
      }
      // one smoothing radius over both tiles: the uniform-radius scalars
      const bool uni = KERN == KERNEL_HIGHORDER && tlo.w == thi.w && slo.w == shi.w && tlo.w == slo.w;
      if (diag && uni)
        tile_near<DIFF, true, P, R, TB, KERN, NX, NU, true>(sp, sv, spl, svl, g, skip, T, tpl, tvl, a,
                                                            slo.w);
      else if (diag)
        tile_near<DIFF, true, P, R, TB, KERN, NX, NU>(sp, sv, spl, svl, g, skip, T, tpl, tvl, a);
      else if (uni)
        tile_near<DIFF, false, P, R, TB, KERN, NX, NU, true>(sp, sv, spl, svl, g, skip, T, tpl, tvl,
                                                             a, slo.w);
      else
        tile_near<DIFF, false, P, R, TB, KERN, NX, NU>(sp, sv, spl, svl, g, skip, T, tpl, tvl, a);
      // undo the uniform-radius scaling: qh = sigma^2 qs, fh = sigma^2 fs, Dp = 32 ds
      const double As2 = uni ? A * 2.0 * (double)slo.w : A;
      const double cd = uni ? 32.0 * cnu : cnu;
#pragma unroll
      for (int r = 0; r < R; ++r) {
        ou[r][0] += As2 * a[r].ux;
        ou[r][1] += As2 * a[r].uy;
        ou[r][2] += As2 * a[r].uz;
        oa[r][0] += As2 * a[r].qx + 3.0 * As2 * a[r].gx;
        oa[r][1] += As2 * a[r].qy + 3.0 * As2 * a[r].gy;
        oa[r][2] += As2 * a[r].qz + 3.0 * As2 * a[r].gz;
        if (DIFF) {
          const double v = T[r].v;
          oa[r][0] += cd * (v * a[r].ex + (double)a[r].ev * ax[r]);
          oa[r][1] += cd * (v * a[r].ey + (double)a[r].ev * ay[r]);
          oa[r][2] += cd * (v * a[r].ez + (double)a[r].ev * az[r]);
        }
      }
    }

    const size_t fi = (size_t)(w.t0 / TPB) * (size_t)sg.nchunks + (size_t)w.chunk;
    if (any) {
      if (P > 1) {
#pragma unroll
        for (int off = 1; off < P; off <<= 1) {
#pragma unroll
          for (int k = 0; k < 3; ++k) {
            ou[0][k] += __shfl_xor_sync(0xffffffffu, ou[0][k], off);
            oa[0][k] += __shfl_xor_sync(0xffffffffu, oa[0][k], off);
          }
        }
      }
      if (g == 0) {
        double *ns = sg.near_partial + fi * 6 * (size_t)TPB;
#pragma unroll
        for (int r = 0; r < R; ++r) {
          if (!valid[r]) continue;
          const int q = ti[r] - w.t0;
#pragma unroll
          for (int k = 0; k < 3; ++k) {
            ns[(size_t)k * TPB + q] = ou[r][k];
            ns[(size_t)(3 + k) * TPB + q] = oa[r][k];
          }
        }
      }
    }
    if (tid == 0) sg.near_flag[fi] = any ? 1 : 0;
  }
}

using KernelFn = void (*)(const WorkItem *, int, const SegDesc *, int *);

// The kernels of a tiling: the pair kernel (the far pass when split) and,
// for split tilings, the near pass.
struct Kernels {
  KernelFn main = nullptr;
  KernelFn near = nullptr;
};

template <bool DIFF>
Kernels select_highorder(const PairConfig &c) {
#define PAWAN_F32_CASE_PK(TB_, P_, R_, U_, MINB_, PK_)                                   \
  PAWAN_F32_CASE_K(TB_, P_, R_, U_, MINB_, PK_, KERNEL_HIGHORDER)
#define PAWAN_F32_MATCH(TB_, P_, R_, U_, MINB_, PK_)                                     \
  (c.tb == TB_ && c.p == P_ && c.r == R_ && c.unroll == U_ && c.packed == PK_ &&         \
   (c.minb == MINB_ || (c.minb == 0 && MINB_ == (TB_ <= 128 ? 4 : 2))))
#define PAWAN_F32_CASE_K(TB_, P_, R_, U_, MINB_, PK_, KERN_)                             \
  if (c.split == 0 && PAWAN_F32_MATCH(TB_, P_, R_, U_, MINB_, PK_))                       \
    return Kernels{&pairs_f32_kernel<TB_, P_, R_, U_, DIFF, MINB_, PK_, KERN_>, nullptr};
#define PAWAN_F32_CASE_SPLIT(TB_, U_, MINB_, PK_)                                        \
  if (c.split == 1 && PAWAN_F32_MATCH(TB_, 1, 1, U_, MINB_, PK_))                         \
    return Kernels{&pairs_f32_kernel<TB_, 1, 1, U_, DIFF, MINB_, PK_, KERNEL_HIGHORDER, true>, \
                   &pairs_f32_near_kernel<TB_, 1, 1, DIFF, MINB_, KERNEL_HIGHORDER, 1>};
#define PAWAN_F32_CASE_SPLIT2(TB_, U_, MINB_, PK_)                                       \
  if (c.split == 2 && PAWAN_F32_MATCH(TB_, 1, 1, U_, MINB_, PK_))                         \
    return Kernels{&pairs_f32_kernel<TB_, 1, 1, U_, DIFF, MINB_, PK_, KERNEL_HIGHORDER, true>, \
                   &pairs_f32_near_kernel<TB_, 1, 1, DIFF, MINB_, KERNEL_HIGHORDER, 1, 2, 1, PK_>};
#define PAWAN_F32_CASE(TB_, P_, R_, U_, MINB_) PAWAN_F32_CASE_PK(TB_, P_, R_, U_, MINB_, 0)
  PAWAN_F32_CASE_PK(128, 1, 1, 1, 4, 1)
  PAWAN_F32_CASE_PK(128, 1, 1, 2, 4, 1)
  PAWAN_F32_CASE_PK(128, 1, 1, 4, 4, 1)
  PAWAN_F32_CASE_PK(128, 1, 1, 1, 5, 1)
  PAWAN_F32_CASE_PK(128, 1, 1, 2, 5, 1)
  PAWAN_F32_CASE_PK(128, 1, 1, 2, 4, 2)
  PAWAN_F32_CASE_PK(128, 1, 1, 4, 4, 2)
  PAWAN_F32_CASE_PK(256, 1, 1, 2, 2, 1)
  PAWAN_F32_CASE_PK(256, 1, 1, 4, 2, 1)
  PAWAN_F32_CASE_PK(256, 1, 1, 2, 2, 2)
  PAWAN_F32_CASE_PK(256, 1, 1, 4, 2, 2)
  PAWAN_F32_CASE_PK(128, 1, 1, 8, 4, 2)
  PAWAN_F32_CASE_PK(128, 1, 1, 4, 3, 2)
  PAWAN_F32_CASE_PK(128, 1, 1, 8, 3, 2)
  PAWAN_F32_CASE_PK(256, 1, 1, 8, 2, 2)
  PAWAN_F32_CASE(128, 1, 1, 2, 4)
  PAWAN_F32_CASE(128, 1, 1, 4, 4)
  PAWAN_F32_CASE(128, 2, 1, 2, 4)
  PAWAN_F32_CASE(128, 2, 1, 4, 4)
  PAWAN_F32_CASE(128, 4, 1, 4, 4)
  PAWAN_F32_CASE(128, 1, 2, 1, 4)
  PAWAN_F32_CASE(128, 1, 2, 2, 4)
  PAWAN_F32_CASE(128, 1, 1, 2, 5)
  PAWAN_F32_CASE(128, 1, 1, 4, 5)
  PAWAN_F32_CASE(128, 1, 1, 2, 6)
  PAWAN_F32_CASE(128, 1, 1, 4, 6)
  PAWAN_F32_CASE(256, 1, 1, 2, 2)
  PAWAN_F32_CASE(256, 1, 1, 4, 2)
  PAWAN_F32_CASE(256, 2, 1, 4, 2)
  PAWAN_F32_CASE(256, 4, 1, 4, 2)
  PAWAN_F32_CASE(256, 1, 2, 1, 2)
  PAWAN_F32_CASE(256, 1, 2, 2, 2)
  PAWAN_F32_CASE(256, 1, 1, 4, 3)
  PAWAN_F32_CASE_SPLIT(256, 4, 2, 1)
  PAWAN_F32_CASE_SPLIT(256, 4, 2, 2)
  PAWAN_F32_CASE_SPLIT(128, 4, 4, 1)
  PAWAN_F32_CASE_SPLIT(128, 4, 4, 2)
  PAWAN_F32_CASE_SPLIT2(256, 4, 2, 1)
  PAWAN_F32_CASE_SPLIT2(256, 4, 2, 2)
  PAWAN_F32_CASE_SPLIT2(128, 4, 4, 1)
  PAWAN_F32_CASE_SPLIT2(128, 4, 4, 2)
  return Kernels{};
}

// The Gaussian kernel is compiled for the default tilings only (packed mode 2:
// its far tiles never take the uniform-radius branch that modes 1 and 2 differ in).
template <bool DIFF>
Kernels select_gaussian(const PairConfig &c) {
  PAWAN_F32_CASE_K(128, 1, 1, 4, 4, 2, KERNEL_GAUSSIAN)
  PAWAN_F32_CASE_K(128, 1, 1, 2, 4, 0, KERNEL_GAUSSIAN)
  PAWAN_F32_CASE_K(128, 2, 1, 4, 4, 0, KERNEL_GAUSSIAN)
  PAWAN_F32_CASE_K(256, 1, 1, 4, 2, 2, KERNEL_GAUSSIAN)
  return Kernels{};
}
#undef PAWAN_F32_CASE
#undef PAWAN_F32_CASE_PK
#undef PAWAN_F32_CASE_K
#undef PAWAN_F32_CASE_SPLIT
#undef PAWAN_F32_CASE_SPLIT2
#undef PAWAN_F32_MATCH

Kernels select(const PairConfig &c, bool diffusion, int kernel) {
  if (kernel == KERNEL_GAUSSIAN) return diffusion ? select_gaussian<true>(c) : select_gaussian<false>(c);
  if (kernel == KERNEL_HIGHORDER)
    return diffusion ? select_highorder<true>(c) : select_highorder<false>(c);
  return Kernels{};
}

// Dynamic shared memory of a tiling: the staged ring plus the packed far format.
size_t smem_bytes(const PairConfig &c) {
  const size_t fq = c.packed ? (size_t)c.tb / 2 : 1;
  return 8 * (size_t)c.tb * sizeof(float4) + 10 * fq * sizeof(float4) + 2 * fq * sizeof(float2);
}

// Opts a kernel in to its dynamic shared memory beyond the default 48 KB (once
// per kernel and device).
cudaError_t prepare(KernelFn f, size_t bytes) {
  static std::mutex mu;
  static std::set<std::pair<int, KernelFn>> done;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  std::lock_guard<std::mutex> lk(mu);
  if (done.count({dev, f})) return cudaSuccess;
  e = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  if (e == cudaSuccess) done.insert({dev, f});
  return e;
}

}  // namespace

bool pairs_f32_supported(const PairConfig &c, int kernel) {
  return select(c, true, kernel).main != nullptr;
}

cudaError_t pairs_f32_occupancy(const PairConfig &c, bool diffusion, int kernel, int *blocks_per_sm) {
  const Kernels k = select(c, diffusion, kernel);
  if (!k.main) return cudaErrorInvalidValue;
  const size_t bytes = smem_bytes(c);
  cudaError_t e = prepare(k.main, bytes);
  if (e != cudaSuccess) return e;
  return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, k.main, c.tb, bytes);
}

cudaError_t launch_pairs_f32(const PairConfig &c, bool diffusion, int kernel, int grid,
                             const WorkItem *items, int n_items, const SegDesc *segs,
                             int *next_item, cudaStream_t s) {
  const Kernels k = select(c, diffusion, kernel);
  if (!k.main) return cudaErrorInvalidValue;
  const size_t bytes = smem_bytes(c);
  cudaError_t e = prepare(k.main, bytes);
  if (e != cudaSuccess) return e;
  if (k.near) {
    // the near pass first (static shared memory only), on the second counter
    k.near<<<grid, c.tb, 0, s>>>(items, n_items, segs, next_item + 1);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  k.main<<<grid, c.tb, bytes, s>>>(items, n_items, segs, next_item);
  return cudaGetLastError();
}

}  // namespace pawan

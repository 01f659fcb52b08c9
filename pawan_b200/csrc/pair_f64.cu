// All-pairs interaction in FP64 with the kernel algebra of the FP32 kernel
// (pair_f32.cu): two rsqrt per pair, no pow, no division; alpha_i x alpha_j
// per pair as the reference forms it, and the diffusion as
// v_i sum(Dp alpha_j) - alpha_i sum(Dp v_j), taken after the pair loop.
// (Forming the stretching's q-term as alpha_i x sum(q alpha_j) and the triple
// product from the velocity's cross product as well saves six more operations
// per pair but sums nearly parallel neighbours' terms coherently before the
// cross product: 100 times the rounding error of the per-pair form.)  This is the
// "tuned FP64" variant, reported beside the FP32 kernel and the plain FP64
// comparator (pair_plain.cu).  Same work items, partial layout and gather form.
//
// Reference: INTERACT (src/interaction/interaction_utils.h:363-407), KERNEL
// (src/interaction/highorder.h:48-60), __interaction::interact
// (src/interaction/interaction.cpp:95-108).  The Gaussian kernel
// (src/interaction/gaussian.h:20-59) in the same units: with x2 = rho^2/sigma^2,
// e = exp(-x2/2), K = sqrt(2/pi), gq = (erf(x/sqrt 2)/x - K e)/x2 and
// gf = (K e - 3 gq)/x2: qh = gq/sigma^3, fh = gf/(3 sigma^5),
// dp = (2/15) K e / sigma^5 (closed forms, as the reference evaluates them).
#include "device.cuh"
#include "kernels.h"

namespace pawan {
namespace {

__device__ __forceinline__ void load_source_f64(const SegDesc &sg, int j, int s1, double4 &p,
                                                double4 &v) {
  if (j < s1) {
    p = sg.pos64[j];
    v = sg.vor64[j];
  } else {
    p = make_double4(1e150, 1e150, 1e150, 1.0);
    v = make_double4(0.0, 0.0, 0.0, 0.0);
  }
}

// Gaussian qh, fh, dp (see the file comment) from r2, sig2 and 1/rho.
__device__ __forceinline__ void gauss_f64(double r2, double sig2, double ri, double &qh,
                                          double &fh, double &dp) {
  const double is = rsqrt(sig2);
  const double is2 = is * is;
  const double is3 = is2 * is;
  const double x2 = r2 * is2;
  const double e = exp(-0.5 * x2);
  const double x = r2 * ri * is;
  const double gq = (erf(kSqrtHalf * x) / x - kSqrt2OverPi * e) / x2;
  const double gf = (kSqrt2OverPi * e - 3.0 * gq) / x2;
  qh = gq * is3;
  fh = gf * is3 * is2 / 3.0;
  dp = (2.0 / 15.0) * kSqrt2OverPi * e * is3 * is2;
}

template <int TB, bool DIFF, int KERN>
__global__ void __launch_bounds__(TB)
    pairs_f64_kernel(const WorkItem *__restrict__ items, int n_items,
                     const SegDesc *__restrict__ segs, int *__restrict__ next_item) {
  __shared__ double4 sp[2][TB];
  __shared__ double4 sv[2][TB];
  __shared__ int s_item, s_last;
  const int tid = threadIdx.x;

  for (;;) {
    if (tid == 0) s_item = atomicAdd(next_item, 1);
    __syncthreads();
    const int it = s_item;
    __syncthreads();
    if (it >= n_items) break;

    const WorkItem w = items[it];
    const SegDesc sg = segs[w.seg];
    const int i = w.t0 + tid;
    const bool valid = i < sg.n;
    double4 pi = make_double4(0.0, 0.0, 0.0, 1.0);
    double4 vi = make_double4(0.0, 0.0, 0.0, 0.0);
    if (valid) {
      pi = sg.pos64[i];
      vi = sg.vor64[i];
    }
    const double hi = 0.5 * pi.w * pi.w;
    // u = sum qh (alpha_j x d); q = sum qh (alpha_i x alpha_j);
    // G = sum fh [d.(alpha_i x alpha_j)] d; E = sum Dp alpha_j, V = sum Dp v_j
    // (the diffusion is v_i E - V alpha_i)
    double ux = 0, uy = 0, uz = 0, qx = 0, qy = 0, qz = 0, gx = 0, gy = 0, gz = 0;
    double ex = 0, ey = 0, ez = 0, ev = 0;

    const int ntiles = (w.s1 - w.s0 + TB - 1) / TB;
    double4 rp, rv;
    load_source_f64(sg, w.s0 + tid, w.s1, rp, rv);
    for (int t = 0; t < ntiles; ++t) {
      const int buf = t & 1;
      sp[buf][tid] = rp;
      sv[buf][tid] = rv;
      __syncthreads();
      const int ts = w.s0 + t * TB;
      if (t + 1 < ntiles) load_source_f64(sg, ts + TB + tid, w.s1, rp, rv);
      const int skip = i - ts;
#pragma unroll 2
      for (int jj = 0; jj < TB; ++jj) {
        const double4 p = sp[buf][jj];
        const double4 s = sv[buf][jj];
        const double dx = pi.x - p.x, dy = pi.y - p.y, dz = pi.z - p.z;
        const double r2 = fma(dz, dz, fma(dy, dy, dx * dx));
        const double sig2 = fma(0.5 * p.w, p.w, hi);
        const double ri = rsqrt(r2);
        double qh, fh, dp;
        if (KERN == KERNEL_GAUSSIAN) {
          gauss_f64(r2, sig2, ri, qh, fh, dp);
        } else {
          const double wr = rsqrt(r2 + sig2);
          const double ri2 = ri * ri;
          const double w2 = wr * wr;
          const double w4 = w2 * w2;
          const double uu = sig2 * w2;
          const double u2 = uu * uu;
          const double u4 = u2 * u2;
          dp = u4 * uu * (w4 * wr);
          const double zc = dp * sig2;
          const double ph = fma(1.5, sig2, r2) * w4 * ri;
          qh = fma(-7.5, zc, ph) * sig2 * ri2;
          fh = fma(2.5, zc, -qh) * ri2;
        }
        const double cx = fma(s.y, dz, -s.z * dy);
        const double cy = fma(s.z, dx, -s.x * dz);
        const double cz = fma(s.x, dy, -s.y * dx);
        const double wx = fma(vi.y, s.z, -vi.z * s.y);
        const double wy = fma(vi.z, s.x, -vi.x * s.z);
        const double wz = fma(vi.x, s.y, -vi.y * s.x);
        const double tt = fma(dz, wz, fma(dy, wy, dx * wx));
        double ft = fh * tt;
        const bool self = (jj == skip);
        qh = self ? 0.0 : qh;
        ft = self ? 0.0 : ft;
        dp = self ? 0.0 : dp;
        ux = fma(qh, cx, ux);
        uy = fma(qh, cy, uy);
        uz = fma(qh, cz, uz);
        qx = fma(qh, wx, qx);
        qy = fma(qh, wy, qy);
        qz = fma(qh, wz, qz);
        gx = fma(ft, dx, gx);
        gy = fma(ft, dy, gy);
        gz = fma(ft, dz, gz);
        if (DIFF) {
          ex = fma(dp, s.x, ex);
          ey = fma(dp, s.y, ey);
          ez = fma(dp, s.z, ez);
          ev = fma(dp, s.w, ev);
        }
      }
    }

    if (valid) {
      const double A = kInv4Pi;
      double dax = A * qx + 3.0 * A * gx;
      double day = A * qy + 3.0 * A * gy;
      double daz = A * qz + 3.0 * A * gz;
      if (DIFF) {
        // v_i E - V alpha_i
        const double c = 15.0 * sg.nu * A;
        dax += c * fma(vi.w, ex, -ev * vi.x);
        day += c * fma(vi.w, ey, -ev * vi.y);
        daz += c * fma(vi.w, ez, -ev * vi.z);
      }
      const ItemOut o = item_out(sg, w.t0, w.chunk, TB);
      double *out = o.base + (i - w.t0);
      out[0] = A * ux;
      out[o.stride] = A * uy;
      out[2 * o.stride] = A * uz;
      out[3 * o.stride] = dax;
      out[4 * o.stride] = day;
      out[5 * o.stride] = daz;
    }
    if (sg.nchunks > 1) finish_item<TB>(sg, w.t0, TB, &s_last);
  }
}

using KernelFn = void (*)(const WorkItem *, int, const SegDesc *, int *);

template <int KERN>
KernelFn select_k(const PairConfig &c, bool diffusion) {
  if (c.tb == 128)
    return diffusion ? &pairs_f64_kernel<128, true, KERN> : &pairs_f64_kernel<128, false, KERN>;
  if (c.tb == 256)
    return diffusion ? &pairs_f64_kernel<256, true, KERN> : &pairs_f64_kernel<256, false, KERN>;
  return nullptr;
}

KernelFn select(const PairConfig &c, bool diffusion, int kernel) {
  if (c.p != 1 || c.r != 1 || c.packed != 0) return nullptr;
  if (kernel == KERNEL_GAUSSIAN) return select_k<KERNEL_GAUSSIAN>(c, diffusion);
  if (kernel == KERNEL_HIGHORDER) return select_k<KERNEL_HIGHORDER>(c, diffusion);
  return nullptr;
}

}  // namespace

bool pairs_f64_supported(const PairConfig &c, int kernel) { return select(c, true, kernel) != nullptr; }

cudaError_t pairs_f64_occupancy(const PairConfig &c, bool diffusion, int kernel, int *blocks_per_sm) {
  KernelFn f = select(c, diffusion, kernel);
  if (!f) return cudaErrorInvalidValue;
  return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, f, c.tb, 0);
}

cudaError_t launch_pairs_f64(const PairConfig &c, bool diffusion, int kernel, int grid,
                             const WorkItem *items, int n_items, const SegDesc *segs,
                             int *next_item, cudaStream_t s) {
  KernelFn f = select(c, diffusion, kernel);
  if (!f) return cudaErrorInvalidValue;
  f<<<grid, c.tb, 0, s>>>(items, n_items, segs, next_item);
  return cudaGetLastError();
}

}  // namespace pawan

// All-pairs interaction, plain FP64: the reference's pair formula written out
// term by term on the GPU -- rho from a square root, rho_bar = rho/sigma,
// pow(rho_bar^2 + 1, 7.5), pow(sigma, 3), pow(rho_bar^2 + 1, 2) and the
// divisions of KERNEL -- accumulated directly in FP64.  This is the
// straightforward GPU port that the FP32 kernel is measured against, and the
// FP64 path whose results track the reference to rounding.  Compiled with
// --fmad=false so that, like the reference's x86-64 build, no multiply-add is
// contracted.
//
// Reference, line by line:
//   sigma = sqrt(0.5*(s_src^2 + s_trg^2))              interaction_utils.h:452
//   d = r_trg - r_src, rho = |d|                        :447-450
//   Z = 1.875/pi / pow(rho_bar^2+1, 7.5) / pow(sigma,3) highorder.h:20-23
//   phi = 0.25/pi (rho_bar^2+1.5)/pow(rho_bar^2+1,2)/sigma^3, q, F   highorder.h:48-60
//   u += q (alpha_src x d)                              interaction_utils.h:458-459, :52-58
//   da = q (a_trg x a_src) + F [d.(a_trg x a_src)] d    :466, VORSTRETCH :69-100
//   da += (Z nu / (sigma^2/2)) (v_trg a_src - v_src a_trg)   :467, DIFFUSION :253-286
// written for target i (the reference's target role; the source role is the
// same sum with d -> -d, see pair_f32.cu).  With the Gaussian kernel
// (gaussian.h:20-59): Z = exp(-rho_bar^2/2)/pow(sigma,3)/pow(2 pi,1.5),
// phi = 0.25/pi erf(rho_bar/sqrt 2)/sigma^3, q and F as above.
#include "device.cuh"
#include "kernels.h"

namespace pawan {
namespace {

template <int TB, int KERN>
__global__ void __launch_bounds__(TB)
    pairs_plain_kernel(const WorkItem *__restrict__ items, int n_items,
                       const SegDesc *__restrict__ segs, int *__restrict__ next_item) {
  __shared__ double4 sp[TB];
  __shared__ double4 sv[TB];
  __shared__ int s_item, s_last;
  const int tid = threadIdx.x;
  const double one_over_pi = kInvPi;

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
    const double nu = sg.nu;
    double u0 = 0, u1 = 0, u2 = 0, a0 = 0, a1 = 0, a2 = 0;

    for (int ts = w.s0; ts < w.s1; ts += TB) {
      __syncthreads();
      const int j = ts + tid;
      if (j < w.s1) {
        sp[tid] = sg.pos64[j];
        sv[tid] = sg.vor64[j];
      }
      __syncthreads();
      const int cnt = min(TB, w.s1 - ts);
      for (int jj = 0; jj < cnt; ++jj) {
        if (ts + jj == i) continue;
        const double4 p = sp[jj];
        const double4 s = sv[jj];
        const double d0 = pi.x - p.x, d1 = pi.y - p.y, d2 = pi.z - p.z;
        const double rho = sqrt(d0 * d0 + d1 * d1 + d2 * d2);
        const double sigma = sqrt(0.5 * (p.w * p.w + pi.w * pi.w));
        // KERNEL
        const double rho_bar = rho / sigma;
        const double rho_bar2 = rho_bar * rho_bar;
        const double sig3 = sigma * sigma * sigma;
        double Z, phi;
        if (KERN == KERNEL_GAUSSIAN) {
          Z = exp(-0.5 * rho_bar * rho_bar) / pow(sigma, 3.0) / pow(2.0 * kPi, 1.5);
          phi = 0.25 * one_over_pi * erf(kSqrtHalf * rho_bar) / sig3;
        } else {
          Z = 1.875 * one_over_pi / pow(rho_bar * rho_bar + 1.0, 7.5) / pow(sigma, 3.0);
          phi = 0.25 * one_over_pi * (rho_bar2 + 1.5) / pow(rho_bar2 + 1.0, 2.0) / sig3;
        }
        const double q = (phi / rho_bar - Z) / rho_bar2;
        const double F = (Z - 3.0 * q) / (rho * rho);
        // VELOCITY: q (alpha_src x d)
        u0 += q * (s.y * d2 - s.z * d1);
        u1 += q * (s.z * d0 - s.x * d2);
        u2 += q * (s.x * d1 - s.y * d0);
        // VORSTRETCH: a_trg x a_src
        const double c0 = vi.y * s.z - vi.z * s.y;
        const double c1 = vi.z * s.x - vi.x * s.z;
        const double c2 = vi.x * s.y - vi.y * s.x;
        const double roaxa = d0 * c0 + d1 * c1 + d2 * c2;
        // DIFFUSION
        const double sig12 = 0.5 * sigma * sigma;
        const double dscale = Z * nu / sig12;
        a0 += (q * c0 + F * roaxa * d0) + dscale * (vi.w * s.x - s.w * vi.x);
        a1 += (q * c1 + F * roaxa * d1) + dscale * (vi.w * s.y - s.w * vi.y);
        a2 += (q * c2 + F * roaxa * d2) + dscale * (vi.w * s.z - s.w * vi.z);
      }
    }

    if (valid) {
      const ItemOut o = item_out(sg, w.t0, w.chunk, TB);
      double *out = o.base + (i - w.t0);
      out[0] = u0;
      out[o.stride] = u1;
      out[2 * o.stride] = u2;
      out[3 * o.stride] = a0;
      out[4 * o.stride] = a1;
      out[5 * o.stride] = a2;
    }
    if (sg.nchunks > 1) finish_item<TB>(sg, w.t0, TB, &s_last);
  }
}

using KernelFn = void (*)(const WorkItem *, int, const SegDesc *, int *);

KernelFn select(const PairConfig &c, int kernel) {
  if (c.p != 1 || c.r != 1 || c.packed != 0) return nullptr;
  const bool g = kernel == KERNEL_GAUSSIAN;
  if (kernel != KERNEL_HIGHORDER && !g) return nullptr;
  if (c.tb == 128) return g ? &pairs_plain_kernel<128, 1> : &pairs_plain_kernel<128, 0>;
  if (c.tb == 256) return g ? &pairs_plain_kernel<256, 1> : &pairs_plain_kernel<256, 0>;
  return nullptr;
}

}  // namespace

bool pairs_plain_supported(const PairConfig &c, int kernel) { return select(c, kernel) != nullptr; }

cudaError_t pairs_plain_occupancy(const PairConfig &c, int kernel, int *blocks_per_sm) {
  KernelFn f = select(c, kernel);
  if (!f) return cudaErrorInvalidValue;
  return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, f, c.tb, 0);
}

cudaError_t launch_pairs_plain(const PairConfig &c, int kernel, int grid, const WorkItem *items,
                               int n_items, const SegDesc *segs, int *next_item, cudaStream_t s) {
  KernelFn f = select(c, kernel);
  if (!f) return cudaErrorInvalidValue;
  f<<<grid, c.tb, 0, s>>>(items, n_items, segs, next_item);
  return cudaGetLastError();
}

}  // namespace pawan

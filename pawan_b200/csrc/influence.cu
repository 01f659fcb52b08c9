// Smoothed vorticity field of a system, FP64: the counterpart of
// __interaction::influence (src/interaction/interaction.cpp:110-155), which
// __interaction::resolve (:45-47) runs for the influence-matrix path of
// __resolve::rebuild (src/resolve/resolve.cpp:10-57).
//
// Reference: every unordered pair once, INFLUENCE
// (src/interaction/interaction_utils.h:519-556) with
// sigma = sqrt((s_i^2 + s_j^2)/2), Z = ZETASIG(rho, sigma)
// (src/interaction/highorder.h:20-23), K_target += Z alpha_source and
// K_source += Z alpha_target; plus SELFINFLUENCE (:593-605),
// K_i += ZETASIG(0, s_i) alpha_i.  In gather form
//   K_i = sum_j Z(rho_ij, sigma_ij) alpha_j   over every j, i included:
// the j = i term has rho = 0 and sigma = s_i, which is SELFINFLUENCE.
// With w = (rho^2 + sigma^2)^(-1/2) and u = sigma^2 w^2 = 1/(rho_bar^2 + 1):
//   Z = (15 / 8 pi) sigma^-3 (rho_bar^2 + 1)^-7.5 = (15 / 8 pi) u^6 w^3,
// or with the Gaussian kernel (src/interaction/gaussian.h:20-23)
//   Z = exp(-rho_bar^2 / 2) / (sigma^3 (2 pi)^1.5).
//
// One thread per target (registers), sources staged through shared memory
// in tiles, summed in source order: deterministic.  ~20 FP64 operations and
// one rsqrt per pair; the path is small next to the interaction (it is run
// once per influence-matrix column), so FP64 throughout keeps the resolve's
// linear solve as accurate as the reference's.
#include "device.cuh"
#include "kernels.h"

namespace pawan {
namespace {

constexpr int kInfThreads = 128;

template <int KERN>
__global__ void __launch_bounds__(kInfThreads)
    influence_kernel(int n, const double4 *__restrict__ pos, const double4 *__restrict__ vor,
                     double *__restrict__ field) {
  __shared__ double4 sp[kInfThreads];
  __shared__ double4 sv[kInfThreads];
  const int tid = threadIdx.x;
  const int i = blockIdx.x * kInfThreads + tid;
  const bool valid = i < n;
  const double4 ri = valid ? pos[i] : make_double4(0.0, 0.0, 0.0, 1.0);
  const double hi = 0.5 * ri.w * ri.w;
  const double c = 1.875 * kInvPi;  // 15 / (8 pi)
  const double cg = 0.06349363593424096978;  // (2 pi)^-1.5
  double kx = 0.0, ky = 0.0, kz = 0.0;
  for (int ts = 0; ts < n; ts += kInfThreads) {
    __syncthreads();
    const int j = ts + tid;
    if (j < n) {
      sp[tid] = pos[j];
      sv[tid] = vor[j];
    }
    __syncthreads();
    const int cnt = min(kInfThreads, n - ts);
    for (int jj = 0; jj < cnt; ++jj) {
      const double4 rj = sp[jj], aj = sv[jj];
      const double dx = ri.x - rj.x, dy = ri.y - rj.y, dz = ri.z - rj.z;
      const double rho2 = dx * dx + dy * dy + dz * dz;
      const double sig2 = hi + 0.5 * rj.w * rj.w;
      double z;
      if (KERN == KERNEL_GAUSSIAN) {
        const double is = rsqrt(sig2);
        z = exp(-0.5 * rho2 * is * is) * (is * is * is) * cg;
      } else {
        const double w = rsqrt(rho2 + sig2);
        const double w2 = w * w;
        const double u = sig2 * w2;
        const double u2 = u * u;
        const double u6 = u2 * u2 * u2;
        z = c * u6 * w2 * w;
      }
      kx += z * aj.x;
      ky += z * aj.y;
      kz += z * aj.z;
    }
  }
  if (valid) {
    field[3 * (size_t)i] = kx;
    field[3 * (size_t)i + 1] = ky;
    field[3 * (size_t)i + 2] = kz;
  }
}

}  // namespace

cudaError_t launch_influence(int n, int kernel, const double4 *pos64, const double4 *vor64,
                             double *field, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  const int blocks = (n + kInfThreads - 1) / kInfThreads;
  if (kernel == KERNEL_GAUSSIAN)
    influence_kernel<KERNEL_GAUSSIAN><<<blocks, kInfThreads, 0, s>>>(n, pos64, vor64, field);
  else
    influence_kernel<KERNEL_HIGHORDER><<<blocks, kInfThreads, 0, s>>>(n, pos64, vor64, field);
  return cudaGetLastError();
}

}  // namespace pawan

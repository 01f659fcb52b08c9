// Conserved / monitored quantities of a system, all in FP64.
//
// Reference (src/interaction/interaction.cpp):
//   total vorticity  sum alpha                       :240-246
//   linear impulse   1/2 sum x x alpha               :248-259
//   angular impulse  1/3 sum x x (x x alpha)         :261-275
//   enstrophy        sum_i 5/(4 pi s_i^3)|alpha_i|^2 + sum_{i != j} [F1 (a_i.a_j)
//                    + F2 (a_i.x_ij)(a_j.x_ij)]      :277-315, ENSTROPHY
//                    (interaction_utils.h:107-156), ENST (highorder.h:69-86)
//   helicity         sum_{i != j} q(rho,sigma) x_ij.(a_i x a_j)     :317-349,
//                    HELICITY (interaction_utils.h:167-190)
//   kinetic energy   2 sum_i |a_i|^2/(8 pi s_i) + sum_{i != j} w_ij KE_ij with
//                    w_ij = 2 inside a wake, 1 across wakes      :351-383,
//                    KINETICENERGY (interaction_utils.h:197-240)
// With the Gaussian kernel (src/interaction/gaussian.h) the enstrophy terms
// are the reference's stub ENST = 0 (gaussian.h:67-86) and helicity uses the
// Gaussian QSIG (:30-38): q = (phi/rho_bar - Z)/rho_bar^2 with
// phi = erf(rho_bar/sqrt 2)/(4 pi sigma^3), Z = exp(-rho_bar^2/2)/(sigma^3 (2 pi)^1.5).
// The reference's pair loops visit i<j and double (or, across wakes, double
// the full cross sum); both equal one term per ordered pair, which is the
// gather sum written here.  Per-target sums are reduced per block in a fixed
// tree and the block partials by one block in fixed order: deterministic.
#include "device.cuh"
#include "kernels.h"

namespace pawan {
namespace {

constexpr int kDiagThreads = 128;
constexpr int kLin = 9;   // linear quantities
constexpr int kQuad = 3;  // enstrophy, helicity, kinetic energy

template <int K>
__device__ void block_sum(double (&v)[K], double *smem /* [K][kDiagThreads] */, double *out) {
  const int t = threadIdx.x;
#pragma unroll
  for (int k = 0; k < K; ++k) smem[k * kDiagThreads + t] = v[k];
  __syncthreads();
  for (int s = kDiagThreads / 2; s > 0; s >>= 1) {
    if (t < s) {
#pragma unroll
      for (int k = 0; k < K; ++k) smem[k * kDiagThreads + t] += smem[k * kDiagThreads + t + s];
    }
    __syncthreads();
  }
  if (t == 0) {
#pragma unroll
    for (int k = 0; k < K; ++k) out[k] = smem[k * kDiagThreads];
  }
}

__global__ void __launch_bounds__(kDiagThreads)
    diag_linear_kernel(int n, const double4 *__restrict__ pos, const double4 *__restrict__ vor,
                       double *__restrict__ block_out) {
  __shared__ double smem[kLin * kDiagThreads];
  const int i = blockIdx.x * kDiagThreads + threadIdx.x;
  double v[kLin];
#pragma unroll
  for (int k = 0; k < kLin; ++k) v[k] = 0.0;
  if (i < n) {
    const double4 r = pos[i], a = vor[i];
    const double rxa0 = r.y * a.z - r.z * a.y;
    const double rxa1 = r.z * a.x - r.x * a.z;
    const double rxa2 = r.x * a.y - r.y * a.x;
    v[0] = a.x;
    v[1] = a.y;
    v[2] = a.z;
    v[3] = rxa0;
    v[4] = rxa1;
    v[5] = rxa2;
    v[6] = r.y * rxa2 - r.z * rxa1;
    v[7] = r.z * rxa0 - r.x * rxa2;
    v[8] = r.x * rxa1 - r.y * rxa0;
  }
  block_sum<kLin>(v, smem, block_out + (size_t)blockIdx.x * kLin);
}

template <int KERN>
__global__ void __launch_bounds__(kDiagThreads)
    diag_quadratic_kernel(int n, const double4 *__restrict__ pos, const double4 *__restrict__ vor,
                          const int *__restrict__ wake_id, double *__restrict__ block_out) {
  __shared__ double4 sp[kDiagThreads];
  __shared__ double4 sv[kDiagThreads];
  __shared__ int sw[kDiagThreads];
  __shared__ double smem[kQuad * kDiagThreads];
  const int tid = threadIdx.x;
  const int i = blockIdx.x * kDiagThreads + tid;
  const bool valid = i < n;
  double4 ri = make_double4(0, 0, 0, 1), ai = make_double4(0, 0, 0, 0);
  int wi = -1;
  if (valid) {
    ri = pos[i];
    ai = vor[i];
    wi = wake_id[i];
  }
  const double A = kInv4Pi;
  const double si = ri.w;
  const double hi = 0.5 * si * si;
  const double a2 = ai.x * ai.x + ai.y * ai.y + ai.z * ai.z;
  double ens = (valid && KERN == KERNEL_HIGHORDER) ? 5.0 * kInvPi / 4.0 / (si * si * si) * a2 : 0.0;
  double hel = 0.0;
  double ke = valid ? 2.0 * (kInvPi * a2 / si / 8.0) : 0.0;

  for (int ts = 0; ts < n; ts += kDiagThreads) {
    __syncthreads();
    const int j = ts + tid;
    if (j < n) {
      sp[tid] = pos[j];
      sv[tid] = vor[j];
      sw[tid] = wake_id[j];
    }
    __syncthreads();
    const int cnt = min(kDiagThreads, n - ts);
    for (int jj = 0; jj < cnt; ++jj) {
      if (ts + jj == i) continue;
      const double4 rj = sp[jj], aj = sv[jj];
      const double x0 = rj.x - ri.x, x1 = rj.y - ri.y, x2 = rj.z - ri.z;
      const double rho2 = x0 * x0 + x1 * x1 + x2 * x2;
      const double sig2 = hi + 0.5 * rj.w * rj.w;
      const double w = rsqrt(rho2 + sig2);
      const double w2 = w * w, w3 = w2 * w, w4 = w2 * w2;
      const double aa = ai.x * aj.x + ai.y * aj.y + ai.z * aj.z;
      const double aix = ai.x * x0 + ai.y * x1 + ai.z * x2;
      const double ajx = aj.x * x0 + aj.y * x1 + aj.z * x2;
      const double rinv = rsqrt(rho2);
      double q;
      if (KERN == KERNEL_GAUSSIAN) {
        // QSIG, gaussian.h:30-38
        const double sig = sqrt(sig2);
        const double rho_bar = rho2 * rinv / sig;
        const double sig3 = sig2 * sig;
        const double z = exp(-0.5 * rho_bar * rho_bar) / sig3 / pow(2.0 * kPi, 1.5);
        const double phi = 0.25 * kInvPi * erf(kSqrtHalf * rho_bar) / sig3;
        q = (phi / rho_bar - z) / (rho_bar * rho_bar);
      } else {
        // ENST: factor = (1/8pi) (rho^2 + sigma^2)^(-7/2)
        const double factor = (kInvPi / 8.0) * (w4 * w3);
        const double F1 = factor * (10.0 * sig2 * sig2 - 2.0 * rho2 * rho2 - 7.0 * sig2 * rho2);
        const double F2 = factor * (-15.0 * rho2);
        ens += F1 * aa + F2 * aix * ajx;
        // QSIG: q = (phi/rho_bar - Z)/rho_bar^2
        const double uu = sig2 * w2;
        const double u2 = uu * uu;
        const double zc = u2 * u2 * u2 * w3;
        const double ph = (rho2 + 1.5 * sig2) * w4 * rinv;
        q = A * (ph - 7.5 * zc) * sig2 * (rinv * rinv);
      }
      const double c0 = ai.y * aj.z - ai.z * aj.y;
      const double c1 = ai.z * aj.x - ai.x * aj.z;
      const double c2 = ai.x * aj.y - ai.y * aj.x;
      hel += q * (x0 * c0 + x1 * c1 + x2 * c2);
      // KINETICENERGY
      const double e = ((rho2 + 2.0 * sig2) * aa + aix * ajx) * w3 / 16.0 * kInvPi;
      ke += (sw[jj] == wi ? 2.0 : 1.0) * e;
    }
  }
  double v[kQuad] = {valid ? ens : 0.0, valid ? hel : 0.0, valid ? ke : 0.0};
  __syncthreads();
  block_sum<kQuad>(v, smem, block_out + (size_t)blockIdx.x * kQuad);
}

// One block: sums nblk rows of width K in a fixed order.
template <int K>
__global__ void __launch_bounds__(kDiagThreads)
    diag_final_kernel(int nblk, const double *__restrict__ rows, double *__restrict__ out,
                      double scale_lin) {
  __shared__ double smem[K * kDiagThreads];
  double v[K];
#pragma unroll
  for (int k = 0; k < K; ++k) v[k] = 0.0;
  for (int b = threadIdx.x; b < nblk; b += kDiagThreads) {
#pragma unroll
    for (int k = 0; k < K; ++k) v[k] += rows[(size_t)b * K + k];
  }
  double tot[K];
  block_sum<K>(v, smem, tot);
  if (threadIdx.x == 0) {
    if (K == kLin) {
      for (int k = 0; k < 3; ++k) {
        out[k] = tot[k];
        out[3 + k] = tot[3 + k] * 0.5;
        out[6 + k] = tot[6 + k] * (1.0 / 3.0);
      }
    } else {
      for (int k = 0; k < K; ++k) out[9 + k] = tot[k];
    }
  }
}

}  // namespace

size_t diag_scratch_doubles(int n) {
  const size_t nblk = (size_t)(n + kDiagThreads - 1) / kDiagThreads;
  return nblk * (kLin + kQuad);
}

cudaError_t launch_diagnostics(int n, int kernel, const double4 *pos64, const double4 *vor64,
                               const int *wake_id, double *scratch, double *out, bool quadratic,
                               cudaStream_t s) {
  if (n <= 0) return cudaErrorInvalidValue;
  const int nblk = (n + kDiagThreads - 1) / kDiagThreads;
  double *lin = scratch;
  double *quad = scratch + (size_t)nblk * kLin;
  diag_linear_kernel<<<nblk, kDiagThreads, 0, s>>>(n, pos64, vor64, lin);
  diag_final_kernel<kLin><<<1, kDiagThreads, 0, s>>>(nblk, lin, out, 0.0);
  if (quadratic) {
    if (kernel == KERNEL_GAUSSIAN)
      diag_quadratic_kernel<KERNEL_GAUSSIAN><<<nblk, kDiagThreads, 0, s>>>(n, pos64, vor64, wake_id, quad);
    else
      diag_quadratic_kernel<KERNEL_HIGHORDER><<<nblk, kDiagThreads, 0, s>>>(n, pos64, vor64, wake_id, quad);
    diag_final_kernel<kQuad><<<1, kDiagThreads, 0, s>>>(nblk, quad, out, 0.0);
  }
  return cudaGetLastError();
}

}  // namespace pawan

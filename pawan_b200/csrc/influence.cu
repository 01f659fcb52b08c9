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
//
// The columns kernel evaluates the field of many strength vectors over the
// same positions and radii at once -- the influence-matrix columns of
// __resolve::rebuild (resolve.cpp:19-31), which differ only in alpha.  Z of a
// pair is formed once and applied to kColGroup columns (3 FMAs each), so a
// column costs 3 FMAs per pair instead of ~20 operations.  Both kernels form
// Z with the same function and accumulate with explicit FMAs in source order,
// so a column of the batched kernel is bit-identical to a single-column launch.
#include "device.cuh"
#include "kernels.h"

namespace pawan {
namespace {

constexpr int kInfThreads = 128;
constexpr int kColGroup = kInfluenceColumnGroup;  // 3 x 8 FP64 accumulators per thread

// Z(rho_ij, sigma_ij) for target i (position ri, hi = s_i^2 / 2) and source
// j (rj = position, smoothing radius); operations written out so that every
// kernel rounds them the same way.
template <int KERN>
__device__ __forceinline__ double pair_z(const double4 ri, double hi, const double4 rj) {
  const double dx = __dsub_rn(ri.x, rj.x), dy = __dsub_rn(ri.y, rj.y), dz = __dsub_rn(ri.z, rj.z);
  const double rho2 = __fma_rn(dz, dz, __fma_rn(dy, dy, __dmul_rn(dx, dx)));
  const double sig2 = __fma_rn(0.5 * rj.w, rj.w, hi);
  if (KERN == KERNEL_GAUSSIAN) {
    const double cg = 0.06349363593424096978;  // (2 pi)^-1.5
    const double is = rsqrt(sig2);
    const double is2 = __dmul_rn(is, is);
    return __dmul_rn(__dmul_rn(exp(-0.5 * __dmul_rn(rho2, is2)), __dmul_rn(is2, is)), cg);
  } else {
    const double c = 1.875 * kInvPi;  // 15 / (8 pi)
    const double w = rsqrt(__dadd_rn(rho2, sig2));
    const double w2 = __dmul_rn(w, w);
    const double u = __dmul_rn(sig2, w2);
    const double u2 = __dmul_rn(u, u);
    const double u6 = __dmul_rn(__dmul_rn(u2, u2), u2);
    return __dmul_rn(__dmul_rn(c, u6), __dmul_rn(w2, w));
  }
}

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
  const double hi = __dmul_rn(0.5 * ri.w, ri.w);
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
      const double4 aj = sv[jj];
      const double z = pair_z<KERN>(ri, hi, sp[jj]);
      kx = __fma_rn(z, aj.x, kx);
      ky = __fma_rn(z, aj.y, ky);
      kz = __fma_rn(z, aj.z, kz);
    }
  }
  if (valid) {
    field[3 * (size_t)i] = kx;
    field[3 * (size_t)i + 1] = ky;
    field[3 * (size_t)i + 2] = kz;
  }
}

// Grid: (target blocks, column groups).  cols and field are ncols blocks of
// N x 3 doubles (column c, particle j, component k at (c*N + j)*3 + k).
template <int KERN>
__global__ void __launch_bounds__(kInfThreads)
    influence_columns_kernel(int n, int ncols, const double4 *__restrict__ pos,
                             const double *__restrict__ cols, double *__restrict__ field) {
  // sources' positions, and each column's strengths one double4 per source
  // (x, y, z, unused) so that a source's three components are one load
  __shared__ double4 sp[kInfThreads];
  __shared__ double4 sa[kColGroup][kInfThreads];
  const int tid = threadIdx.x;
  const int i = blockIdx.x * kInfThreads + tid;
  const int c0 = blockIdx.y * kColGroup;
  const int nc = min(kColGroup, ncols - c0);
  const bool valid = i < n;
  const double4 ri = valid ? pos[i] : make_double4(0.0, 0.0, 0.0, 1.0);
  const double hi = __dmul_rn(0.5 * ri.w, ri.w);
  double k[kColGroup][3];
#pragma unroll
  for (int c = 0; c < kColGroup; ++c) k[c][0] = k[c][1] = k[c][2] = 0.0;
  for (int ts = 0; ts < n; ts += kInfThreads) {
    __syncthreads();
    const int cnt = min(kInfThreads, n - ts);
    if (tid < cnt) sp[tid] = pos[ts + tid];
    for (int c = 0; c < nc; ++c) {
      const double *src = cols + ((size_t)(c0 + c) * n + ts) * 3;
      double *dst = reinterpret_cast<double *>(sa[c]);
      for (int e = tid; e < 3 * cnt; e += kInfThreads) dst[4 * (e / 3) + e % 3] = src[e];
    }
    __syncthreads();
    for (int jj = 0; jj < cnt; ++jj) {
      const double z = pair_z<KERN>(ri, hi, sp[jj]);
#pragma unroll
      for (int c = 0; c < kColGroup; ++c) {
        if (c < nc) {
          const double4 a = sa[c][jj];
          k[c][0] = __fma_rn(z, a.x, k[c][0]);
          k[c][1] = __fma_rn(z, a.y, k[c][1]);
          k[c][2] = __fma_rn(z, a.z, k[c][2]);
        }
      }
    }
  }
  if (valid) {
#pragma unroll
    for (int c = 0; c < kColGroup; ++c) {
      if (c < nc) {
        double *o = field + ((size_t)(c0 + c) * n + i) * 3;
        o[0] = k[c][0];
        o[1] = k[c][1];
        o[2] = k[c][2];
      }
    }
  }
}

}  // namespace

cudaError_t launch_influence_columns(int n, int ncols, int kernel, const double4 *pos64,
                                     const double *cols, double *field, cudaStream_t s) {
  if (n <= 0 || ncols <= 0) return cudaSuccess;
  const int groups = (ncols + kColGroup - 1) / kColGroup;
  if (groups > 65535) return cudaErrorInvalidValue;
  const dim3 grid((n + kInfThreads - 1) / kInfThreads, groups);
  if (kernel == KERNEL_GAUSSIAN)
    influence_columns_kernel<KERNEL_GAUSSIAN><<<grid, kInfThreads, 0, s>>>(n, ncols, pos64, cols, field);
  else
    influence_columns_kernel<KERNEL_HIGHORDER><<<grid, kInfThreads, 0, s>>>(n, ncols, pos64, cols, field);
  return cudaGetLastError();
}

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

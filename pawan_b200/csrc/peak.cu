// Arithmetic-throughput probes used as roofline denominators: long chains of
// independent FP32 FFMA (resp. FP64 DFMA), kPeakChains per thread, so the FMA
// pipe, not latency, is the limit.  Each launched FMA counts 2 flops.
#include "kernels.h"

namespace pawan {
namespace {

__global__ void ffma_peak_kernel(int iters, float *sink) {
  float a[kPeakChains];
  const float m = 1.0f - 1e-7f * (float)(threadIdx.x & 7);
  const float c = 1e-7f;
#pragma unroll
  for (int k = 0; k < kPeakChains; ++k) a[k] = (float)(threadIdx.x + k);
  for (int it = 0; it < iters; ++it) {
#pragma unroll
    for (int r = 0; r < 16; ++r) {
#pragma unroll
      for (int k = 0; k < kPeakChains; ++k) a[k] = fmaf(a[k], m, c);
    }
  }
  float s = 0.f;
#pragma unroll
  for (int k = 0; k < kPeakChains; ++k) s += a[k];
  if (s == 1234.5f) sink[blockIdx.x] = s;  // keeps the chains live
}

// The same with packed FP32x2 FMAs (two FMAs per instruction).
__global__ void ffma2_peak_kernel(int iters, float *sink) {
  float2 a[kPeakChains / 2];
  const float m = 1.0f - 1e-7f * (float)(threadIdx.x & 7);
  const float2 m2 = make_float2(m, m), c2 = make_float2(1e-7f, 1e-7f);
#pragma unroll
  for (int k = 0; k < kPeakChains / 2; ++k)
    a[k] = make_float2((float)(threadIdx.x + 2 * k), (float)(threadIdx.x + 2 * k + 1));
  for (int it = 0; it < iters; ++it) {
#pragma unroll
    for (int r = 0; r < 16; ++r) {
#pragma unroll
      for (int k = 0; k < kPeakChains / 2; ++k) a[k] = __ffma2_rn(a[k], m2, c2);
    }
  }
  float s = 0.f;
#pragma unroll
  for (int k = 0; k < kPeakChains / 2; ++k) s += a[k].x + a[k].y;
  if (s == 1234.5f) sink[blockIdx.x] = s;
}

__global__ void dfma_peak_kernel(int iters, double *sink) {
  double a[kPeakChains];
  const double m = 1.0 - 1e-13 * (double)(threadIdx.x & 7);
  const double c = 1e-13;
#pragma unroll
  for (int k = 0; k < kPeakChains; ++k) a[k] = (double)(threadIdx.x + k);
  for (int it = 0; it < iters; ++it) {
#pragma unroll
    for (int r = 0; r < 16; ++r) {
#pragma unroll
      for (int k = 0; k < kPeakChains; ++k) a[k] = fma(a[k], m, c);
    }
  }
  double s = 0.0;
#pragma unroll
  for (int k = 0; k < kPeakChains; ++k) s += a[k];
  if (s == 1234.5) sink[blockIdx.x] = s;
}

}  // namespace

// FMAs launched: blocks * threads * iters * 16 * kPeakChains.
cudaError_t launch_ffma_peak(int blocks, int threads, int iters, float *sink, cudaStream_t s) {
  ffma_peak_kernel<<<blocks, threads, 0, s>>>(iters, sink);
  return cudaGetLastError();
}

cudaError_t launch_ffma2_peak(int blocks, int threads, int iters, float *sink, cudaStream_t s) {
  ffma2_peak_kernel<<<blocks, threads, 0, s>>>(iters, sink);
  return cudaGetLastError();
}

cudaError_t launch_dfma_peak(int blocks, int threads, int iters, double *sink, cudaStream_t s) {
  dfma_peak_kernel<<<blocks, threads, 0, s>>>(iters, sink);
  return cudaGetLastError();
}

}  // namespace pawan

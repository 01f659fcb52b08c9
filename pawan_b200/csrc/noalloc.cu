// pawan_interact_noalloc: the FP32 all-pairs interaction for callers that
// cannot allocate device memory.
//
// Who needs it: code that runs where cudaMalloc is not allowed or not safe --
// inside a host callback, under a memory manager that owns every allocation on
// the device (a pool handed to a plugin), or in a hard real-time loop where an
// allocation's implicit synchronisation and latency are unacceptable.  Such a
// caller owns its inputs and outputs but cannot let the library create
// buffers.  This entry point therefore keeps all of its working memory (the
// packed FP32 tile data, tile bounding boxes, per-chunk partial sums, the
// work list, the per-tile counters, the summed rates and the scheduler
// counter) in one file-scope device array,
// `g_noalloc_scratch`, sized for at most kNoallocMaxParticles particles.
// Every GPU that loads the library reserves that array until the process
// exits.
//
// Set-up: the first call on a device (with that device current) looks up the
// array's device address with cudaGetSymbolAddress and caches it; make that
// first call before any stream capture.  Later calls only launch kernels.
// All calls share the one array, so calls whose kernels overlap on the GPU
// (different streams, different host threads) race and must be serialised by
// the caller.  Whatever must start at zero (the scheduler counter and the
// per-tile counters) is cleared by the call itself; the rest is fully
// overwritten before it is read.
//
// The pair kernel is pawan_system_solve's in PAWAN_PREC_F32 with the
// high-order smoothing kernel only, at a fixed tiling (128 threads, one
// target per thread) and 4,096-source chunks.  The FP32 positions are taken
// relative to particle 0 (pawan_system_set_particles uses the centroid), and
// the near-tile radius max(4 s_max, 0.03 x extent) measures the extent from
// particle 0, so it can be up to twice the allocating path's: more tile pairs
// may take the accurate near formulation.  Results therefore agree with
// pawan_system_solve within the FP32 tolerance, not bit for bit.
#include <cmath>
#include <cstddef>
#include <mutex>

#include "../../include/pawan_b200.h"
#include "device.cuh"
#include "kernels.h"

namespace pawan {
namespace {

constexpr int kNoallocMaxParticles = 16384;
constexpr int kNaTB = 128;         // threads per block = sources per tile
constexpr int kNaChunk = 4096;     // sources per work item
constexpr int kNaMaxTiles = (kNoallocMaxParticles + kNaTB - 1) / kNaTB;
constexpr int kNaMaxChunks = (kNoallocMaxParticles + kNaChunk - 1) / kNaChunk;
constexpr int kNaMaxItems = kNaMaxTiles * kNaMaxChunks;
constexpr int kNaPrepBlocks = (kNoallocMaxParticles + kStageThreads - 1) / kStageThreads;

// Layout of the scratch array.  The kernels need 16-byte alignment of the
// float4 arrays (their offsets are multiples of 256 bytes) and natural
// alignment of the rest.
struct NoallocScratch {
  float4 pos32[kNoallocMaxParticles];
  float4 vor32[kNoallocMaxParticles];
  float4 poslo[kNoallocMaxParticles];
  float4 vorlo[kNoallocMaxParticles];
  float4 boxes[2 * kNaMaxTiles];
  double partial[kNaMaxTiles * kNaMaxChunks * 6 * kNaTB];  // [tile][chunk][6][128]
  double rates[6 * kNoallocMaxParticles];                  // [6][n]
  float block_max[2 * kNaPrepBlocks];  // per prepare block: max s, max |x - x0|^2
  WorkItem items[kNaMaxItems];
  int tile_count[kNaMaxTiles];
  SegDesc seg;
  int counter;
};

static_assert(offsetof(NoallocScratch, boxes) % 256 == 0 && offsetof(NoallocScratch, partial) % 256 == 0 &&
                  offsetof(NoallocScratch, rates) % 256 == 0,
              "scratch arrays on 256-byte boundaries");

static __device__ __align__(256) unsigned char g_noalloc_scratch[sizeof(NoallocScratch)];

// Pack: positions relative to particle 0 as FP32 hi/lo, strengths hi/lo,
// s^2/2 and volume; the bounding box (with the range of s^2/2 in w) of each
// 128-particle tile; per-block maxima of the smoothing radius and of the
// distance from particle 0.
__global__ void __launch_bounds__(kStageThreads)
    noalloc_prepare(NoallocScratch *S, const double *pos, const double *vor, const double *rad,
                    const double *vol, int n) {
  __shared__ float lo[4][kStageThreads], hi[4][kStageThreads];
  __shared__ float ms[kStageThreads], me[kStageThreads];
  const int t = threadIdx.x;
  const int l = blockIdx.x * kStageThreads + t;
  const bool has = l < n;
  float4 p = make_float4(0.f, 0.f, 0.f, 0.f);
  float s_l = 0.f, e2 = 0.f;
  if (has) {
    const double rx = pos[3 * l] - pos[0], ry = pos[3 * l + 1] - pos[1], rz = pos[3 * l + 2] - pos[2];
    const float hx = (float)rx, hy = (float)ry, hz = (float)rz;
    const double s = rad[l];
    const float ax = (float)vor[3 * l], ay = (float)vor[3 * l + 1], az = (float)vor[3 * l + 2];
    const float hw = (float)(0.5 * s * s);
    S->pos32[l] = make_float4(hx, hy, hz, hw);
    S->poslo[l] = make_float4((float)(rx - (double)hx), (float)(ry - (double)hy),
                              (float)(rz - (double)hz), 0.f);
    S->vor32[l] = make_float4(ax, ay, az, (float)vol[l]);
    S->vorlo[l] = make_float4((float)(vor[3 * l] - (double)ax), (float)(vor[3 * l + 1] - (double)ay),
                              (float)(vor[3 * l + 2] - (double)az), 0.f);
    p = make_float4(hx, hy, hz, hw);
    s_l = (float)s;
    e2 = (float)(rx * rx + ry * ry + rz * rz);
  }
  lo[0][t] = has ? p.x : INFINITY;
  lo[1][t] = has ? p.y : INFINITY;
  lo[2][t] = has ? p.z : INFINITY;
  lo[3][t] = has ? p.w : INFINITY;
  hi[0][t] = has ? p.x : -INFINITY;
  hi[1][t] = has ? p.y : -INFINITY;
  hi[2][t] = has ? p.z : -INFINITY;
  hi[3][t] = has ? p.w : -INFINITY;
  ms[t] = s_l;
  me[t] = e2;
  __syncthreads();
  for (int s = kStageThreads / 2; s > 0; s >>= 1) {
    if (t < s) {
      ms[t] = fmaxf(ms[t], ms[t + s]);
      me[t] = fmaxf(me[t], me[t + s]);
    }
    if ((t % kNaTB) < s && s < kNaTB) {
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        lo[k][t] = fminf(lo[k][t], lo[k][t + s]);
        hi[k][t] = fmaxf(hi[k][t], hi[k][t + s]);
      }
    }
    __syncthreads();
  }
  if ((t % kNaTB) == 0 && l < n) {
    const int b = l / kNaTB;
    S->boxes[2 * b] = make_float4(lo[0][t], lo[1][t], lo[2][t], lo[3][t]);
    S->boxes[2 * b + 1] = make_float4(hi[0][t], hi[1][t], hi[2][t], hi[3][t]);
  }
  if (t == 0) {
    S->block_max[2 * blockIdx.x] = ms[0];
    S->block_max[2 * blockIdx.x + 1] = me[0];
  }
}

// One block: near-tile radius (the rule of pawan_system_set_particles, with the
// extent measured from particle 0), the segment descriptor, the work list, and
// the cleared scheduler counter.
__global__ void noalloc_plan(NoallocScratch *S, int n, int nblocks, double nu) {
  __shared__ float smax, emax;
  if (threadIdx.x == 0) {
    float a = 0.f, b = 0.f;
    for (int k = 0; k < nblocks; ++k) {
      a = fmaxf(a, S->block_max[2 * k]);
      b = fmaxf(b, S->block_max[2 * k + 1]);
    }
    smax = a;
    emax = b;
    const float r_near = fmaxf(4.f * smax, 0.03f * sqrtf(emax));
    SegDesc d;
    d.pos32 = S->pos32;
    d.vor32 = S->vor32;
    d.poslo = S->poslo;
    d.vorlo = S->vorlo;
    d.pos64 = nullptr;
    d.vor64 = nullptr;
    d.boxes = S->boxes;
    d.partial = S->partial;
    d.rates = S->rates;
    d.tile_count = S->tile_count;
    d.near_partial = nullptr;
    d.near_flag = nullptr;
    d.n = n;
    d.nchunks = (n + kNaChunk - 1) / kNaChunk;
    d.nu = nu;
    d.near2 = r_near * r_near;
    S->seg = d;
    S->counter = 0;
  }
  __syncthreads();
  const int tiles = (n + kNaTB - 1) / kNaTB;
  const int chunks = (n + kNaChunk - 1) / kNaChunk;
  for (int t = threadIdx.x; t < tiles; t += blockDim.x) S->tile_count[t] = 0;
  for (int it = threadIdx.x; it < tiles * chunks; it += blockDim.x) {
    const int c = it / tiles, tt = it % tiles;
    WorkItem w;
    w.seg = 0;
    w.t0 = tt * kNaTB;
    w.chunk = c;
    w.s0 = c * kNaChunk;
    w.s1 = min(n, (c + 1) * kNaChunk);
    S->items[it] = w;
  }
}

// The pair kernel's rates ([6][n], chunks summed in chunk order) into the
// caller's N x 3 outputs.
__global__ void noalloc_reduce(const NoallocScratch *S, int n, double *vel, double *dvor) {
  const int l = blockIdx.x * blockDim.x + threadIdx.x;
  if (l >= n) return;
  for (int k = 0; k < 3; ++k) {
    vel[3 * (size_t)l + k] = S->rates[(size_t)k * n + l];
    dvor[3 * (size_t)l + k] = S->rates[(size_t)(3 + k) * n + l];
  }
}

struct DeviceSlot {
  NoallocScratch *scratch = nullptr;
  int grid = 0;
};
constexpr int kMaxDevices = 64;
DeviceSlot g_slots[kMaxDevices];
std::mutex g_slots_mu;

// Once per device, with that device current: the array's device address (in
// host code the symbol itself names a host-side stand-in, not device memory)
// and the persistent grid size.
cudaError_t device_slot(int dev, DeviceSlot *out) {
  std::lock_guard<std::mutex> lk(g_slots_mu);
  DeviceSlot &s = g_slots[dev];
  if (!s.scratch) {
    void *ptr = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
    if (e != cudaSuccess) return e;
    int sms = 0, bps = 0;
    e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return e;
    e = pairs_f32_occupancy(PairConfig{kNaTB, 1, 2}, true, KERNEL_HIGHORDER, &bps);
    if (e != cudaSuccess) return e;
    int bps0 = 0;
    e = pairs_f32_occupancy(PairConfig{kNaTB, 1, 2}, false, KERNEL_HIGHORDER, &bps0);
    if (e != cudaSuccess) return e;
    s.grid = sms * (bps < bps0 ? bps : bps0);
    s.scratch = static_cast<NoallocScratch *>(ptr);
  }
  *out = s;
  return cudaSuccess;
}

}  // namespace
}  // namespace pawan

extern "C" int pawan_interact_noalloc(const double *position, const double *vorticity,
                                      const double *radius, const double *volume, size_t n,
                                      double nu, double *velocity, double *retvorcity,
                                      void *stream) {
  using namespace pawan;
  if (!position || !vorticity || !radius || !volume || !velocity || !retvorcity)
    return PAWAN_ERR_INVALID;
  if (n < 2 || n > (size_t)kNoallocMaxParticles || !std::isfinite(nu) || nu < 0.0)
    return PAWAN_ERR_INVALID;
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return PAWAN_ERR_CUDA;
  DeviceSlot slot;
  if (device_slot(dev, &slot) != cudaSuccess) return PAWAN_ERR_CUDA;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const int ni = (int)n;
  const int pblocks = (ni + kStageThreads - 1) / kStageThreads;
  noalloc_prepare<<<pblocks, kStageThreads, 0, s>>>(slot.scratch, position, vorticity, radius,
                                                     volume, ni);
  noalloc_plan<<<1, 256, 0, s>>>(slot.scratch, ni, pblocks, nu);
  const int items = ((ni + kNaTB - 1) / kNaTB) * ((ni + kNaChunk - 1) / kNaChunk);
  cudaError_t e = launch_pairs_f32(PairConfig{kNaTB, 1, 2}, nu != 0.0, KERNEL_HIGHORDER, slot.grid,
                                   slot.scratch->items, items, &slot.scratch->seg,
                                   &slot.scratch->counter, s);
  if (e != cudaSuccess) return PAWAN_ERR_CUDA;
  noalloc_reduce<<<(ni + 255) / 256, 256, 0, s>>>(slot.scratch, ni, velocity, retvorcity);
  if (cudaGetLastError() != cudaSuccess) return PAWAN_ERR_CUDA;
  return PAWAN_OK;
}

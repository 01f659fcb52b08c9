// Time integration with .wake frames written asynchronously: the counterpart of
// __integration::integrate (src/integration/integration.cpp:16-35).
//
// The reference writes a frame -- t, then __interaction::write (nWake, and per
// wake N, x (N x 3), alpha (N x 3), s (N); interaction.cpp:197-202,
// wake.cpp:68-73) -- at t = 0 and after every step i at t = i*dt, dt = T/n
// (integration.cpp:10-14, 24-30), on the integrating thread.  Here the steps
// stay on the device and each frame leaves it without stopping them: after a
// step the state is copied to a device snapshot on the integration stream
// (ordered after the step, so the next step may overwrite the state), a copy
// stream waits for that and moves the snapshot to pinned host memory, and a
// writer thread waits for the copy and writes the frame.  Three snapshot /
// pinned slots rotate; a slot is reused only after its frame is on disk.  The
// smoothing radii do not change during integration and are read once.
#include <condition_variable>
#include <cstdio>
#include <string>
#include <deque>
#include <mutex>
#include <thread>
#include <vector>

#include "runtime.h"

using namespace pawan;

// The writer's CUDA calls report through the context like the rest of the ABI.
#define PAWAN_CUDA_RET(expr)                                  \
  do {                                                        \
    cudaError_t e_ = (expr);                                  \
    if (e_ != cudaSuccess) return cuda_fail(ctx_, e_, #expr); \
  } while (0)

namespace {

constexpr int kSlots = 3;

class FrameWriter {
 public:
  FrameWriter(pawan_system *sys, FILE *f) : sys_(sys), ctx_(sys->ctx), f_(f) {}
  ~FrameWriter() { stop(); }

  int start() {
    const size_t N = sys_->n;
    rad_.resize(N);
    PAWAN_CUDA_RET(cudaMemcpyAsync(rad_.data(), sys_->rad.p, N * sizeof(double),
                                   cudaMemcpyDeviceToHost, ctx_->stream));
    PAWAN_CUDA_RET(cudaStreamSynchronize(ctx_->stream));
    PAWAN_CUDA_RET(cudaStreamCreateWithFlags(&copy_, cudaStreamNonBlocking));
    for (int k = 0; k < kSlots; ++k) {
      PAWAN_CUDA_RET(snap_[k].alloc(6 * N));
      PAWAN_CUDA_RET(cudaMallocHost(reinterpret_cast<void **>(&host_[k]), 6 * N * sizeof(double)));
      PAWAN_CUDA_RET(cudaEventCreateWithFlags(&ready_[k], cudaEventDisableTiming));
      PAWAN_CUDA_RET(cudaEventCreateWithFlags(&copied_[k], cudaEventDisableTiming));
      free_[k] = true;
    }
    thread_ = std::thread([this] { run(); });
    started_ = true;
    return PAWAN_OK;
  }

  // Snapshot of the current state as the frame at time t.
  int push(double t) {
    int k;
    {
      std::unique_lock<std::mutex> lk(mu_);
      cv_.wait(lk, [&] { return free_[next_] || failed_; });
      if (failed_) return fail(ctx_, PAWAN_ERR_INVALID, err_);
      k = next_;
      free_[k] = false;
      next_ = (next_ + 1) % kSlots;
    }
    const size_t bytes = 6 * sys_->n * sizeof(double);
    PAWAN_CUDA_RET(cudaMemcpyAsync(snap_[k].p, sys_->X.p, bytes, cudaMemcpyDeviceToDevice, ctx_->stream));
    PAWAN_CUDA_RET(cudaEventRecord(ready_[k], ctx_->stream));
    PAWAN_CUDA_RET(cudaStreamWaitEvent(copy_, ready_[k], 0));
    PAWAN_CUDA_RET(cudaMemcpyAsync(host_[k], snap_[k].p, bytes, cudaMemcpyDeviceToHost, copy_));
    PAWAN_CUDA_RET(cudaEventRecord(copied_[k], copy_));
    {
      std::lock_guard<std::mutex> lk(mu_);
      queue_.push_back({k, t});
    }
    cv_.notify_all();
    return PAWAN_OK;
  }

  // Waits for every pushed frame to be written; returns the first error.
  int finish() {
    stop();
    if (failed_) return fail(ctx_, PAWAN_ERR_INVALID, err_);
    return PAWAN_OK;
  }

 private:
  struct Job {
    int slot;
    double t;
  };

  void run() {
    const size_t N = sys_->n;
    for (;;) {
      Job j;
      {
        std::unique_lock<std::mutex> lk(mu_);
        cv_.wait(lk, [&] { return !queue_.empty() || done_; });
        if (queue_.empty()) return;
        j = queue_.front();
        queue_.pop_front();
      }
      bool ok = cudaEventSynchronize(copied_[j.slot]) == cudaSuccess;
      const double *x = host_[j.slot];
      const size_t nw = sys_->counts.size();
      ok = ok && std::fwrite(&j.t, sizeof(double), 1, f_) == 1;
      ok = ok && std::fwrite(&nw, sizeof(size_t), 1, f_) == 1;
      for (size_t w = 0; w < nw && ok; ++w) {
        const size_t o = sys_->offsets[w], c = sys_->counts[w];
        ok = ok && std::fwrite(&c, sizeof(size_t), 1, f_) == 1;
        ok = ok && std::fwrite(x + 3 * o, sizeof(double), 3 * c, f_) == 3 * c;
        ok = ok && std::fwrite(x + 3 * N + 3 * o, sizeof(double), 3 * c, f_) == 3 * c;
        ok = ok && std::fwrite(rad_.data() + o, sizeof(double), c, f_) == c;
      }
      {
        std::lock_guard<std::mutex> lk(mu_);
        free_[j.slot] = true;
        if (!ok && !failed_) {
          failed_ = true;
          err_ = "frame write failed";
        }
      }
      cv_.notify_all();
    }
  }

  void stop() {
    if (started_) {
      {
        std::lock_guard<std::mutex> lk(mu_);
        done_ = true;
      }
      cv_.notify_all();
      if (thread_.joinable()) thread_.join();
      started_ = false;
    }
    if (copy_) {
      cudaStreamSynchronize(copy_);
      cudaStreamDestroy(copy_);
      copy_ = nullptr;
    }
    for (int k = 0; k < kSlots; ++k) {
      if (host_[k]) cudaFreeHost(host_[k]);
      host_[k] = nullptr;
      if (ready_[k]) cudaEventDestroy(ready_[k]);
      if (copied_[k]) cudaEventDestroy(copied_[k]);
      ready_[k] = copied_[k] = nullptr;
      snap_[k].reset();
    }
  }

  pawan_system *sys_;
  pawan_ctx *ctx_;
  FILE *f_;
  std::vector<double> rad_;
  cudaStream_t copy_ = nullptr;
  DBuf<double> snap_[kSlots];
  double *host_[kSlots] = {};
  cudaEvent_t ready_[kSlots] = {}, copied_[kSlots] = {};
  bool free_[kSlots] = {};
  int next_ = 0;
  std::mutex mu_;
  std::condition_variable cv_;
  std::deque<Job> queue_;
  bool done_ = false, failed_ = false, started_ = false;
  std::string err_;
  std::thread thread_;
};

// Steps on the device, frames through the writer (see the file comment).
int integrate(pawan_system *sys, double T, size_t n, FILE *f, int method) {
  pawan_ctx *ctx = sys->ctx;
  if (!(T > 0.0) || n == 0) return fail(ctx, PAWAN_ERR_INVALID, "integrate needs T > 0 and n > 0");
  if (method != PAWAN_INTEGRATE_RK4 && method != PAWAN_INTEGRATE_EULER)
    return fail(ctx, PAWAN_ERR_INVALID, "unknown integration method");
  if (sys->shard.active)
    return fail(ctx, PAWAN_ERR_STATE, "system is sharded over processes");
  PAWAN_TRY(system_ensure_plan(sys));
  const double dt = T / (double)n;  // integration.cpp:11
  PAWAN_TRY(set_plan_dt(ctx, *sys->plan, nullptr, dt));
  FrameWriter w(sys, f);
  PAWAN_TRY(w.start());
  int st = w.push(0.0);
  for (size_t i = 1; i <= n && st == PAWAN_OK; ++i) {
    if (method == PAWAN_INTEGRATE_RK4) {
      st = rk4_steps(ctx, *sys->plan, 1, true);
    } else {
      st = launch_pairs(ctx, *sys->plan);
      if (st == PAWAN_OK) st = launch_stage_mode(ctx, *sys->plan, STAGE_EULER);
    }
    if (st == PAWAN_OK) st = w.push((double)i * dt);  // integration.cpp:26
  }
  const int fs = w.finish();
  if (st != PAWAN_OK) return st;
  if (fs != PAWAN_OK) return fs;
  cudaError_t e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "integrate");
  return PAWAN_OK;
}

}  // namespace

extern "C" {

int pawan_system_integrate(pawan_system *sys, double T, size_t n, const char *path, int method) {
  if (!sys || !sys->ctx) return PAWAN_ERR_INVALID;
  if (!path) return fail(sys->ctx, PAWAN_ERR_INVALID, "null path");
  if (!sys->has_particles) return fail(sys->ctx, PAWAN_ERR_STATE, "particles not set");
  FILE *f = std::fopen(path, "wb");
  if (!f) return fail(sys->ctx, PAWAN_ERR_INVALID, std::string("cannot open ") + path);
  const int st = integrate(sys, T, n, f, method);
  const bool closed = std::fclose(f) == 0;
  if (st != PAWAN_OK) return st;
  return closed ? PAWAN_OK : fail(sys->ctx, PAWAN_ERR_INVALID, std::string("cannot close ") + path);
}

int pawan_system_integrate_file(pawan_system *sys, double T, size_t n, void *file, int method) {
  if (!sys || !sys->ctx) return PAWAN_ERR_INVALID;
  if (!file) return fail(sys->ctx, PAWAN_ERR_INVALID, "null FILE");
  if (!sys->has_particles) return fail(sys->ctx, PAWAN_ERR_STATE, "particles not set");
  const int st = integrate(sys, T, n, static_cast<FILE *>(file), method);
  if (st == PAWAN_OK && std::fflush(static_cast<FILE *>(file)) != 0)
    return fail(sys->ctx, PAWAN_ERR_INVALID, "cannot flush the frame file");
  return st;
}

}  // extern "C"

// Internal declarations shared by the C ABI (abi.cu) and the solvers.
#pragma once
#include <cuda_runtime.h>

#include <cstdarg>
#include <cstdio>
#include <memory>
#include <string>
#include <vector>

#include "../../include/gerjoii_gpu.h"

namespace gj {

// Error carrier: every internal function returns a gj_status and records text.
struct Err {
  gj_status code = GJ_OK;
  std::string msg;
  gj_status set(gj_status c, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    code = c;
    msg = buf;
    return c;
  }
};

#define GJ_CUDA(err, call)                                                                   \
  do {                                                                                       \
    cudaError_t e_ = (call);                                                                 \
    if (e_ != cudaSuccess)                                                                   \
      return (err).set(e_ == cudaErrorMemoryAllocation ? GJ_ENOMEM : GJ_ECUDA, "%s: %s (%s:%d)", \
                       #call, cudaGetErrorString(e_), __FILE__, __LINE__);                   \
  } while (0)

#define GJ_TRY(x)                    \
  do {                               \
    gj_status s_ = (x);              \
    if (s_ != GJ_OK) return s_;      \
  } while (0)

// Owned device allocation.
struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  ~DevBuf() { if (p) cudaFree(p); }
  gj_status alloc(Err& err, size_t n) {
    if (n <= bytes && p) return GJ_OK;
    if (p) { cudaFree(p); p = nullptr; bytes = 0; }
    if (n == 0) return GJ_OK;
    cudaError_t e = cudaMalloc(&p, n);
    if (e != cudaSuccess) {
      cudaGetLastError();
      p = nullptr;
      return err.set(GJ_ENOMEM, "cudaMalloc(%zu bytes) failed: %s", n, cudaGetErrorString(e));
    }
    bytes = n;
    return GJ_OK;
  }
  template <class T> T* as() const { return static_cast<T*>(p); }
};

// Host-side shot description after validation (device node indices).
struct ShotHost {
  long src;                 // device linear index (i + j*ld), -1 = no source effect
  std::vector<double> wav;  // nt
  std::vector<long> rec;    // device linear indices
  std::vector<int> sel;     // receivers whose node appears last (hard-set order of w_grad.m:72)
};

class WSolverBase {
 public:
  virtual ~WSolverBase() = default;
};

// Optional per-kernel device timing: CUDA events around the launches of the
// hot kernels, summed after each call's final synchronisation.
struct KernelTimer {
  bool on = false;
  std::vector<cudaEvent_t> pool;
  size_t used = 0;
  std::vector<std::pair<int, size_t>> marks;  // (kind, first event index)
  double ms[8] = {0};
  long count[8] = {0};
  ~KernelTimer() {
    for (auto e : pool) cudaEventDestroy(e);
  }
  cudaEvent_t next() {
    if (used == pool.size()) {
      cudaEvent_t e;
      cudaEventCreate(&e);
      pool.push_back(e);
    }
    return pool[used++];
  }
  void begin(int kind, cudaStream_t st) {
    if (!on) return;
    marks.push_back({kind, used});
    cudaEventRecord(next(), st);
  }
  void end(cudaStream_t st) {
    if (!on) return;
    cudaEventRecord(next(), st);
  }
  // Call after the stream is synchronised.
  void collect() {
    for (auto& mk : marks) {
      float t = 0;
      if (cudaEventElapsedTime(&t, pool[mk.second], pool[mk.second + 1]) == cudaSuccess) {
        ms[mk.first] += t;
        count[mk.first] += 1;
      }
    }
    marks.clear();
    used = 0;
  }
  void reset() {
    for (int k = 0; k < 8; ++k) { ms[k] = 0; count[k] = 0; }
  }
};

// Kernel kinds reported by gj_kernel_time().
enum KernelKind { KK_FWD_STEP = 0, KK_REF_STEP = 1, KK_ADJ_STEP = 2, KK_IO = 3, KK_PLAIN = 4, KK_DC = 5 };

struct Ctx {
  int device = 0;
  Err err;
  long launches = 0;
  KernelTimer timer;
  std::unique_ptr<WSolverBase> wsolver;  // cached radar plan
  std::string wkey;
};

// Radar entry points implemented in w_solver.cu.
gj_status w_forward(Ctx& c, const gj_w_grid& g, gj_precision prec, const double* eps,
                    const double* sig, const gj_w_shot* shots, int nshots, double* d_out,
                    double* jz_out, double* u_out);
gj_status w_gradient(Ctx& c, const gj_w_grid& g, gj_precision prec, const void* eps,
                     const void* sig, bool dev_inputs, const gj_w_shot* shots, int nshots,
                     const void* d_obs, bool dev_dobs, gj_adj_mode mode, gj_misfit_kind mk,
                     const gj_w_opts& o, void* g_eps, void* g_sig, bool dev_out,
                     double* misfit_out, double* d_out, double* e_out, cudaStream_t stream);
gj_status w_grad_only(Ctx& c, const gj_w_grid& g, gj_precision prec, const double* eps,
                      const double* sig, const gj_w_shot& shot, const double* e, const double* u,
                      double* gout, double* amax);

}  // namespace gj

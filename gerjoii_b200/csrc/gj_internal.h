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

struct Ctx {
  int device = 0;
  Err err;
  long launches = 0;
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

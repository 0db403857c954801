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

// Device allocation, owned (cudaMalloc) or borrowed from a caller-owned pool.
struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
  bool owned = true;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  ~DevBuf() { if (p && owned) cudaFree(p); }
  // Points at n bytes of memory owned elsewhere (never freed here).
  void borrow(void* q, size_t n) {
    if (p && owned) cudaFree(p);
    p = q; bytes = n; owned = false;
  }
  gj_status alloc(Err& err, size_t n) {
    if (n <= bytes && p && owned) return GJ_OK;
    if (p && owned) cudaFree(p);
    p = nullptr; bytes = 0; owned = true;
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
  void release() {
    if (p && owned) cudaFree(p);
    p = nullptr;
    bytes = 0;
    owned = true;
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

// Cached state of gj_w_gradient_batch (plans, pool, wave graphs).
class WBatchBase {
 public:
  virtual ~WBatchBase() = default;
};

// Kernel kinds reported by gj_kernel_time().
enum KernelKind {
  KK_FWD_STEP = 0, KK_REF_STEP = 1, KK_ADJ_STEP = 2, KK_IO = 3, KK_PLAIN = 4, KK_DC_FACTOR = 5, KK_IMAGE = 6,
  KK_DC_PRECOND = 7, KK_TB_PASS = 8, KK_NKINDS = 9
};

// Optional per-kernel device timing: CUDA events around sampled launches of
// the hot kernels, also inside captured CUDA graphs (external event-record
// nodes).  The step kernels are timed in runs of `span` consecutive launches
// (one run starts at every `stride`-th launch of a kind), so the cost of the
// event records is spread over the run; a run that another timed kernel
// interrupts (the imaging kernel between adjoint steps) is dropped.  Other
// kinds are timed one launch at a time (every `stride`-th; every launch of
// the DC factor and substitution, which run a few times per call).  A Marks
// list belongs to one launch sequence (a direct enqueue, or one captured graph
// that is replayed); collect() adds its elapsed times after the stream has
// been synchronised.
struct Marks {
  std::vector<cudaEvent_t> ev;            // owned events, in pairs
  std::vector<int> kind;                  // per pair (-1: dropped run)
  std::vector<int> count;                 // per pair: launches inside it
  long launches[KK_NKINDS] = {0};         // every launch of each kind in this sequence
  long shot_launches[KK_NKINDS] = {0};    // sum of shots over those launches
  ~Marks() { for (auto e : ev) cudaEventDestroy(e); }
};

struct KernelTimer {
  bool on = false;
  int stride = 16, span = 8;
  double ms[KK_NKINDS] = {0};
  long sampled[KK_NKINDS] = {0};
  long launches[KK_NKINDS] = {0};
  long shot_launches[KK_NKINDS] = {0};
  long seen[KK_NKINDS] = {0};
  Marks* cur = nullptr;  // list receiving new marks
  int open = -1;         // kind of the run being timed, or -1
  int open_n = 0;        // launches in it so far
  static void rec(cudaEvent_t e, cudaStream_t st) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    cudaStreamIsCapturing(st, &cs);
    if (cs == cudaStreamCaptureStatusActive) cudaEventRecordWithFlags(e, st, cudaEventRecordExternal);
    else cudaEventRecord(e, st);
  }
  static bool step_kind(int k) { return k == KK_FWD_STEP || k == KK_REF_STEP || k == KK_ADJ_STEP; }
  // begin/end bracket one launch of `shots` shots; begin returns whether it is timed.
  bool begin(int kind, cudaStream_t st, int shots = 1) {
    if (!on || !cur) return false;
    cur->launches[kind] += 1;
    cur->shot_launches[kind] += shots;
    if (open >= 0 && open != kind) {  // another kernel inside the run: drop it
      rec(cur->ev.back(), st);
      cur->kind.back() = -1;
      open = -1;
    }
    if (open == kind) return true;
    const int every = (kind == KK_DC_FACTOR || kind == KK_DC_PRECOND) ? 1 : kind == KK_TB_PASS ? 4 : stride;
    if ((seen[kind]++ % every) != 0) return false;
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    cur->ev.push_back(a);
    cur->ev.push_back(b);
    cur->kind.push_back(kind);
    cur->count.push_back(0);
    rec(a, st);
    open = kind;
    open_n = 0;
    return true;
  }
  void end(bool timed, cudaStream_t st) {
    if (!timed || open < 0) return;
    cur->count.back() += 1;
    if (++open_n >= (step_kind(open) ? span : 1)) {
      rec(cur->ev.back(), st);
      open = -1;
    }
  }
  // Ends an open run (shorter than span) before the sequence ends.
  void close(cudaStream_t st) {
    if (open >= 0 && cur) rec(cur->ev.back(), st);
    open = -1;
  }
  // Adds one execution of the sequence `m` (after its stream has completed).
  void collect(const Marks& m) {
    if (!on) return;
    for (size_t q = 0; q < m.kind.size(); ++q) {
      float t = 0;
      if (m.kind[q] >= 0 && m.count[q] > 0 && cudaEventElapsedTime(&t, m.ev[2 * q], m.ev[2 * q + 1]) == cudaSuccess) {
        ms[m.kind[q]] += t;
        sampled[m.kind[q]] += m.count[q];
      }
    }
    for (int k = 0; k < KK_NKINDS; ++k) { launches[k] += m.launches[k]; shot_launches[k] += m.shot_launches[k]; }
    cudaGetLastError();
  }
  void reset() {
    for (int k = 0; k < KK_NKINDS; ++k) { ms[k] = 0; sampled[k] = 0; launches[k] = 0; shot_launches[k] = 0; seen[k] = 0; }
    open = -1;
  }
};


struct Ctx {
  int device = 0;
  Err err;
  long launches = 0;
  KernelTimer timer;
  std::unique_ptr<WSolverBase> wsolver;  // cached radar plan
  // DC band factors and CG vectors, kept between DC calls (tens of GB for a
  // survey: allocating them costs milliseconds per GB); a radar call releases
  // them before it plans its own memory.
  DevBuf dc_fac, dc_vec;
  std::string wkey;
  std::unique_ptr<WBatchBase> wbatch;  // gj_w_gradient_batch's plans and wave graphs
};

// Radar entry points implemented in w_solver.cu.
gj_status w_forward(Ctx& c, const gj_w_grid& g, gj_precision prec, const double* eps,
                    const double* sig, const gj_w_shot* shots, int nshots, double* d_out,
                    double* jz_out, double* u_out);
gj_status w_gradient(Ctx& c, const gj_w_grid& g, gj_precision prec, const void* eps,
                     const void* sig, bool dev_inputs, const gj_w_shot* shots, int nshots,
                     const void* d_obs, bool dev_dobs, gj_adj_mode mode, gj_misfit_kind mk,
                     const gj_w_opts& o, void* g_eps, void* g_sig, bool dev_out,
                     double* misfit_out, double* d_out, double* e_out, cudaStream_t stream,
                     bool e_given = false);
gj_status w_misfit(Ctx& c, const gj_w_grid& g, gj_precision prec, const double* eps, const double* sig,
                   const gj_w_shot* shots, int nshots, const double* dobs, gj_misfit_kind mk, double* misfit_out,
                   int ntrial = 1, const gj_w_opts* opts = nullptr);
gj_status w_grad_only(Ctx& c, const gj_w_grid& g, gj_precision prec, const double* eps,
                      const double* sig, const gj_w_shot& shot, const double* e, const double* u,
                      double* gout, double* amax);

gj_status w_gradient_batch(Ctx& c, gj_precision prec, const gj_w_problem* probs, int nprob, gj_adj_mode mode,
                           const gj_w_opts& o, int* nwaves_out);

// DC entry point implemented in dc_solver.cu.
gj_status dc_run(Ctx& c, const gj_dc_grid& g, const double* sigma, const gj_dc_src* srcs, int nsrc, bool grad,
                 const gj_dc_opts& o, double* d_out, double* e_out, double* u_out, double* g_out,
                 double* misfit_out, gj_dc_stats* stats, double* uk_out = nullptr);

}  // namespace gj

// gj_w_forward_noalloc: the single-shot FP32 radar forward model for callers
// that cannot allocate device memory at call time -- for example a MEX
// function running inside MATLAB, whose GPU memory belongs to MATLAB's own
// pool, or a host application that reserves the whole device up front and
// treats any later cudaMalloc as an error.  The caller passes device inputs
// and outputs; every intermediate buffer (Yee fields of both time levels,
// split PML fields, update coefficients, PML profiles, source tables) lives in
// one file-scope __device__ array of fixed size, so this path never calls
// cudaMalloc, cudaFree or any allocating library routine.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>

#include "../../include/gerjoii_gpu.h"
#include "w_kernels.cuh"

namespace gj {
namespace {

// Every GPU that loads this library keeps this array resident until exit.
constexpr size_t kNoallocScratchBytes = size_t(GJ_W_NOALLOC_SCRATCH_BYTES);
__device__ __align__(256) unsigned char g_noalloc_scratch[kNoallocScratchBytes];

// Device address of g_noalloc_scratch per device.  It is looked up again on
// every call made outside stream capture (so a context re-created after
// cudaDeviceReset gets its own address); a call made while `stream` is being
// captured uses the address of the last uncaptured call on that device.
constexpr int kMaxDevices = 64;
std::mutex g_mtx;
void* g_addr[kMaxDevices] = {nullptr};

void set_err(char* buf, size_t len, const char* msg) {
  if (buf && len) {
    std::strncpy(buf, msg, len - 1);
    buf[len - 1] = 0;
  }
}

// Host code cannot use the array's name as a device address; resolve it with
// the right device current.
gj_status scratch_address(int dev, cudaStream_t st, void** out, char* eb, size_t el) {
  if (dev < 0 || dev >= kMaxDevices) {
    set_err(eb, el, "device ordinal out of range");
    return GJ_EINVAL;
  }
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(st, &cs) != cudaSuccess) {
    cudaGetLastError();
    cs = cudaStreamCaptureStatusActive;  // treat as captured: use the cached address
  }
  std::lock_guard<std::mutex> lk(g_mtx);
  if (cs == cudaStreamCaptureStatusActive && !g_addr[dev]) {
    set_err(eb, el, "first call on this device made during stream capture: call once outside capture first");
    return GJ_EINVAL;
  }
  if (cs != cudaStreamCaptureStatusActive) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
      char m[256];
      snprintf(m, sizeof m, "cudaGetSymbolAddress(g_noalloc_scratch) failed: %s", cudaGetErrorString(e));
      set_err(eb, el, m);
      return GJ_ECUDA;
    }
    g_addr[dev] = p;
  }
  *out = g_addr[dev];
  return GJ_OK;
}

// PML profiles (w_cpml.m grading) and the source tables, computed on the device.
__global__ void k_noalloc_setup(int NX, int NY, int P, int Pt, int order, double sx, double sy, double rm,
                                double* sex, double* smx, double* sey, double* smy, long* src, long src_val) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const double Pd = P;
  if (t < NX + 2) {
    const int I = t;
    double e = 0, mm = 0;
    if (I >= 1 && I <= Pt) e = sx * pow((Pd - I + 0.25) / Pd, order);
    if (I >= 0 && I <= Pt - 1) mm = rm * sx * pow((Pd - I - 0.25) / Pd, order);
    if (I >= NX - P && I <= NX - 1) {
      const double k = I - (NX - P) + 1;
      e = sx * pow((k - 0.75) / Pd, order);
      mm = rm * sx * pow((k - 0.25) / Pd, order);
    }
    sex[I] = e; smx[I] = mm;
  }
  if (t < NY + 2) {
    const int J = t;
    double e = 0, mm = 0;
    if (J >= 1 && J <= P) e = sy * pow((Pd - J + 0.25) / Pd, order);
    if (J >= 0 && J <= P - 1) mm = rm * sy * pow((Pd - J - 0.25) / Pd, order);
    if (J >= NY - P && J <= NY - 1) {
      const double k = J - (NY - P) + 1;
      e = sy * pow((k - 0.75) / Pd, order);
      mm = rm * sy * pow((k - 0.25) / Pd, order);
    }
    sey[J] = e; smy[J] = mm;
  }
  if (t == 0) src[0] = src_val;
}

__global__ void k_noalloc_cezj(CoefBuild c, const float* eps, const float* sig, int si, int sj, float* cezj) {
  double e = 1, s = 0;
  pad_model(c, eps, sig, si, sj, e, s);
  cezj[0] = float(-(2 * c.dt) / (2 * e * c.eps0 + c.dt * s));  // w_coeff.m:44-45
}

// d[it + r*nt] = Ez(rec[r]); rec holds 0-based (NX+1)-linear node indices.
// A receiver outside the nnodes = (NX+1)(NY+1) Ez nodes is never read: its
// trace gets NaN (the host rejects such receivers before the time loop, so
// this guard only matters if the caller changes rec_dev during the call).
__global__ void k_noalloc_record(const float* Ez, int NX1, long nnodes, int ld, const long* rec, int nr, int it,
                                 int nt, float* d) {
  for (int r = threadIdx.x + blockIdx.x * blockDim.x; r < nr; r += blockDim.x * gridDim.x) {
    const long L = rec[r];
    d[size_t(it) + size_t(r) * nt] = (L >= 0 && L < nnodes) ? Ez[(L % NX1) + (L / NX1) * ld] : __int_as_float(0x7fc00000);
  }
}

// Counts receivers outside [0, nnodes) into *bad.
__global__ void k_noalloc_check_rec(const long* rec, int nr, long nnodes, int* bad) {
  for (int r = threadIdx.x + blockIdx.x * blockDim.x; r < nr; r += blockDim.x * gridDim.x)
    if (rec[r] < 0 || rec[r] >= nnodes) atomicAdd(bad, 1);
}

// NaN into every sample of the nt x nr traces (the output of a rejected call).
__global__ void k_noalloc_fill_nan(float* d, size_t n) {
  for (size_t q = threadIdx.x + size_t(blockIdx.x) * blockDim.x; q < n; q += size_t(blockDim.x) * gridDim.x)
    d[q] = __int_as_float(0x7fc00000);
}

inline size_t align256(size_t b) { return (b + 255) / 256 * 256; }

}  // namespace
}  // namespace gj

extern "C" gj_status gj_w_forward_noalloc(const gj_w_grid* grid, const float* eps_dev, const float* sigma_dev,
                                          int src_i, int src_j, const float* wavelet_dev, int nr,
                                          const long* rec_dev, float* d_out_dev, void* stream, char* errbuf,
                                          size_t errlen) {
  using namespace gj;
  set_err(errbuf, errlen, "");
  if (!grid || !eps_dev || !sigma_dev || !wavelet_dev || !d_out_dev || (nr > 0 && !rec_dev) || nr < 0) {
    set_err(errbuf, errlen, "null pointer or negative receiver count");
    return GJ_EINVAL;
  }
  const gj_w_grid& g = *grid;
  if (g.m < 3 || g.n < 3 || g.pml < 1 || g.nt < 3 || !(g.pml_top == 0 || g.pml_top == g.pml) ||
      g.air < 0 || (g.pml_top == 0 && g.air < 1) || !(g.dx > 0 && g.dy > 0 && g.dt > 0) ||
      !(g.R0 > 0 && g.R0 < 1) || !(g.eps0 > 0 && g.mu0 > 0)) {
    set_err(errbuf, errlen, "invalid grid");
    return GJ_EINVAL;
  }
  const int NX = g.pml_top + g.air + g.m + g.pml, NY = g.n + 2 * g.pml;
  if (src_i < 1 || src_i > NX - 1 || src_j < 1 || src_j > NY - 1) {
    set_err(errbuf, errlen, "source must be an updated Ez node (1..NX-1, 1..NY-1)");
    return GJ_EINVAL;
  }
  const int ld = (NX + 2 + 31) / 32 * 32;
  const size_t fstride = size_t(ld) * size_t(NY + 3);
  const size_t sstride = size_t(NFIELDS) * fstride;
  // scratch layout: 12 coefficient arrays, two states, profiles, source tables
  const size_t b_coef = align256(12 * fstride * sizeof(float));
  const size_t b_state = align256(sstride * sizeof(float));
  const size_t b_prof = align256(size_t(2 * (NX + 2) + 2 * (NY + 2)) * sizeof(double));
  const size_t need = b_coef + 2 * b_state + b_prof + 512;
  if (need > kNoallocScratchBytes) {
    char m[256];
    snprintf(m, sizeof m, "grid needs %zu bytes of scratch, above the %zu-byte limit of gj_w_forward_noalloc",
             need, kNoallocScratchBytes);
    set_err(errbuf, errlen, m);
    return GJ_EINVAL;
  }
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    set_err(errbuf, errlen, "cudaGetDevice failed");
    return GJ_ECUDA;
  }
  void* base = nullptr;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  gj_status st0 = scratch_address(dev, st, &base, errbuf, errlen);
  if (st0 != GJ_OK) return st0;
  unsigned char* p = static_cast<unsigned char*>(base);
  float* coef = reinterpret_cast<float*>(p);
  float* stA = reinterpret_cast<float*>(p + b_coef);
  float* stB = reinterpret_cast<float*>(p + b_coef + b_state);
  double* prof = reinterpret_cast<double*>(p + b_coef + 2 * b_state);
  long* d_src = reinterpret_cast<long*>(p + b_coef + 2 * b_state + b_prof);
  float* d_cezj = reinterpret_cast<float*>(d_src + 1);
  int* d_bad = reinterpret_cast<int*>(p + b_coef + 2 * b_state + b_prof + 256);
  const long nnodes = long(NX + 1) * long(NY + 1);

  // Receivers must be Ez nodes of the padded grid.  They are device data, so
  // they are checked on the device and the count read back (this waits for
  // the work already queued on `stream`).  Rejected calls return GJ_EINVAL
  // with NaN in every trace sample.
  if (nr > 0) {
    int bad = 0;
    if (cudaMemsetAsync(d_bad, 0, sizeof(int), st) != cudaSuccess) {
      set_err(errbuf, errlen, "cudaMemsetAsync on the scratch array failed");
      return GJ_ECUDA;
    }
    k_noalloc_check_rec<<<(nr + 255) / 256, 256, 0, st>>>(rec_dev, nr, nnodes, d_bad);
    if (cudaMemcpyAsync(&bad, d_bad, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess) {
      set_err(errbuf, errlen, "reading the receiver check back failed");
      return GJ_ECUDA;
    }
    if (bad > 0) {
      k_noalloc_fill_nan<<<64, 256, 0, st>>>(d_out_dev, size_t(nr) * size_t(g.nt));
      char m[256];
      snprintf(m, sizeof m, "%d receiver(s) outside the (NX+1)x(NY+1) = %ld Ez nodes", bad, nnodes);
      set_err(errbuf, errlen, m);
      return GJ_EINVAL;
    }
  }

  // Everything that must start at zero is cleared on every call: the array
  // keeps whatever the previous call left in it.
  if (cudaMemsetAsync(p, 0, b_coef + 2 * b_state, st) != cudaSuccess) {
    set_err(errbuf, errlen, "cudaMemsetAsync on the scratch array failed");
    return GJ_ECUDA;
  }
  WDev<float> w{};
  w.NX = NX; w.NY = NY; w.ld = ld; w.P = g.pml; w.Pt = g.pml_top; w.m = g.m; w.n = g.n;
  w.di0 = g.pml_top + g.air; w.dj0 = g.pml;
  w.hr0 = w.di0 / 4 * 4; w.hld = (w.di0 + g.m + 3) / 4 * 4 - w.hr0;
  w.ei0 = g.pml_top + 1; w.ei1 = NX - g.pml - 1; w.ej0 = g.pml + 1; w.ej1 = NY - g.pml - 1;
  w.hyi0 = g.pml_top; w.hyi1 = NX - g.pml - 1; w.hxj0 = g.pml; w.hxj1 = NY - g.pml - 1;
  w.chxez = float(-(2 * g.dt / g.dy) / (2 * g.mu0));
  w.chyez = float((2 * g.dt / g.dx) / (2 * g.mu0));
  w.rxy = float(-g.dx / g.dy);
  float* arr[12];
  for (int q = 0; q < 12; ++q) arr[q] = coef + ld + q * fstride;
  w.ce = arr[0]; w.chy = arr[1]; w.ax = arr[2]; w.bx = arr[3]; w.ay = arr[4]; w.by = arr[5];
  w.hxa = arr[6]; w.hxb = arr[7]; w.hya = arr[8]; w.hyb = arr[9];

  const bool interior = src_i >= g.pml_top + 1 && src_i <= NX - g.pml - 1 && src_j >= g.pml + 1 &&
                        src_j <= NY - g.pml - 1;
  const long src_lin = interior ? long(src_i) + long(src_j) * ld : -1;  // PML-band sources have no effect
  const double c0 = 1.0 / std::sqrt(g.mu0 * g.eps0);
  const double sx = -(g.order + 1) * g.eps0 * c0 * std::log(g.R0) / (2.0 * g.dx * g.pml);
  const double sy = -(g.order + 1) * g.eps0 * c0 * std::log(g.R0) / (2.0 * g.dy * g.pml);
  double* sex = prof; double* smx = sex + NX + 2; double* sey = smx + NX + 2; double* smy = sey + NY + 2;
  const int nset = std::max(NX, NY) + 2;
  k_noalloc_setup<<<(nset + 127) / 128, 128, 0, st>>>(NX, NY, g.pml, g.pml_top, g.order, sx, sy, g.mu0 / g.eps0,
                                                      sex, smx, sey, smy, d_src, src_lin);
  CoefBuild cb;
  cb.NX = NX; cb.NY = NY; cb.ld = ld; cb.P = g.pml; cb.Pt = g.pml_top; cb.air = g.air; cb.m = g.m; cb.n = g.n;
  cb.dx = g.dx; cb.dy = g.dy; cb.dt = g.dt; cb.eps0 = g.eps0; cb.mu0 = g.mu0;
  cb.sex = sex; cb.smx = smx; cb.sey = sey; cb.smy = smy;
  k_build_coefs<float, float><<<dim3((NX + 1 + 31) / 32, (NY + 1 + 7) / 8), dim3(32, 8), 0, st>>>(
      cb, eps_dev, sigma_dev, arr[0], arr[1], arr[2], arr[3], arr[4], arr[5], arr[6], arr[7], arr[8], arr[9],
      arr[10], arr[11], nullptr, nullptr);
  k_noalloc_cezj<<<1, 1, 0, st>>>(cb, eps_dev, sigma_dev, src_i, src_j, d_cezj);
  // time loop (w_solve.m:80-105) with the same fused step as gj_w_forward
  float* A = stA + ld;
  float* B = stB + ld;
  const int bx = 128, tj = 16;
  const dim3 grd((ld + bx - 1) / bx, (NY + 1 + tj - 1) / tj, 1);
  for (int it = 0; it < g.nt; ++it) {
    StepArgs<float> a{};
    a.A = A; a.B = B; a.fstride = fstride; a.sstride = sstride; a.shot0 = 0; a.tj = tj; a.it = it;
    a.src = d_src; a.cezj = d_cezj; a.wav = wavelet_dev; a.nt = g.nt; a.hist = nullptr; a.kahan = 1;
    k_step<float, 0><<<grd, bx, 0, st>>>(w, a);
    if (nr > 0)
      k_noalloc_record<<<(nr + 127) / 128, 128, 0, st>>>(B, NX + 1, nnodes, ld, rec_dev, nr, it, g.nt, d_out_dev);
    float* t = A; A = B; B = t;
  }
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_err(errbuf, errlen, cudaGetErrorString(e));
    return GJ_ECUDA;
  }
  return GJ_OK;
}

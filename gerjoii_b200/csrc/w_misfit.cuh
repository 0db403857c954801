// Envelope (env_L2) adjoint source and misfit on the device (w_bozdag.m:51-60,
// instant_.m:14-20, w_E.m with d and d_o replaced by their envelopes,
// w_update_e.m:75-76):
//   E = |analytic(d)|, Eo = |analytic(d_o)|, Hd = imag(analytic(d))
//   f = (E - Eo) / E,  e = d f - imag(analytic(f Hd)),  e(NaN) = 0
//   misfit = 0.5 sum (E - Eo)^2 / sum Eo^2.
// The analytic signal follows MATLAB's hilbert: FFT along time, keep DC and
// Nyquist, double positive frequencies, zero negative ones, inverse FFT.
#pragma once
#include <cuComplex.h>
#include <cuda_runtime.h>
#include <cufft.h>

namespace gj {

template <class T> struct CplxT;
template <> struct CplxT<float> { using type = cuComplex; };
template <> struct CplxT<double> { using type = cuDoubleComplex; };

__device__ __forceinline__ void cset(cuComplex& c, float re, float im) { c = make_cuComplex(re, im); }
__device__ __forceinline__ void cset(cuDoubleComplex& c, double re, double im) { c = make_cuDoubleComplex(re, im); }
__device__ __forceinline__ float cre(const cuComplex& c) { return c.x; }
__device__ __forceinline__ float cim(const cuComplex& c) { return c.y; }
__device__ __forceinline__ double cre(const cuDoubleComplex& c) { return c.x; }
__device__ __forceinline__ double cim(const cuDoubleComplex& c) { return c.y; }

// real traces [trace][t] -> complex
template <class T, class C>
__global__ void k_env_to_complex(const T* x, C* y, size_t n) {
  for (size_t i = threadIdx.x + size_t(blockIdx.x) * blockDim.x; i < n; i += size_t(blockDim.x) * gridDim.x)
    cset(y[i], x[i], T(0));
}

// spectrum -> analytic-signal spectrum, with the 1/nt of the inverse FFT folded in
template <class T, class C>
__global__ void k_env_mask(C* X, int nt, size_t ntr) {
  const size_t n = size_t(nt) * ntr;
  const T inv = T(1) / T(nt);
  for (size_t i = threadIdx.x + size_t(blockIdx.x) * blockDim.x; i < n; i += size_t(blockDim.x) * gridDim.x) {
    const int k = int(i % nt);
    T h;
    if (k == 0) h = T(1);
    else if (nt % 2 == 0 && k == nt / 2) h = T(1);
    else if (k < (nt + 1) / 2) h = T(2);
    else h = T(0);
    cset(X[i], cre(X[i]) * h * inv, cim(X[i]) * h * inv);
  }
}

// From the analytic signals of d (A) and d_o (Ao): f into F, f*Hd into G
// (complex, for the second Hilbert transform), misfit sums per shot.
template <class T, class C>
__global__ void k_env_mid(const C* A, const C* Ao, T* F, C* G, int nt, int ntr_per_shot, int nshots,
                          double* sums) {
  const int s = blockIdx.y;
  if (s >= nshots) return;
  const size_t per = size_t(nt) * ntr_per_shot, base = size_t(s) * per;
  double num = 0, den = 0;
  for (size_t i = threadIdx.x + size_t(blockIdx.x) * blockDim.x; i < per; i += size_t(blockDim.x) * gridDim.x) {
    const C a = A[base + i], ao = Ao[base + i];
    const T E = sqrt(cre(a) * cre(a) + cim(a) * cim(a));
    const T Eo = sqrt(cre(ao) * cre(ao) + cim(ao) * cim(ao));
    const T f = (E - Eo) / E;  // NaN where E = 0 (zeroed at the end, w_bozdag.m:60)
    F[base + i] = f;
    cset(G[base + i], f * cim(a), T(0));
    num += double(E - Eo) * double(E - Eo);
    den += double(Eo) * double(Eo);
  }
  for (int o = 16; o > 0; o >>= 1) {
    num += __shfl_down_sync(0xffffffffu, num, o);
    den += __shfl_down_sync(0xffffffffu, den, o);
  }
  if ((threadIdx.x & 31) == 0) {
    atomicAdd(sums + 2 * s, num);
    atomicAdd(sums + 2 * s + 1, den);
  }
}

// e = d f - imag(analytic(f Hd)), NaN -> 0
template <class T, class C>
__global__ void k_env_final(const T* d, const T* F, const C* HG, T* e, size_t n) {
  for (size_t i = threadIdx.x + size_t(blockIdx.x) * blockDim.x; i < n; i += size_t(blockDim.x) * gridDim.x) {
    const T v = d[i] * F[i] - cim(HG[i]);
    e[i] = isnan(v) ? T(0) : v;
  }
}

// ---------------------------------------------------------------------------
// Gaussian band filter of residual traces (filt_gauss.m:16-47, applied to
// e_2d in w_update_e.m:69-70): Tukey(0.1) taper, zero padding to ntp = 2^k,
// FFT, product with the fftshift-ed Gaussian, inverse FFT, real part, trim.
// The taper (nt) and the filter (ntp, with the 1/ntp of the inverse FFT folded
// in) are computed on the host in double.

// traces [trace][t] (nt) -> tapered, zero-padded complex [trace][k] (ntp)
template <class T, class C>
__global__ void k_filt_pre(const T* e, const T* win, C* X, int nt, int ntp, size_t ntr) {
  const size_t n = size_t(ntp) * ntr;
  for (size_t i = threadIdx.x + size_t(blockIdx.x) * blockDim.x; i < n; i += size_t(blockDim.x) * gridDim.x) {
    const int k = int(i % ntp);
    const size_t tr = i / ntp;
    cset(X[i], k < nt ? e[tr * nt + k] * win[k] : T(0), T(0));
  }
}

template <class T, class C>
__global__ void k_filt_mul(C* X, const T* G, int ntp, size_t ntr) {
  const size_t n = size_t(ntp) * ntr;
  for (size_t i = threadIdx.x + size_t(blockIdx.x) * blockDim.x; i < n; i += size_t(blockDim.x) * gridDim.x) {
    const T gk = G[i % ntp];
    cset(X[i], cre(X[i]) * gk, cim(X[i]) * gk);
  }
}

template <class T, class C>
__global__ void k_filt_post(const C* X, T* e, int nt, int ntp, size_t ntr) {
  const size_t n = size_t(nt) * ntr;
  for (size_t i = threadIdx.x + size_t(blockIdx.x) * blockDim.x; i < n; i += size_t(blockDim.x) * gridDim.x) {
    const size_t tr = i / nt;
    const int t = int(i % nt);
    e[i] = cre(X[tr * ntp + t]);
  }
}

}  // namespace gj

// Envelope and phase adjoint sources and misfits on the device (w_bozdag.m:16-54,
// instant_.m:14-20; w_E.m:7-16 on the envelopes or phases that w_fwd.m:34-35
// stores in place of d and d_o; normalised as w_update_e.m:75-76):
//   E = |analytic(d)|, Eo = |analytic(d_o)|, Hd = imag(analytic(d)),
//   phi, phi_o the angles of the analytic signals, H = imag(analytic(.))
//   env_L2  : f = (E - Eo) / E,        e = d f - H(f Hd),          e(NaN) = 0,
//             misfit 0.5 sum (E - Eo)^2 / sum Eo^2
//   phase_L2: g = (phi - phi_o) / E^2, e = -g + H(g d),
//             misfit 0.5 sum (phi - phi_o)^2 / sum phi_o^2
//   env_L22 : f = E^2 - Eo^2,          e = d f - H(f Hd),
//             misfit 0.5 sum (E^2 - Eo^2)^2 / sum Eo^2
//   env_LOG : f = log(Eo / E),         e = -f d / E^2 + H(f Hd / E^2), e(NaN) = 0,
//             misfit 0.5 sum (log E - log Eo)^2 / sum Eo^2
// The analytic signal follows MATLAB's hilbert: FFT along time, keep DC and
// Nyquist, double positive frequencies, zero negative ones, inverse FFT.
#pragma once
#include <cuComplex.h>
#include <cuda_runtime.h>
#include <cufft.h>

namespace gj {

// misfit kinds, as gj_misfit_kind
constexpr int MK_ENV_L2 = 1, MK_PHASE_L2 = 2, MK_ENV_L22 = 3, MK_ENV_LOG = 4;

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

// From the traces d and the analytic signals of d (A) and d_o (Ao): the
// pointwise factor into F and the operand of the second Hilbert transform into
// G (complex), misfit sums per shot; `kind` as gj_misfit_kind.
template <class T, class C>
__global__ void k_env_mid(const T* d, const C* A, const C* Ao, T* F, C* G, int nt, int ntr_per_shot, int nshots,
                          int kind, double* sums) {
  const int s = blockIdx.y;
  if (s >= nshots) return;
  const size_t per = size_t(nt) * ntr_per_shot, base = size_t(s) * per;
  double num = 0, den = 0;
  for (size_t i = threadIdx.x + size_t(blockIdx.x) * blockDim.x; i < per; i += size_t(blockDim.x) * gridDim.x) {
    const C a = A[base + i], ao = Ao[base + i];
    const T E = sqrt(cre(a) * cre(a) + cim(a) * cim(a));
    const T Eo = sqrt(cre(ao) * cre(ao) + cim(ao) * cim(ao));
    T f, g;
    double r;
    if (kind == MK_PHASE_L2) {
      const T ph = atan2(cim(a), cre(a)), pho = atan2(cim(ao), cre(ao));
      f = (ph - pho) / (E * E);
      g = f * d[base + i];
      r = double(ph - pho);
      den += double(pho) * double(pho);
    } else {
      if (kind == MK_ENV_L22) {
        f = E * E - Eo * Eo;
        g = f * cim(a);
        r = double(f);
      } else if (kind == MK_ENV_LOG) {
        f = log(Eo / E) / (E * E);  // NaN / inf where E = 0 (zeroed at the end, w_bozdag.m:54)
        g = f * cim(a);
        r = double(log(E)) - double(log(Eo));
      } else {
        f = (E - Eo) / E;  // NaN where E = 0 (zeroed at the end, w_bozdag.m:25)
        g = f * cim(a);
        r = double(E - Eo);
      }
      den += double(Eo) * double(Eo);
    }
    F[base + i] = f;
    cset(G[base + i], g, T(0));
    num += r * r;
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

// The adjoint source from F and HG = analytic(G) (formulas above).
template <class T, class C>
__global__ void k_env_final(const T* d, const T* F, const C* HG, T* e, size_t n, int kind) {
  for (size_t i = threadIdx.x + size_t(blockIdx.x) * blockDim.x; i < n; i += size_t(blockDim.x) * gridDim.x) {
    if (kind == MK_PHASE_L2) {
      e[i] = -F[i] + cim(HG[i]);
    } else if (kind == MK_ENV_L22) {
      e[i] = d[i] * F[i] - cim(HG[i]);
    } else if (kind == MK_ENV_LOG) {
      const T v = -F[i] * d[i] + cim(HG[i]);
      e[i] = isnan(v) ? T(0) : v;
    } else {
      const T v = d[i] * F[i] - cim(HG[i]);
      e[i] = isnan(v) ? T(0) : v;
    }
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

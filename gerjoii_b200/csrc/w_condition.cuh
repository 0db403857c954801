// Per-shot conditioning of the radar gradients before they are averaged over
// shots (w_update_e.m:99-137 for eps, w_update_s.m:96-137 for sigma,
// averaged in w_update_e_.m:38 / w_update_s_.m:38):
//   1. source taper (gaussi.m): g *= normali(1 - exp(-(dx^2 + dz^2) / L^2)),
//      L = 2 * (2 * lo), lo = c / sqrt(eps_r(source)) / fo
//   2. k-space low-pass (image_gaussian.m, 'LOW_PASS'): zero padding to
//      powers of two, 2-D FFT, product with the fftshift-ed Gaussian, inverse
//      FFT, real part, trim
//   3. normali.m: divide by max |g| (1 when that is 0)
//   4. NaN guard (w_update_e.m:131-135): a shot with a NaN gets a zero gradient
// All in double on per-shot m x n column-major gradients.
#pragma once
#include <cuComplex.h>
#include <cuda_runtime.h>

namespace gj {

// par: per shot {a_s, b_s, L, 1 / max taper}
__global__ void k_cond_taper(double* g, int nshots, int m, int n, double dx, double dz, const double* par) {
  const size_t mn = size_t(m) * n, tot = mn * nshots;
  for (size_t i = threadIdx.x + size_t(blockIdx.x) * blockDim.x; i < tot; i += size_t(blockDim.x) * gridDim.x) {
    const int s = int(i / mn);
    const size_t p = i % mn;
    const int a = int(p % m), b = int(p / m);
    const double* q = par + 4 * s;
    const double xa = (b - q[1]) * dx / q[2], za = (a - q[0]) * dz / q[2];
    g[i] *= (1.0 - exp(-(xa * xa + za * za))) * q[3];
  }
}

// g [shot][m x n] -> zero-padded complex [shot][m_ x n_] (column-major, a fastest)
__global__ void k_cond_pad(const double* g, cuDoubleComplex* X, int nshots, int m, int n, int m_, int n_) {
  const size_t per = size_t(m_) * n_, tot = per * nshots;
  for (size_t i = threadIdx.x + size_t(blockIdx.x) * blockDim.x; i < tot; i += size_t(blockDim.x) * gridDim.x) {
    const int s = int(i / per);
    const size_t p = i % per;
    const int a = int(p % m_), b = int(p / m_);
    const double v = (a < m && b < n) ? g[size_t(s) * m * n + a + size_t(b) * m] : 0.0;
    X[i] = make_cuDoubleComplex(v, 0.0);
  }
}

__global__ void k_cond_mul(cuDoubleComplex* X, const double* F, size_t per, int nshots) {
  const size_t tot = per * nshots;
  for (size_t i = threadIdx.x + size_t(blockIdx.x) * blockDim.x; i < tot; i += size_t(blockDim.x) * gridDim.x) {
    const double f = F[i % per];
    X[i] = make_cuDoubleComplex(cuCreal(X[i]) * f, cuCimag(X[i]) * f);
  }
}

__global__ void k_cond_trim(const cuDoubleComplex* X, double* g, int nshots, int m, int n, int m_, int n_) {
  const size_t mn = size_t(m) * n, tot = mn * nshots;
  for (size_t i = threadIdx.x + size_t(blockIdx.x) * blockDim.x; i < tot; i += size_t(blockDim.x) * gridDim.x) {
    const int s = int(i / mn);
    const size_t p = i % mn;
    const int a = int(p % m), b = int(p / m);
    g[i] = cuCreal(X[size_t(s) * m_ * n_ + a + size_t(b) * m_]);
  }
}

// One block per shot: max |g| and a NaN flag, then g /= max (or 0 on NaN).
__global__ void k_cond_norm(double* g, size_t mn) {
  __shared__ double smax[32];
  __shared__ int snan[32];
  double* G = g + size_t(blockIdx.x) * mn;
  double mx = 0.0;
  int nan = 0;
  for (size_t i = threadIdx.x; i < mn; i += blockDim.x) {
    const double v = G[i];
    if (isnan(v)) nan = 1;
    else mx = fmax(mx, fabs(v));
  }
  for (int o = 16; o > 0; o >>= 1) {
    mx = fmax(mx, __shfl_down_sync(0xffffffffu, mx, o));
    nan |= __shfl_down_sync(0xffffffffu, nan, o);
  }
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) { smax[wid] = mx; snan[wid] = nan; }
  __syncthreads();
  if (wid == 0) {
    const int nw = blockDim.x >> 5;
    mx = lane < nw ? smax[lane] : 0.0;
    nan = lane < nw ? snan[lane] : 0;
    for (int o = 16; o > 0; o >>= 1) {
      mx = fmax(mx, __shfl_down_sync(0xffffffffu, mx, o));
      nan |= __shfl_down_sync(0xffffffffu, nan, o);
    }
    if (lane == 0) { smax[0] = mx; snan[0] = nan; }
  }
  __syncthreads();
  const double scale = snan[0] ? 0.0 : 1.0 / (smax[0] == 0.0 ? 1.0 : smax[0]);
  for (size_t i = threadIdx.x; i < mn; i += blockDim.x) G[i] = snan[0] ? 0.0 : G[i] * scale;
}

// out[p] = sum_s g[s][p] / nshots
__global__ void k_shot_mean(const double* g, int nshots, size_t mn, double* out) {
  for (size_t p = threadIdx.x + size_t(blockIdx.x) * blockDim.x; p < mn; p += size_t(blockDim.x) * gridDim.x) {
    double sacc = 0.0;
    for (int s = 0; s < nshots; ++s) sacc += g[size_t(s) * mn + p];
    out[p] = sacc / nshots;
  }
}

}  // namespace gj

// PML band terms of the exact gradient.
//
// w_exp2pml.m:21-33 replicates the model's edge columns and bottom row of
// eps_r into the PML, and w_cpml.m builds the split-field coefficients of the
// bottom and lateral strips from that eps_r (Ezx: w_cpml.m:93-96, 133-134,
// 174-175; Ezy: w_cpml.m:103-104, 141-144, 182-185; Hx: w_cpml.m:123-126,
// 164-167; Hy bottom: w_cpml.m:83).  So dJ/d(eps_r) of the model's first and
// last column and of its last row collects, besides the interior imaging
// condition, the derivatives of those PML coefficients.  Per band node and
// time step they are (forward values before (0) and after (1) the step,
// adjoint values of that step):
//   Ezx:  lx (Ezx1 - Ezx0) * (-2 eps0 / (2 eps0 eps + dt sex))   bottom strip
//         lx (Ezx1 - Ezx0) * (-1 / eps)                          lateral strips
//   Ezy:  ly (Ezy1 - Ezy0) * (-2 eps0 / (2 eps0 eps + dt sey))   lateral strips
//         ly (Ezy1 - Ezy0) * (-1 / eps)                          bottom strip
//   Hx:   ltx (Hx1 + Hx0) * dt sm / (eps (2 mu0 + dt sm)), sm = smy / eps
//   Hy:   lty (Hy1 + Hy0) * dt sm / (eps (2 mu0 + dt sm)), sm = smx / eps (bottom)
// with lx = lEzx + lE, ly = lEzy + lE, ltx = lHx + py(j) - py(j+1),
// lty = lHy + px(i) - px(i+1) the transposed update's intermediate values.
//
// The forward stores the band fields of every step in a band history (the
// band frame of WDev: two row-contiguous rectangles), the adjoint stores its
// band values in a ring of slots, k_image_band correlates them, and
// k_band_finish maps every band node onto the model cell whose eps_r it
// replicates (the transpose of w_exp2pml.m).
#pragma once
#include "w_kernels.cuh"
#include "w_kernels_vec.cuh"

namespace gj {

template <class T>
inline void band_geometry(WDev<T>& w) {
  w.bR0 = (w.NX - w.P) / 4 * 4;
  w.bRB = (w.NX + 3) / 4 * 4;
  w.bBh = w.bRB - w.bR0;
  w.bLsz = long(w.bRB) * 2 * (w.P + 1);
  w.bBsz = long(w.bBh) * (w.NY + 1);
  w.bsz = 3 * (w.bLsz + w.bBsz);
}

template <class T>
__device__ __forceinline__ bool ez_interior(const WDev<T>& w, int I, int J) {
  return I >= w.ei0 && I <= w.ei1 && J >= w.ej0 && J <= w.ej1;
}
template <class T>
__device__ __forceinline__ bool ez_bandnode(const WDev<T>& w, int I, int J) {
  return I >= 1 && I <= w.NX - 1 && J >= 1 && J <= w.NY - 1 && !ez_interior(w, I, J);
}

// Entry q of a band slot: its plane (0 Ezx, 1 Ezy, 2 Hx, 3 Hy; -1 = an
// unused entry: lateral E planes of rows >= bR0) and node (I, J).
template <class T>
__device__ __forceinline__ int band_node(const WDev<T>& w, long q, int& I, int& J) {
  if (q < 3 * w.bLsz) {
    const int p = int(q / w.bLsz);
    const long r = q - p * w.bLsz;
    I = int(r % w.bRB);
    const int cl = int(r / w.bRB);
    J = cl <= w.P ? cl : w.NY - w.P + (cl - w.P - 1);
    if (p < 2) return I < w.bR0 ? p : -1;
    return 2;
  }
  const long q2 = q - 3 * w.bLsz;
  const int p = int(q2 / w.bBsz);
  const long r = q2 - p * w.bBsz;
  I = w.bR0 + int(r % w.bBh);
  J = int(r / w.bBh);
  return p < 2 ? p : 3;
}

template <class T>
__device__ __forceinline__ long band_lat_col(const WDev<T>& w, int J) {
  if (J >= 0 && J <= w.P) return J;
  if (J >= w.NY - w.P && J <= w.NY) return J - (w.NY - w.P) + w.P + 1;
  return -1;
}
// Offsets of node (I, J) in a band slot; -1 when the frame does not hold it.
template <class T>
__device__ __forceinline__ long band_off_e(const WDev<T>& w, int I, int J, int p) {
  if (I >= w.bR0) return 3 * w.bLsz + p * w.bBsz + (I - w.bR0) + long(J) * w.bBh;
  const long cl = band_lat_col(w, J);
  return cl < 0 ? -1 : p * w.bLsz + I + cl * w.bRB;
}
template <class T>
__device__ __forceinline__ long band_off_hx(const WDev<T>& w, int I, int J) {
  const long cl = band_lat_col(w, J);
  return cl < 0 ? -1 : 2 * w.bLsz + I + cl * w.bRB;
}
template <class T>
__device__ __forceinline__ long band_off_hy(const WDev<T>& w, int I, int J) {
  return I < w.bR0 ? -1 : 3 * w.bLsz + 2 * w.bBsz + (I - w.bR0) + long(J) * w.bBh;
}

// Band fields of a forward state (after a step) into one history slot per
// shot: Ezx, Ezy at band nodes (0 elsewhere), Hx, Hy as stored.
// Grid: x = grid-stride over the slot, y = shots.
template <class T>
__global__ void k_band_rec(const WDev<T> w, const T* state, size_t sstride, size_t fstride, T* slot) {
  const int zl = blockIdx.y;
  const T* Ez = state + size_t(zl) * sstride;
  const T* Hx = Ez + fstride;
  const T* Hy = Ez + 2 * fstride;
  const T* Ex = Ez + 3 * fstride;
  const T* Ey = Ez + 4 * fstride;
  T* out = slot + size_t(zl) * w.bsz;
  for (long q = threadIdx.x + long(blockIdx.x) * blockDim.x; q < w.bsz; q += long(blockDim.x) * gridDim.x) {
    int I, J;
    const int p = band_node(w, q, I, J);
    T v = T(0);
    if (p >= 0) {
      const size_t k = nidx(I, J, w.ld);
      if (p == 0) v = ez_bandnode(w, I, J) ? Ex[k] : T(0);
      else if (p == 1) v = ez_bandnode(w, I, J) ? Ey[k] : T(0);
      else if (p == 2) v = Hx[k];
      else v = Hy[k];
    }
    out[q] = v;
  }
}

// Band values of the transposed update of one step, from the adjoint state
// before that step (after the injection of its adjoint source): lx, ly at band
// E nodes, ltx at Hx nodes, lty at Hy nodes.  Same grid as k_band_rec.
template <class T>
__global__ void k_band_adj(const WDev<T> w, const T* state, size_t sstride, size_t fstride, T* slot) {
  const int zl = blockIdx.y;
  const T* L = state + size_t(zl) * sstride;
  const T* Lx = L + fstride;
  const T* Ly = L + 2 * fstride;
  const T* Sx = L + 3 * fstride;
  const T* Sy = L + 4 * fstride;
  const int ld = w.ld;
  T* out = slot + size_t(zl) * w.bsz;
  for (long q = threadIdx.x + long(blockIdx.x) * blockDim.x; q < w.bsz; q += long(blockDim.x) * gridDim.x) {
    int I, J;
    const int p = band_node(w, q, I, J);
    T v = T(0);
    const size_t k = nidx(I, J, ld);
    if (p == 0 || p == 1) {
      if (ez_bandnode(w, I, J)) v = (p == 0 ? Sx[k] : Sy[k]) + L[k];
    } else if (p == 2) {
      if (I <= w.NX && J <= w.NY - 1) {
        T px, py0, py1, lm, lx, ly;
        adj_p(w, I, J, k, L[k], Sx[k], Sy[k], px, py0, lm, lx, ly);
        adj_p(w, I, J + 1, k + ld, L[k + ld], Sx[k + ld], Sy[k + ld], px, py1, lm, lx, ly);
        v = Lx[k] + py0 - py1;
      }
    } else if (p == 3) {
      if (I <= w.NX - 1) {
        T px0, px1, py, lm, lx, ly;
        adj_p(w, I, J, k, L[k], Sx[k], Sy[k], px0, py, lm, lx, ly);
        adj_p(w, I + 1, J, k + 1, L[k + 1], Sx[k + 1], Sy[k + 1], px1, py, lm, lx, ly);
        v = Ly[k] + px0 - px1;
      }
    }
    out[q] = v;
  }
}

// Band imaging over a window of cnt adjoint steps: slot r of the adjoint band
// ring holds step k = kA - r, the band history slot of step k sits at
// Fk0 - r * hsl.  S += sum_r lam_r (F^k - F^{k-1}) on the E planes and
// lam_r (F^k + F^{k-1}) on the H planes, compensated when kahan.
// Accumulators per shot: [sum | compensation], bsz each.
template <class T>
__global__ void k_image_band(const WDev<T> w, const T* lam, size_t lsl, const T* Fk0, size_t hsl, int cnt, T* bacc,
                             size_t bstride, int shot0, int kahan) {
  const int zl = blockIdx.y;
  const int s = shot0 + zl;
  for (long q = threadIdx.x + long(blockIdx.x) * blockDim.x; q < w.bsz; q += long(blockDim.x) * gridDim.x) {
    int I, J;
    const int p = band_node(w, q, I, J);
    if (p < 0) continue;
    const T sg = p >= 2 ? T(1) : T(-1);
    const T* L = lam + size_t(zl) * w.bsz + q;
    const T* F = Fk0 + size_t(zl) * w.bsz + q;
    T fh = F[0], acc = T(0);
    for (int r = 0; r < cnt; ++r) {
      const T fl = *(F - size_t(r + 1) * hsl);
      acc += L[size_t(r) * lsl] * (fh + sg * fl);
      fh = fl;
    }
    T* A = bacc + size_t(s) * bstride + q;
    if (kahan) {
      T sum = A[0], comp = A[w.bsz];
      kahan_add(&sum, &comp, acc);
      A[0] = sum;
      A[w.bsz] = comp;
    } else {
      A[0] += acc;
    }
  }
}

struct BandFinish {
  double dt, eps0, mu0;
  int Pt, air;
  const double* eps_m;  // model eps_r, m x n
  const double* sex; const double* smx; const double* sey; const double* smy;  // PML profiles
};

// Adds the band terms to g_eps (double, m x n per shot with per_shot, else
// summed): every model cell on the edges gathers the nodes of its preimage
// under w_exp2pml.m (the PML rows and columns that replicate it).  One warp
// per model cell (warp-uniform skip of the cells off the edges); the lanes
// stride over the preimage and a fixed-order shuffle reduction keeps the sum
// deterministic.
template <class T>
__global__ void k_band_finish(const WDev<T> w, const T* bacc, size_t bstride, int nshots, int per_shot,
                              const BandFinish f, double* geps) {
  const int m = w.m, n = w.n, NX = w.NX, NY = w.NY, P = w.P;
  const size_t mn = size_t(m) * n;
  const int lane = threadIdx.x & 31;
  const size_t warp = (size_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  const size_t nwarps = (size_t(gridDim.x) * blockDim.x) >> 5;
  for (size_t p = warp; p < mn; p += nwarps) {
    const int a = int(p % m), b = int(p / m);
    const bool top = a == 0 && f.air == 0 && f.Pt > 0;
    if (!(b == 0 || b == n - 1 || a == m - 1 || top)) continue;
    int I0 = f.Pt + f.air + a, I1 = I0, J0 = P + b, J1 = J0;
    if (a == m - 1) I1 = NX - 1;
    if (top) I0 = 0;
    if (b == 0) J0 = 0;
    if (b == n - 1) J1 = NY - 1;
    const int ni = I1 - I0 + 1, cnt = ni * (J1 - J0 + 1);
    const double eps = f.eps_m[p], e0 = f.eps0, dt = f.dt, u0 = f.mu0;
    double tot = 0.0;
    for (int s = 0; s < nshots; ++s) {
      const T* A = bacc + size_t(s) * bstride;
      auto S = [&](long q) { return double(A[q]) - double(A[w.bsz + q]); };
      double g = 0.0;
      for (int q = lane; q < cnt; q += 32) {
        const int I = I0 + q % ni, J = J0 + q / ni;
        const bool xbot = I >= NX - P && I <= NX - 1;
        const bool xtop = I >= 1 && I <= f.Pt;
        const bool ystrip = (J >= 1 && J <= P) || (J >= NY - P && J <= NY - 1);
        if (ez_bandnode(w, I, J)) {
          double cx = 0.0, cy = 0.0;
          if (xbot) cx = -2.0 * e0 / (2.0 * e0 * eps + dt * f.sex[I]);
          else if (!xtop) cx = -1.0 / eps;
          if (ystrip) cy = -2.0 * e0 / (2.0 * e0 * eps + dt * f.sey[J]);
          else if (xbot) cy = -1.0 / eps;
          const long ox = band_off_e(w, I, J, 0), oy = band_off_e(w, I, J, 1);
          if (cx != 0.0 && ox >= 0) g += cx * S(ox);
          if (cy != 0.0 && oy >= 0) g += cy * S(oy);
        }
        if (J <= NY - 1 && !(J >= w.hxj0 && J <= w.hxj1) && I >= 1 && I <= NX - 1) {
          const double sm = f.smy[J] / eps;
          const long o = band_off_hx(w, I, J);
          if (o >= 0) g += dt * sm / (eps * (2.0 * u0 + dt * sm)) * S(o);
        }
        if (xbot && !(I >= w.hyi0 && I <= w.hyi1) && J >= 1 && J <= NY - 1) {
          const double sm = f.smx[I] / eps;
          const long o = band_off_hy(w, I, J);
          if (o >= 0) g += dt * sm / (eps * (2.0 * u0 + dt * sm)) * S(o);
        }
      }
      for (int o = 16; o > 0; o >>= 1) g += __shfl_down_sync(0xffffffffu, g, o);
      if (per_shot) {
        if (lane == 0) geps[size_t(s) * mn + p] += g;
      } else {
        tot += g;
      }
    }
    if (!per_shot && lane == 0) geps[p] += tot;
  }
}

}  // namespace gj

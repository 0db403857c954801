// Radar (GPR) FDTD kernels for sm_100a: coefficient build, fused Yee step
// (forward and reference adjoint), exact adjoint step, imaging, receiver I/O,
// and the plain one-half-step-per-launch kernels used as the FP64 baseline.
//
// Storage (per shot, per field): column-major node arrays with leading
// dimension ld >= NX+2 (a multiple of 32) and NY+3 columns; the array base
// points one column in, so node (i, j) lives at base[i + j*ld] for
// i in [-1, ld-1], j in [-1, NY+1].  Rows NX+1..ld-1 and the columns -1 and
// NY+1 are zero padding that nothing writes, which lets the stencils read
// one node past every edge without bounds checks.  The Yee grid of w_solve.m
// (Ez (NX+1)x(NY+1), Hx (NX+1)xNY, Hy NXx(NY+1)) maps onto the node range
// [0, NX] x [0, NY]; entries outside a field's own extent stay zero.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace gj {

enum Field { F_EZ = 0, F_HX = 1, F_HY = 2, F_EZX = 3, F_EZY = 4, NFIELDS = 5 };

// Problem-level geometry and coefficient arrays, shared by all shots.
template <class T>
struct WDev {
  int NX, NY, ld, P, Pt, m, n, di0, dj0;
  int hr0, hld;            // rows [hr0, hr0 + hld) of the domain-node layout (the model rows, 4-aligned)
  int ei0, ei1, ej0, ej1;  // interior Ez nodes (w_solve.m:201)
  int hyi0, hyi1;          // interior Hy rows (w_solve.m:146)
  int hxj0, hxj1;          // interior Hx columns (w_solve.m:144)
  T chxez, chyez;          // interior H coefficients (w_coeff.m:34-40 with mu_r=1, sigma_m=0)
  T rxy;                   // Cezhx / Cezhy = -dx/dy (w_coeff.m:29-30)
  const T* ce;             // Ceze, interior nodes
  const T* chy;            // Cezhy, interior nodes
  const T* ax; const T* bx; const T* ay; const T* by;      // split-field PML (band nodes)
  const T* hxa; const T* hxb; const T* hya; const T* hyb;  // H in the PML strips
  // Band frame (w_band.cuh): the PML nodes whose update coefficients depend on
  // the edge-replicated eps_r, stored per time step in two row-contiguous
  // rectangles: lateral (rows [0, bRB), columns [0, P] and [NY-P, NY]; planes
  // Ezx, Ezy, Hx) and bottom (rows [bR0, bRB), columns [0, NY]; planes Ezx,
  // Ezy, Hy).  E planes of rows >= bR0 live in the bottom rectangle.
  int bR0, bRB, bBh;       // bottom rows [bR0, bRB) (multiples of 4), bBh = bRB - bR0
  long bLsz, bBsz, bsz;    // lateral plane, bottom plane, whole slot (3 bLsz + 3 bBsz)
};

// Per-launch arguments of the fused step kernels.
template <class T>
struct StepArgs {
  const T* A;          // input state, [shot][field][node]
  T* B;                // output state
  size_t fstride;      // elements per field (ld*(NY+3))
  size_t sstride;      // elements per shot (NFIELDS*fstride)
  int shot0;           // first shot of this launch
  int tj;              // columns per block
  int it;              // time index (forward source sample)
  // forward source (w_solve.m:92)
  const long* src;     // per shot linear node index, -1 = none
  const T* cezj;       // per shot
  const T* wav;        // [shot][nt]
  int nt;
  // history write: domain Ez after the step into hist + shot*hstride
  T* hist; size_t hstride;
  // reference-adjoint imaging (w_grad.m:86-87 with differentiate_cube.m)
  const T* u0; const T* u1; const T* u2;  // three history slots for d/dt u
  T c0, c1, c2;                           // differentiation weights
  const T* uk;                            // u(k) slot
  T* acc; size_t astride;                 // accumulators [shot][4][dstride]: sumE, compE, sumS, compS
  int kahan;
  T* band;             // ring forward: band history slot of this step (w.bsz per shot), or nullptr
};

__device__ __forceinline__ size_t nidx(int i, int j, int ld) { return size_t(i) + size_t(j) * size_t(ld); }

template <class T>
__device__ __forceinline__ void kahan_add(T* sum, T* comp, T v) {
  T s = *sum, c = *comp;
  T y = v - c;
  T t = s + y;
  *comp = (t - s) - y;
  *sum = t;
}

// Hx / Hy coefficient pair at a node (interior scalars or strip arrays).
template <class T>
__device__ __forceinline__ void hx_coef(const WDev<T>& w, int i, int j, T& a, T& b) {
  if (j >= w.hxj0 && j <= w.hxj1) { a = T(1); b = w.chxez; }
  else { size_t k = nidx(i, j, w.ld); a = w.hxa[k]; b = w.hxb[k]; }
}
template <class T>
__device__ __forceinline__ void hy_coef(const WDev<T>& w, int i, int j, T& a, T& b) {
  if (i >= w.hyi0 && i <= w.hyi1) { a = T(1); b = w.chyez; }
  else { size_t k = nidx(i, j, w.ld); a = w.hya[k]; b = w.hyb[k]; }
}

// --------------------------------------------------------------------------
// Fused Yee step: new_H + new_H_pml + new_Ez + source + new_Ez_pml
// (w_solve.m:85-94).  MODE 0 = forward (source, history write);
// MODE 1 = reference adjoint (no source, imaging into accumulators).
//
// Each warp owns 32 consecutive rows (i) and marches along tj columns (j),
// keeping Ez(i, j), Ez(i, j+1) and Hx_new(i, j-1) in registers; the i
// neighbours come from warp shuffles, with lanes 0 and 31 loading the halo.
// A/B ping-pong keeps every halo read on the previous time level.
// --------------------------------------------------------------------------
template <class T, int MODE>
__global__ void __launch_bounds__(128) k_step(const WDev<T> w, const StepArgs<T> a) {
  const int lane = threadIdx.x & 31;
  const int i0w = blockIdx.x * blockDim.x + (threadIdx.x & ~31);
  const int ld = w.ld, NX = w.NX, NY = w.NY;
  if (i0w >= ld) return;  // whole warp beyond the padded rows
  const int I = i0w + lane;
  const int j0 = blockIdx.y * a.tj;
  if (j0 > NY) return;
  const int j1 = min(j0 + a.tj - 1, NY);
  const int s = a.shot0 + blockIdx.z;
  const size_t off = size_t(s) * a.sstride;
  const size_t fs = a.fstride;
  const T* __restrict__ EzA = a.A + off;
  const T* __restrict__ HxA = EzA + fs;
  const T* __restrict__ HyA = EzA + 2 * fs;
  const T* __restrict__ ExA = EzA + 3 * fs;
  const T* __restrict__ EyA = EzA + 4 * fs;
  T* __restrict__ EzB = a.B + off;
  T* __restrict__ HxB = EzB + fs;
  T* __restrict__ HyB = EzB + 2 * fs;
  T* __restrict__ ExB = EzB + 3 * fs;
  T* __restrict__ EyB = EzB + 4 * fs;

  long src = -1; T sval = T(0);
  if (MODE == 0) {
    src = a.src[s];
    if (src >= 0) sval = a.cezj[s] * a.wav[size_t(s) * a.nt + a.it];
  }
  const bool rowE = I >= 1 && I <= NX - 1;
  const bool rowHx = I <= NX;
  const bool rowHy = I <= NX - 1;
  const bool rowInt = I >= w.ei0 && I <= w.ei1;
  const bool rowDom = I >= w.di0 && I < w.di0 + w.m;

  // Preload Ez(I, j0) and Hx_new(I, j0-1).
  T ez_c = EzA[nidx(I, j0, ld)];
  T hx_prev = T(0);
  if (j0 >= 1 && rowHx) {
    T ha, hb; hx_coef(w, I, j0 - 1, ha, hb);
    hx_prev = ha * HxA[nidx(I, j0 - 1, ld)] + hb * (ez_c - EzA[nidx(I, j0 - 1, ld)]);
  }
  for (int J = j0; J <= j1; ++J) {
    const size_t k = nidx(I, J, ld);
    const T ez_n = EzA[k + ld];
    T ez_dn = __shfl_down_sync(0xffffffffu, ez_c, 1);
    T ez_up = __shfl_up_sync(0xffffffffu, ez_c, 1);
    if (lane == 31) ez_dn = EzA[k + 1];
    if (lane == 0) ez_up = EzA[k - 1];
    // new_H / new_H_pml (w_solve.m:136-187)
    T hx_new = T(0), hy_new = T(0);
    if (rowHx && J <= NY - 1) {
      T ha, hb; hx_coef(w, I, J, ha, hb);
      hx_new = ha * HxA[k] + hb * (ez_n - ez_c);
      HxB[k] = hx_new;
    }
    if (rowHy) {
      T ha, hb; hy_coef(w, I, J, ha, hb);
      hy_new = ha * HyA[k] + hb * (ez_dn - ez_c);
      HyB[k] = hy_new;
    }
    T hy_up = __shfl_up_sync(0xffffffffu, hy_new, 1);
    if (lane == 0) {
      hy_up = T(0);
      if (I >= 1 && I - 1 <= NX - 1) {
        T ha, hb; hy_coef(w, I - 1, J, ha, hb);
        hy_up = ha * HyA[k - 1] + hb * (ez_c - ez_up);
      }
    }
    // new_Ez + source + new_Ez_pml (w_solve.m:193-268)
    if (rowE && J >= 1 && J <= NY - 1) {
      const T dhy = hy_new - hy_up;
      const T dhx = hx_new - hx_prev;
      T e;
      if (rowInt && J >= w.ej0 && J <= w.ej1) {
        const T ch = w.chy[k];
        e = w.ce[k] * ez_c + ch * dhy + (w.rxy * ch) * dhx;
        if (MODE == 0 && long(k) == src) e += sval;
      } else {
        const T ex = w.ax[k] * ExA[k] + w.bx[k] * dhy;
        const T ey = w.ay[k] * EyA[k] + w.by[k] * dhx;
        ExB[k] = ex; EyB[k] = ey;
        e = ex + ey;
      }
      EzB[k] = e;
      if (rowDom && J >= w.dj0 && J < w.dj0 + w.n) {
        const size_t p = size_t(I - w.di0) + size_t(J - w.dj0) * size_t(w.m);
        if (MODE == 0) {
          if (a.hist) a.hist[size_t(s) * a.hstride + p] = e;
        } else {
          const size_t hs = size_t(s) * a.hstride;
          const T du = a.c0 * a.u0[hs + p] + a.c1 * a.u1[hs + p] + a.c2 * a.u2[hs + p];
          const T uk = a.uk[hs + p];
          T* acc = a.acc + size_t(s) * a.astride;
          const size_t mn = size_t(w.m) * size_t(w.n);
          if (a.kahan) {
            kahan_add(acc + p, acc + mn + p, -du * e);
            kahan_add(acc + 2 * mn + p, acc + 3 * mn + p, -uk * e);
          } else {
            acc[p] -= du * e;
            acc[2 * mn + p] -= uk * e;
          }
        }
      }
    }
    hx_prev = hx_new;
    ez_c = ez_n;
  }
}

// --------------------------------------------------------------------------
// Exact adjoint step: transpose of one k_step<MODE 0>, applied to the adjoint
// state (lE, lHx, lHy, lEzx, lEzy) after the injection of e(k).  With
// l = lE (+lEzx / lEzy in the PML band):
//   px = Cezhy*l | bx*lx,  py = Cezhx*l | by*ly,  lE_mid = Ceze*l | 0
//   lHx_t(i,j) = lHx + py(i,j) - py(i,j+1);  lHy_t = lHy + px(i,j) - px(i+1,j)
//   lHx' = hxa*lHx_t, qx = hxb*lHx_t (same for y)
//   lE'(i,j) = lE_mid + qx(i,j-1) - qx(i,j) + qy(i-1,j) - qy(i,j)
// The neighbour pattern mirrors the forward (+1 neighbours for the H-like
// half, -1 neighbours for the E-like half), so the same marching scheme applies.
// Imaging at interior model nodes: S1 += l*(E^k - E^{k-1}), S2 += l*(E^k + E^{k-1}).
// --------------------------------------------------------------------------
template <class T>
struct AdjArgs {
  const T* A; T* B; size_t fstride, sstride;
  int shot0, tj;
  const T* ek; const T* ekm1;  // history slots E^k, E^{k-1}
  size_t hstride;
  T* acc; size_t astride; int kahan;
};

template <class T>
__device__ __forceinline__ void adj_p(const WDev<T>& w, int i, int j, size_t k, T lE, T lx_, T ly_,
                                      T& px, T& py, T& lmid, T& lx, T& ly) {
  // p-values of node (i, j) given its adjoint (lE) and split adjoints.
  if (i >= w.ei0 && i <= w.ei1 && j >= w.ej0 && j <= w.ej1) {
    const T ch = w.chy[k];
    px = ch * lE; py = (w.rxy * ch) * lE; lmid = w.ce[k] * lE; lx = ly = T(0);
  } else if (i >= 1 && i <= w.NX - 1 && j >= 1 && j <= w.NY - 1) {
    lx = lx_ + lE; ly = ly_ + lE;
    px = w.bx[k] * lx; py = w.by[k] * ly; lmid = T(0);
  } else {
    px = py = lmid = lx = ly = T(0);
  }
}

// --------------------------------------------------------------------------
// Receiver I/O and small helpers
// --------------------------------------------------------------------------
// d[s][r*nt + it] = Ez(rec[s][r]) (w_solve.m:100); also Jz (w_solve.m:104).
template <class T>
__global__ void k_record(const T* state, size_t sstride, const long* rec, int nr, const int* nrs,
                         int it, int nt, T* d, const long* src, T* jz, int nshots) {
  const int s = blockIdx.y;
  if (s >= nshots) return;
  const T* Ez = state + size_t(s) * sstride;
  for (int r = threadIdx.x + blockIdx.x * blockDim.x; r < nrs[s]; r += blockDim.x * gridDim.x)
    d[(size_t(s) * nr + r) * nt + it] = Ez[rec[size_t(s) * nr + r]];
  if (jz && threadIdx.x == 0 && blockIdx.x == 0 && src[s] >= 0) jz[size_t(s) * nt + it] = Ez[src[s]];
}

// Reference adjoint: Ez(rec) = e(k, :) before the step (w_grad.m:72).
// `rec` holds, per shot, receivers with duplicates removed (last one kept).
template <class T>
__global__ void k_inject_set(T* state, size_t sstride, const long* rec, const int* rsel, int nr,
                             const int* nrs, const T* e, int k, int nt, int nshots) {
  const int s = blockIdx.y;
  if (s >= nshots) return;
  T* Ez = state + size_t(s) * sstride;
  for (int q = threadIdx.x + blockIdx.x * blockDim.x; q < nrs[s]; q += blockDim.x * gridDim.x) {
    const int r = rsel[size_t(s) * nr + q];
    Ez[rec[size_t(s) * nr + r]] = e[(size_t(s) * nr + r) * nt + k];
  }
}

// Exact adjoint: lE(rec) += e(k, :) (transpose of the recording).
template <class T>
__global__ void k_inject_add(T* state, size_t sstride, const long* rec, int nr, const int* nrs,
                             const T* e, int k, int nt, int nshots) {
  const int s = blockIdx.y;
  if (s >= nshots) return;
  T* L = state + size_t(s) * sstride;
  for (int r = threadIdx.x + blockIdx.x * blockDim.x; r < nrs[s]; r += blockDim.x * gridDim.x)
    atomicAdd(L + rec[size_t(s) * nr + r], e[(size_t(s) * nr + r) * nt + k]);
}

// History slots and imaging accumulators use the "domain-node" layout: per
// shot hld x n elements, element (i, j) of a model column j in [dj0, dj0+n)
// and a row i in [hr0, hr0 + hld) at (j - dj0)*hld + (i - hr0).  hr0 and hld
// are multiples of 4, so a lane's 16-byte row vector is either wholly inside
// or wholly outside, and the kernels read and write the layout with the same
// aligned vector accesses as the fields.  Rows outside the model are unused.
template <class T>
__device__ __forceinline__ size_t dnode(const WDev<T>& w, int i, int j) {
  return size_t(j - w.dj0) * size_t(w.hld) + size_t(i - w.hr0);
}
template <class T>
__device__ __forceinline__ bool drow(const WDev<T>& w, int i) { return i >= w.hr0 && i < w.hr0 + w.hld; }

// Copies the model columns of Ez (state) into a history slot (the checkpoint's u).
template <class T>
__global__ void k_domain_copy(const WDev<T> w, const T* state, size_t sstride, T* hist,
                              size_t hstride, int nshots) {
  const size_t dn = size_t(w.hld) * w.n;
  const int s = blockIdx.y;
  if (s >= nshots) return;
  for (size_t q = threadIdx.x + size_t(blockIdx.x) * blockDim.x; q < dn; q += size_t(blockDim.x) * gridDim.x) {
    const int I = w.hr0 + int(q % w.hld), b = int(q / w.hld);
    hist[size_t(s) * hstride + q] = state[size_t(s) * sstride + nidx(I, w.dj0 + b, w.ld)];
  }
}

// Counts the non-finite values of x[0, n) into *count (NaN / Inf detection of
// results; the reference's caller zeroes NaN gradients, w_update_e.m:131-137).
template <class T>
__global__ void k_count_nonfinite(const T* x, size_t n, unsigned* count) {
  unsigned c = 0;
  for (size_t i = threadIdx.x + size_t(blockIdx.x) * blockDim.x; i < n; i += size_t(blockDim.x) * gridDim.x)
    c += isfinite(x[i]) ? 0u : 1u;
  for (int o = 16; o > 0; o >>= 1) c += __shfl_down_sync(0xffffffffu, c, o);
  if ((threadIdx.x & 31) == 0 && c) atomicAdd(count, c);
}

// Final gradient: out[p] = scale(p) * sum over shots of acc, in double.
// kind 0 (reference): g_eps = dt*sumE, g_sig = dt*sumS (w_grad.m:108).
// kind 1 (exact): g_eps = -2 eps0/D * S1, g_sig = -dt/D * S2 at interior model
// nodes (D = 2 eps_r eps0 + dt sigma); the PML band terms are added separately.
template <class T>
__global__ void k_finish(const WDev<T> w, const T* acc, size_t astride, int nshots, int per_shot,
                         int kind, double dt, double eps0, const double* eps_m, const double* sig_m,
                         double* geps, double* gsig) {
  const size_t mn = size_t(w.m) * w.n;
  const size_t dn = size_t(w.hld) * w.n;
  for (size_t p = threadIdx.x + size_t(blockIdx.x) * blockDim.x; p < mn; p += size_t(blockDim.x) * gridDim.x) {
    double fe, fs;
    if (kind == 0) { fe = dt; fs = dt; }
    else {
      const double D = 2.0 * eps_m[p] * eps0 + dt * sig_m[p];
      fe = -2.0 * eps0 / D; fs = -dt / D;
    }
    const size_t q = dnode(w, w.di0 + int(p % w.m), w.dj0 + int(p / w.m));
    double se = 0, ss = 0;
    for (int s = 0; s < nshots; ++s) {
      const T* A = acc + size_t(s) * astride;
      // Kahan: the compensation term holds the excess of the running sum.
      const double ve = double(A[q]) - double(A[dn + q]);
      const double vs = double(A[2 * dn + q]) - double(A[3 * dn + q]);
      if (per_shot) {
        geps[size_t(s) * mn + p] = fe * ve;
        gsig[size_t(s) * mn + p] = fs * vs;
      } else { se += ve; ss += vs; }
    }
    if (!per_shot) { geps[p] = fe * se; gsig[p] = fs * ss; }
  }
}

// --------------------------------------------------------------------------
// Plain kernels: one half-step per launch, one thread per node, in place.
// The FP64 instantiation is the "plain per-shot FP64 GPU form" baseline.
// --------------------------------------------------------------------------
template <class T>
__global__ void k_plain_h(const WDev<T> w, T* st, size_t fs) {
  const int I = blockIdx.x * blockDim.x + threadIdx.x;
  const int J = blockIdx.y * blockDim.y + threadIdx.y;
  if (I > w.NX || J > w.NY) return;
  T* Ez = st; T* Hx = st + fs; T* Hy = st + 2 * fs;
  const size_t k = nidx(I, J, w.ld);
  if (J <= w.NY - 1) { T a, b; hx_coef(w, I, J, a, b); Hx[k] = a * Hx[k] + b * (Ez[k + w.ld] - Ez[k]); }
  if (I <= w.NX - 1) { T a, b; hy_coef(w, I, J, a, b); Hy[k] = a * Hy[k] + b * (Ez[k + 1] - Ez[k]); }
}

template <class T>
__global__ void k_plain_e(const WDev<T> w, T* st, size_t fs, long src, T sval, T* hist) {
  const int I = blockIdx.x * blockDim.x + threadIdx.x;
  const int J = blockIdx.y * blockDim.y + threadIdx.y;
  if (I < 1 || I > w.NX - 1 || J < 1 || J > w.NY - 1) return;
  T* Ez = st; T* Hx = st + fs; T* Hy = st + 2 * fs; T* Ex = st + 3 * fs; T* Ey = st + 4 * fs;
  const size_t k = nidx(I, J, w.ld);
  const T dhy = Hy[k] - Hy[k - 1], dhx = Hx[k] - Hx[k - w.ld];
  T e;
  if (I >= w.ei0 && I <= w.ei1 && J >= w.ej0 && J <= w.ej1) {
    e = w.ce[k] * Ez[k] + w.chy[k] * dhy + (w.rxy * w.chy[k]) * dhx;
    if (long(k) == src) e += sval;
  } else {
    const T ex = w.ax[k] * Ex[k] + w.bx[k] * dhy, ey = w.ay[k] * Ey[k] + w.by[k] * dhx;
    Ex[k] = ex; Ey[k] = ey; e = ex + ey;
  }
  Ez[k] = e;
  if (hist && J >= w.dj0 && J < w.dj0 + w.n && drow(w, I)) hist[dnode(w, I, J)] = e;
}

// Plain reference-adjoint imaging: g -= du*a, g -= u*a (separate pass).
template <class T>
__global__ void k_plain_img_ref(const WDev<T> w, const T* st, const T* u0, const T* u1, const T* u2,
                                T c0, T c1, T c2, const T* uk, T* acc) {
  const size_t mn = size_t(w.m) * w.n;
  const size_t dn = size_t(w.hld) * w.n;
  for (size_t p = threadIdx.x + size_t(blockIdx.x) * blockDim.x; p < mn; p += size_t(blockDim.x) * gridDim.x) {
    const int I = w.di0 + int(p % w.m), J = w.dj0 + int(p / w.m);
    const size_t q = dnode(w, I, J);
    const T av = st[nidx(I, J, w.ld)];
    acc[q] -= (c0 * u0[q] + c1 * u1[q] + c2 * u2[q]) * av;
    acc[2 * dn + q] -= uk[q] * av;
  }
}

// Plain exact adjoint, three launches per step.
// (1) E part: p-values and lE_mid into scratch, split adjoints in place, imaging.
template <class T>
__global__ void k_plain_adj_e(const WDev<T> w, T* st, size_t fs, T* px, T* py, T* lm,
                              const T* ek, const T* ekm1, T* acc) {
  const int I = blockIdx.x * blockDim.x + threadIdx.x;
  const int J = blockIdx.y * blockDim.y + threadIdx.y;
  if (I > w.NX || J > w.NY) return;
  const size_t k = nidx(I, J, w.ld);
  T* L = st; T* Sx = st + 3 * fs; T* Sy = st + 4 * fs;
  T pxv, pyv, lmv, lx, ly;
  const T l = L[k];
  adj_p(w, I, J, k, l, Sx[k], Sy[k], pxv, pyv, lmv, lx, ly);
  px[k] = pxv; py[k] = pyv; lm[k] = lmv;
  const bool interior = I >= w.ei0 && I <= w.ei1 && J >= w.ej0 && J <= w.ej1;
  if (!interior && I >= 1 && I <= w.NX - 1 && J >= 1 && J <= w.NY - 1) {
    Sx[k] = w.ax[k] * lx; Sy[k] = w.ay[k] * ly;
  }
  if (interior && I >= w.di0 && I < w.di0 + w.m && J >= w.dj0 && J < w.dj0 + w.n) {
    const size_t q = dnode(w, I, J);
    const size_t dn = size_t(w.hld) * w.n;
    acc[q] += l * (ek[q] - ekm1[q]);
    acc[2 * dn + q] += l * (ek[q] + ekm1[q]);
  }
}
// (2) H part: lH update, q into scratch.
template <class T>
__global__ void k_plain_adj_h(const WDev<T> w, T* st, size_t fs, const T* px, const T* py, T* qx, T* qy) {
  const int I = blockIdx.x * blockDim.x + threadIdx.x;
  const int J = blockIdx.y * blockDim.y + threadIdx.y;
  if (I > w.NX || J > w.NY) return;
  const size_t k = nidx(I, J, w.ld);
  T* Lx = st + fs; T* Ly = st + 2 * fs;
  if (J <= w.NY - 1) {
    T a, b; hx_coef(w, I, J, a, b);
    const T lt = Lx[k] + py[k] - py[k + w.ld];
    Lx[k] = a * lt; qx[k] = b * lt;
  } else qx[k] = T(0);
  if (I <= w.NX - 1) {
    T a, b; hy_coef(w, I, J, a, b);
    const T lt = Ly[k] + px[k] - px[k + 1];
    Ly[k] = a * lt; qy[k] = b * lt;
  } else qy[k] = T(0);
}
// (3) lE assembly.
template <class T>
__global__ void k_plain_adj_assemble(const WDev<T> w, T* st, const T* lm, const T* qx, const T* qy) {
  const int I = blockIdx.x * blockDim.x + threadIdx.x;
  const int J = blockIdx.y * blockDim.y + threadIdx.y;
  if (I < 1 || I > w.NX - 1 || J < 1 || J > w.NY - 1) return;
  const size_t k = nidx(I, J, w.ld);
  st[k] = lm[k] + qx[k - w.ld] - qx[k] + qy[k - 1] - qy[k];
}

// --------------------------------------------------------------------------
// Coefficient build on the device: w_exp2pml.m (padding), w_cpml.m (PML
// strips) and w_coeff.m (interior) for every node, from the m x n model.
// sex/smx (per row) and sey/smy (per column) are the graded PML profiles.
// --------------------------------------------------------------------------
struct CoefBuild {
  int NX, NY, ld, P, Pt, air, m, n;
  double dx, dy, dt, eps0, mu0;
  const double* sex; const double* smx; const double* sey; const double* smy;
};

template <class TM>
__device__ __forceinline__ void pad_model(const CoefBuild& c, const TM* eps, const TM* sig, int I,
                                          int J, double& e, double& s) {
  // w_exp2pml.m:19-34: rows [pml_top | air | model | pml], cols [pml | model | pml].
  const int rows_mid = c.air + c.m;
  int r = I - c.Pt; r = r < 0 ? 0 : (r > rows_mid - 1 ? rows_mid - 1 : r);
  int jm = J - c.P; jm = jm < 0 ? 0 : (jm > c.n - 1 ? c.n - 1 : jm);
  if (r < c.air) { e = 1.0; s = 0.0; return; }
  e = double(eps[size_t(r - c.air) + size_t(jm) * c.m]);
  const bool in_model = (I >= c.Pt + c.air) && (I < c.Pt + rows_mid) && (J >= c.P) && (J < c.P + c.n);
  s = in_model ? double(sig[size_t(r - c.air) + size_t(J - c.P) * c.m]) : 0.0;
}

// ce_r / chy_r receive the sigma-flipped interior coefficients of w_grad.m:26-27.
template <class T, class TM>
__global__ void k_build_coefs(const CoefBuild c, const TM* eps, const TM* sig, T* ce, T* chy, T* ax,
                              T* bx, T* ay, T* by, T* hxa, T* hxb, T* hya, T* hyb, T* ce_r, T* chy_r,
                              double* eps_model, double* sig_model) {
  const int I = blockIdx.x * blockDim.x + threadIdx.x;
  const int J = blockIdx.y * blockDim.y + threadIdx.y;
  if (I > c.NX || J > c.NY) return;
  const size_t k = nidx(I, J, c.ld);
  const double dt = c.dt, dx = c.dx, dy = c.dy, e0 = c.eps0, u0 = c.mu0;
  double e = 1.0, s = 0.0;
  if (I < c.NX && J < c.NY) pad_model(c, eps, sig, I, J, e, s);
  // Hx (w_solve.m:144, 180-186)
  double ha = 1.0, hb = 0.0;
  if (J <= c.NY - 1) {
    if (J >= c.P && J <= c.NY - c.P - 1) { hb = -(2 * dt / dy) / (2 * u0); }
    else if (I >= 1 && I <= c.NX - 1) {
      const double sm = c.smy[J] / e;  // w_cpml.m:123, 164
      ha = (2 * u0 - dt * sm) / (2 * u0 + dt * sm);
      hb = -(2 * dt / dy) / (2 * u0 + dt * sm);
    }
  }
  hxa[k] = T(ha); hxb[k] = T(hb);
  // Hy (w_solve.m:146, 170-176)
  ha = 1.0; hb = 0.0;
  if (I <= c.NX - 1) {
    if (I >= c.Pt && I <= c.NX - c.P - 1) { hb = (2 * dt / dx) / (2 * u0); }
    else if (J >= 1 && J <= c.NY - 1) {
      double sm = c.smx[I];
      if (I >= c.NX - c.P) sm /= e;  // bottom strip only (w_cpml.m:83)
      ha = (2 * u0 - dt * sm) / (2 * u0 + dt * sm);
      hb = (2 * dt / dx) / (2 * u0 + dt * sm);
    }
  }
  hya[k] = T(ha); hyb[k] = T(hb);
  // Ez
  double vce = 0, vch = 0, vax = 0, vbx = 0, vay = 0, vby = 0, rce = 0, rch = 0;
  const bool interior = I >= c.Pt + 1 && I <= c.NX - c.P - 1 && J >= c.P + 1 && J <= c.NY - c.P - 1;
  const bool band = !interior && I >= 1 && I <= c.NX - 1 && J >= 1 && J <= c.NY - 1;
  if (interior) {  // w_coeff.m:28-29
    const double D = 2 * e * e0 + dt * s;
    vce = (2 * e * e0 - dt * s) / D;
    vch = (2 * dt / dx) / D;
    const double Dr = 2 * e * e0 - dt * s;
    rce = (2 * e * e0 + dt * s) / Dr;
    rch = (2 * dt / dx) / Dr;
  } else if (band) {
    const bool xtop = I >= 1 && I <= c.Pt, xbot = I >= c.NX - c.P;
    const bool ystrip = (J <= c.P) || (J >= c.NY - c.P);
    if (xtop) {  // w_cpml.m:60-61
      const double sx = c.sex[I];
      vax = (2 * e0 - dt * sx) / (2 * e0 + dt * sx); vbx = (2 * dt / dx) / (2 * e0 + dt * sx);
    } else if (xbot) {  // w_cpml.m:93-96
      const double sx = c.sex[I];
      vax = (2 * e0 * e - dt * sx) / (2 * e0 * e + dt * sx); vbx = (2 * dt / dx) / (2 * e0 * e + dt * sx);
    } else {  // w_cpml.m:133-134, 174-175
      vax = 1.0; vbx = dt / (dx * e0 * e);
    }
    if (ystrip) {  // w_cpml.m:141-144, 182-185
      const double sy = c.sey[J];
      vay = (2 * e0 * e - dt * sy) / (2 * e0 * e + dt * sy); vby = -(2 * dt / dy) / (2 * e0 * e + dt * sy);
    } else if (xtop) {  // w_cpml.m:63-64
      vay = 1.0; vby = -dt / (dy * e0);
    } else {  // w_cpml.m:103-104
      vay = 1.0; vby = -dt / (dy * e0 * e);
    }
  }
  // Free top: the Ez = 0 row keeps Ez (Ceze = 1, Cezhy = 0) in the interior
  // columns, so a kernel may apply the interior update there without a branch.
  if (c.Pt == 0 && I == 0 && J >= c.P + 1 && J <= c.NY - c.P - 1) { vce = 1.0; vch = 0.0; }
  ce[k] = T(vce); chy[k] = T(vch);
  ce_r[k] = T(rce); chy_r[k] = T(rch);
  ax[k] = T(vax); bx[k] = T(vbx); ay[k] = T(vay); by[k] = T(vby);
  // model copy in double for the exact-gradient scaling
  if (eps_model && I >= c.Pt + c.air && I < c.Pt + c.air + c.m && J >= c.P && J < c.P + c.n) {
    const size_t p = size_t(I - c.Pt - c.air) + size_t(J - c.P) * c.m;
    eps_model[p] = e; sig_model[p] = s;
  }
}

}  // namespace gj

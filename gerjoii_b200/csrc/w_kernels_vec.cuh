// Vectorised marching kernels: each lane owns V = 16/sizeof(T) consecutive rows
// (float4 / double2 loads and stores), a warp owns 32*V rows and marches along
// the tile's columns.  Same arithmetic as k_step / k_adj_step in
// w_kernels.cuh, with 4x (FP32) more bytes in flight per load instruction.
//
// Row guards: a lane whose first row is beyond NX issues no loads or stores.
// ld is a multiple of 4 and >= NX+2, so the lane holding row NX stores only
// rows below ld; lanes past NX read nothing.  Lane 31's halo row and lane 0's
// row -1 use the zero padding of the storage layout.
#pragma once
#include "w_kernels.cuh"

namespace gj {

#ifndef GJ_VEC_F32
#define GJ_VEC_F32 4  // rows per lane in FP32 (4: float4 accesses, 2: float2)
#endif
#ifndef GJ_MINB_STEP
#define GJ_MINB_STEP 5  // minimum resident blocks per SM requested for k_stepv (caps registers)
#endif
#ifndef GJ_MINB_ADJ
#define GJ_MINB_ADJ 4  // same for k_adj_stepv
#endif

template <class T> struct VT;
template <> struct VT<float> { static constexpr int V = GJ_VEC_F32; };
template <> struct VT<double> { static constexpr int V = 2; };

__device__ __forceinline__ void vld(const float* p, float (&r)[4]) {
  const float4 x = __ldg(reinterpret_cast<const float4*>(p));
  r[0] = x.x; r[1] = x.y; r[2] = x.z; r[3] = x.w;
}
__device__ __forceinline__ void vld(const float* p, float (&r)[2]) {
  const float2 x = __ldg(reinterpret_cast<const float2*>(p));
  r[0] = x.x; r[1] = x.y;
}
__device__ __forceinline__ void vld(const double* p, double (&r)[2]) {
  const double2 x = __ldg(reinterpret_cast<const double2*>(p));
  r[0] = x.x; r[1] = x.y;
}
// Loads of data written by earlier launches in the same stream: plain loads.
__device__ __forceinline__ void vldw(const float* p, float (&r)[4]) {
  const float4 x = *reinterpret_cast<const float4*>(p);
  r[0] = x.x; r[1] = x.y; r[2] = x.z; r[3] = x.w;
}
__device__ __forceinline__ void vldw(const float* p, float (&r)[2]) {
  const float2 x = *reinterpret_cast<const float2*>(p);
  r[0] = x.x; r[1] = x.y;
}
__device__ __forceinline__ void vldw(const double* p, double (&r)[2]) {
  const double2 x = *reinterpret_cast<const double2*>(p);
  r[0] = x.x; r[1] = x.y;
}
__device__ __forceinline__ void vst(float* p, const float (&r)[4]) {
  *reinterpret_cast<float4*>(p) = make_float4(r[0], r[1], r[2], r[3]);
}
__device__ __forceinline__ void vst(float* p, const float (&r)[2]) {
  *reinterpret_cast<float2*>(p) = make_float2(r[0], r[1]);
}
__device__ __forceinline__ void vst(double* p, const double (&r)[2]) {
  *reinterpret_cast<double2*>(p) = make_double2(r[0], r[1]);
}
template <class T, int V>
__device__ __forceinline__ void vzero(T (&r)[V]) {
#pragma unroll
  for (int v = 0; v < V; ++v) r[v] = T(0);
}

// Fused Yee step (MODE 0 forward, MODE 1 reference adjoint), vectorised.
template <class T, int MODE>
__global__ void __launch_bounds__(128, GJ_MINB_STEP) k_stepv(const WDev<T> w, const StepArgs<T> a) {
  constexpr int V = VT<T>::V;
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  const int i0w = (blockIdx.x * (blockDim.x >> 5) + warp) * (32 * V);
  const int ld = w.ld, NX = w.NX, NY = w.NY;
  if (i0w > NX) return;  // no valid row in this warp
  const int I0 = i0w + lane * V;
  const bool live = I0 <= NX;
  const int j0 = blockIdx.y * a.tj;
  if (j0 > NY) return;
  const int j1 = min(j0 + a.tj - 1, NY);
  const int zl = blockIdx.z;        // shot within this launch: state and history index
  const int s = a.shot0 + zl;       // shot within the call: source, wavelet, accumulators
  const size_t off = size_t(zl) * a.sstride, fs = a.fstride;
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
  // lane-level row classification
  bool hyStrip = false, rowBandAny = false, rowIntAll = true, rowIntAny = false;
#pragma unroll
  for (int v = 0; v < V; ++v) {
    const int I = I0 + v;
    const bool rint = I >= w.ei0 && I <= w.ei1;
    rowIntAll = rowIntAll && rint;
    rowIntAny = rowIntAny || rint;
    if (I <= NX - 1 && !(I >= w.hyi0 && I <= w.hyi1)) hyStrip = true;
    if (I >= 1 && I <= NX - 1 && !rint) rowBandAny = true;
  }
  T ez_c[V], hx_prev[V];
  vzero<T, V>(ez_c); vzero<T, V>(hx_prev);
  if (live) {
    vldw(EzA + nidx(I0, j0, ld), ez_c);
    if (j0 >= 1) {
      T ezm[V], hxo[V];
      vldw(EzA + nidx(I0, j0 - 1, ld), ezm);
      vldw(HxA + nidx(I0, j0 - 1, ld), hxo);
#pragma unroll
      for (int v = 0; v < V; ++v) {
        if (I0 + v <= NX) {
          T ha, hb; hx_coef(w, I0 + v, j0 - 1, ha, hb);
          hx_prev[v] = ha * hxo[v] + hb * (ez_c[v] - ezm[v]);
        }
      }
    }
  }
  for (int J = j0; J <= j1; ++J) {
    const size_t k = nidx(I0, J, ld);
    T ez_n[V], hxo[V], hyo[V];
    vzero<T, V>(ez_n); vzero<T, V>(hxo); vzero<T, V>(hyo);
    if (live) {
      vldw(EzA + k + ld, ez_n);
      vldw(HxA + k, hxo);
      vldw(HyA + k, hyo);
    }
    T nxt = __shfl_down_sync(0xffffffffu, ez_c[0], 1);
    T prv = __shfl_up_sync(0xffffffffu, ez_c[V - 1], 1);
    if (lane == 31) nxt = (I0 + V <= NX) ? EzA[k + V] : T(0);
    if (lane == 0) prv = EzA[k - 1];
    // new_H / new_H_pml (w_solve.m:136-187)
    const bool hxStripCol = !(J >= w.hxj0 && J <= w.hxj1);
    T hxa_[V], hxb_[V], hya_[V], hyb_[V];
    if (live && hxStripCol) { vld(w.hxa + k, hxa_); vld(w.hxb + k, hxb_); }
    else {
#pragma unroll
      for (int v = 0; v < V; ++v) { hxa_[v] = T(1); hxb_[v] = w.chxez; }
    }
    if (live && hyStrip) { vld(w.hya + k, hya_); vld(w.hyb + k, hyb_); }
    T hx_new[V], hy_new[V];
#pragma unroll
    for (int v = 0; v < V; ++v) {
      const int I = I0 + v;
      hx_new[v] = T(0);
      if (I <= NX && J <= NY - 1) hx_new[v] = hxa_[v] * hxo[v] + hxb_[v] * (ez_n[v] - ez_c[v]);
      const T edn = (v < V - 1) ? ez_c[v < V - 1 ? v + 1 : v] : nxt;
      hy_new[v] = T(0);
      if (I <= NX - 1) {
        T ha = T(1), hb = w.chyez;
        if (!(I >= w.hyi0 && I <= w.hyi1)) { ha = hya_[v]; hb = hyb_[v]; }
        hy_new[v] = ha * hyo[v] + hb * (edn - ez_c[v]);
      }
    }
    if (live) { vst(HxB + k, hx_new); vst(HyB + k, hy_new); }
    T hy_up = __shfl_up_sync(0xffffffffu, hy_new[V - 1], 1);
    if (lane == 0) {
      hy_up = T(0);
      if (I0 >= 1 && I0 - 1 <= NX - 1) {
        T ha, hb; hy_coef(w, I0 - 1, J, ha, hb);
        hy_up = ha * HyA[k - 1] + hb * (ez_c[0] - prv);
      }
    }
    // new_Ez + source + new_Ez_pml (w_solve.m:193-268)
    const bool colE = J >= 1 && J <= NY - 1;
    const bool colInt = J >= w.ej0 && J <= w.ej1;
    const bool anyInt = colInt && rowIntAny;
    const bool anyBand = colE && (rowBandAny || (!colInt && rowIntAny));
    T ce_[V], ch_[V], ax_[V], bx_[V], ay_[V], by_[V], exo[V], eyo[V];
    if (live && anyInt) { vld(w.ce + k, ce_); vld(w.chy + k, ch_); }
    if (live && anyBand) {
      vld(w.ax + k, ax_); vld(w.bx + k, bx_); vld(w.ay + k, ay_); vld(w.by + k, by_);
      vldw(ExA + k, exo); vldw(EyA + k, eyo);
    }
    T e_new[V];
#pragma unroll
    for (int v = 0; v < V; ++v) {
      const int I = I0 + v;
      e_new[v] = ez_c[v];
      if (colE && I >= 1 && I <= NX - 1) {
        const T dhy = hy_new[v] - (v > 0 ? hy_new[v > 0 ? v - 1 : 0] : hy_up);
        const T dhx = hx_new[v] - hx_prev[v];
        if (colInt && I >= w.ei0 && I <= w.ei1) {
          e_new[v] = ce_[v] * ez_c[v] + ch_[v] * dhy + (w.rxy * ch_[v]) * dhx;
          if (MODE == 0 && long(k) + v == src) e_new[v] += sval;
        } else {
          exo[v] = ax_[v] * exo[v] + bx_[v] * dhy;
          eyo[v] = ay_[v] * eyo[v] + by_[v] * dhx;
          e_new[v] = exo[v] + eyo[v];
        }
      }
    }
    if (live) {
      vst(EzB + k, e_new);
      if (anyBand) { vst(ExB + k, exo); vst(EyB + k, eyo); }
      if (J >= w.dj0 && J < w.dj0 + w.n && drow(w, I0)) {
        // history / imaging in the domain-node layout (aligned vectors)
        const size_t q = size_t(zl) * a.hstride + dnode(w, I0, J);
        if (MODE == 0) {
          if (a.hist) vst(a.hist + q, e_new);
        } else {
          T u0[V], u1[V], u2[V], uk[V];
          vldw(a.u0 + q, u0); vldw(a.u1 + q, u1); vldw(a.u2 + q, u2); vldw(a.uk + q, uk);
          const size_t dn = size_t(w.hld) * size_t(w.n);
          T* acc = a.acc + size_t(s) * a.astride + dnode(w, I0, J);
          T sE[V], cE[V], sS[V], cS[V];
          vldw(acc, sE); vldw(acc + 2 * dn, sS);
          if (a.kahan) { vldw(acc + dn, cE); vldw(acc + 3 * dn, cS); }
#pragma unroll
          for (int v = 0; v < V; ++v) {
            const T du = a.c0 * u0[v] + a.c1 * u1[v] + a.c2 * u2[v];
            if (a.kahan) {
              kahan_add(&sE[v], &cE[v], -du * e_new[v]);
              kahan_add(&sS[v], &cS[v], -uk[v] * e_new[v]);
            } else {
              sE[v] -= du * e_new[v];
              sS[v] -= uk[v] * e_new[v];
            }
          }
          vst(acc, sE); vst(acc + 2 * dn, sS);
          if (a.kahan) { vst(acc + dn, cE); vst(acc + 3 * dn, cS); }
        }
      }
    }
#pragma unroll
    for (int v = 0; v < V; ++v) { hx_prev[v] = hx_new[v]; ez_c[v] = ez_n[v]; }
  }
}

// p-values of V nodes (rows I0..I0+V-1, column J) from their adjoints.
template <class T, int V>
__device__ __forceinline__ void adj_pv(const WDev<T>& w, int I0, int J, size_t k, bool live, const T (&l)[V],
                                       const T* SxA, const T* SyA, T (&px)[V], T (&py)[V], T (&lm)[V],
                                       T (&lx)[V], T (&ly)[V]) {
  const bool colE = J >= 1 && J <= w.NY - 1;
  const bool colInt = J >= w.ej0 && J <= w.ej1;
  bool anyInt = false, anyBand = false;
#pragma unroll
  for (int v = 0; v < V; ++v) {
    const int I = I0 + v;
    const bool e = colE && I >= 1 && I <= w.NX - 1;
    const bool in = e && colInt && I >= w.ei0 && I <= w.ei1;
    anyInt = anyInt || in;
    anyBand = anyBand || (e && !in);
  }
  T ce_[V], ch_[V], ax_[V], bx_[V], ay_[V], by_[V], sx[V], sy[V];
  if (live && anyInt) { vld(w.ce + k, ce_); vld(w.chy + k, ch_); }
  if (live && anyBand) {
    vld(w.ax + k, ax_); vld(w.bx + k, bx_); vld(w.ay + k, ay_); vld(w.by + k, by_);
    vldw(SxA + k, sx); vldw(SyA + k, sy);
  }
#pragma unroll
  for (int v = 0; v < V; ++v) {
    const int I = I0 + v;
    px[v] = py[v] = lm[v] = lx[v] = ly[v] = T(0);
    if (!(colE && I >= 1 && I <= w.NX - 1)) continue;
    if (colInt && I >= w.ei0 && I <= w.ei1) {
      px[v] = ch_[v] * l[v]; py[v] = (w.rxy * ch_[v]) * l[v]; lm[v] = ce_[v] * l[v];
    } else {
      lx[v] = sx[v] + l[v]; ly[v] = sy[v] + l[v];
      px[v] = bx_[v] * lx[v]; py[v] = by_[v] * ly[v];
    }
  }
}

// Exact adjoint step (see k_adj_step), vectorised.
template <class T>
__global__ void __launch_bounds__(128, GJ_MINB_ADJ) k_adj_stepv(const WDev<T> w, const AdjArgs<T> a) {
  constexpr int V = VT<T>::V;
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  const int i0w = (blockIdx.x * (blockDim.x >> 5) + warp) * (32 * V);
  const int ld = w.ld, NX = w.NX, NY = w.NY;
  if (i0w > NX) return;
  const int I0 = i0w + lane * V;
  const bool live = I0 <= NX;
  const int j0 = blockIdx.y * a.tj;
  if (j0 > NY) return;
  const int j1 = min(j0 + a.tj - 1, NY);
  const int zl = blockIdx.z;
  const int s = a.shot0 + zl;
  const size_t off = size_t(zl) * a.sstride, fs = a.fstride;
  const T* __restrict__ LA = a.A + off;
  const T* __restrict__ LxA = LA + fs;
  const T* __restrict__ LyA = LA + 2 * fs;
  const T* __restrict__ SxA = LA + 3 * fs;
  const T* __restrict__ SyA = LA + 4 * fs;
  T* __restrict__ LB = a.B + off;
  T* __restrict__ LxB = LB + fs;
  T* __restrict__ LyB = LB + 2 * fs;
  T* __restrict__ SxB = LB + 3 * fs;
  T* __restrict__ SyB = LB + 4 * fs;
  bool hyStrip = false;
#pragma unroll
  for (int v = 0; v < V; ++v) {
    const int I = I0 + v;
    if (I <= NX - 1 && !(I >= w.hyi0 && I <= w.hyi1)) hyStrip = true;
  }
  T l_c[V], px_c[V], py_c[V], lm_c[V], lx_c[V], ly_c[V];
  vzero<T, V>(l_c);
  {
    const size_t k = nidx(I0, j0, ld);
    if (live) vldw(LA + k, l_c);
    adj_pv<T, V>(w, I0, j0, k, live, l_c, SxA, SyA, px_c, py_c, lm_c, lx_c, ly_c);
  }
  T qx_prev[V];
  vzero<T, V>(qx_prev);
  if (j0 >= 1) {
    const size_t k = nidx(I0, j0 - 1, ld);
    T l_m[V], px_m[V], py_m[V], lm_m[V], lx_m[V], ly_m[V], lxo[V];
    vzero<T, V>(l_m); vzero<T, V>(lxo);
    if (live) { vldw(LA + k, l_m); vldw(LxA + k, lxo); }
    adj_pv<T, V>(w, I0, j0 - 1, k, live, l_m, SxA, SyA, px_m, py_m, lm_m, lx_m, ly_m);
#pragma unroll
    for (int v = 0; v < V; ++v)
      if (I0 + v <= NX) {
        T ha, hb; hx_coef(w, I0 + v, j0 - 1, ha, hb);
        qx_prev[v] = hb * (lxo[v] + py_m[v] - py_c[v]);
      }
  }
  for (int J = j0; J <= j1; ++J) {
    const size_t k = nidx(I0, J, ld);
    const size_t kn = k + ld;
    T l_n[V], px_n[V], py_n[V], lm_n[V], lx_n[V], ly_n[V], lxo[V], lyo[V];
    vzero<T, V>(l_n); vzero<T, V>(lxo); vzero<T, V>(lyo);
    if (live) { vldw(LA + kn, l_n); vldw(LxA + k, lxo); vldw(LyA + k, lyo); }
    adj_pv<T, V>(w, I0, J + 1, kn, live, l_n, SxA, SyA, px_n, py_n, lm_n, lx_n, ly_n);
    // px at rows I0+V (next lane) and I0-1 (previous lane)
    T px_dn = __shfl_down_sync(0xffffffffu, px_c[0], 1);
    T px_up = __shfl_up_sync(0xffffffffu, px_c[V - 1], 1);
    if (lane == 31) {
      px_dn = T(0);
      const int I = I0 + V;
      if (I <= NX) {
        T a1, a2, a3, a4;
        adj_p(w, I, J, k + V, LA[k + V], SxA[k + V], SyA[k + V], px_dn, a1, a2, a3, a4);
      }
    }
    if (lane == 0) {
      T a1, a2, a3, a4;
      adj_p(w, I0 - 1, J, k - 1, LA[k - 1], SxA[k - 1], SyA[k - 1], px_up, a1, a2, a3, a4);
    }
    // H-like half
    const bool hxStripCol = !(J >= w.hxj0 && J <= w.hxj1);
    T hxa_[V], hxb_[V], hya_[V], hyb_[V];
    if (live && hxStripCol) { vld(w.hxa + k, hxa_); vld(w.hxb + k, hxb_); }
    else {
#pragma unroll
      for (int v = 0; v < V; ++v) { hxa_[v] = T(1); hxb_[v] = w.chxez; }
    }
    if (live && hyStrip) { vld(w.hya + k, hya_); vld(w.hyb + k, hyb_); }
    T qx[V], qy[V], lxn[V], lyn[V];
#pragma unroll
    for (int v = 0; v < V; ++v) {
      const int I = I0 + v;
      qx[v] = qy[v] = lxn[v] = lyn[v] = T(0);
      if (I <= NX && J <= NY - 1) {
        const T lt = lxo[v] + py_c[v] - py_n[v];
        lxn[v] = hxa_[v] * lt;
        qx[v] = hxb_[v] * lt;
      }
      if (I <= NX - 1) {
        T ha = T(1), hb = w.chyez;
        if (!(I >= w.hyi0 && I <= w.hyi1)) { ha = hya_[v]; hb = hyb_[v]; }
        const T pdn = (v < V - 1) ? px_c[v < V - 1 ? v + 1 : v] : px_dn;
        const T lt = lyo[v] + px_c[v] - pdn;
        lyn[v] = ha * lt;
        qy[v] = hb * lt;
      }
    }
    if (live) { vst(LxB + k, lxn); vst(LyB + k, lyn); }
    T qy_up = __shfl_up_sync(0xffffffffu, qy[V - 1], 1);
    if (lane == 0) {
      qy_up = T(0);
      if (I0 >= 1) {
        T ha, hb; hy_coef(w, I0 - 1, J, ha, hb);
        qy_up = hb * (LyA[k - 1] + px_up - px_c[0]);
      }
    }
    // E-like half
    const bool colE = J >= 1 && J <= NY - 1;
    const bool colInt = J >= w.ej0 && J <= w.ej1;
    T le[V], sxn[V], syn[V], axv[V], ayv[V];
    bool anyBand = false;
#pragma unroll
    for (int v = 0; v < V; ++v) {
      const int I = I0 + v;
      const bool e = colE && I >= 1 && I <= NX - 1;
      anyBand = anyBand || (e && !(colInt && I >= w.ei0 && I <= w.ei1));
    }
    if (live && anyBand) { vld(w.ax + k, axv); vld(w.ay + k, ayv); }
    const bool dom = live && J >= w.dj0 && J < w.dj0 + w.n && colInt && drow(w, I0);
    T img1[V], img2[V];
    vzero<T, V>(img1); vzero<T, V>(img2);
#pragma unroll
    for (int v = 0; v < V; ++v) {
      const int I = I0 + v;
      le[v] = T(0); sxn[v] = T(0); syn[v] = T(0);
      if (!(colE && I >= 1 && I <= NX - 1)) continue;
      const T qym = (v > 0) ? qy[v > 0 ? v - 1 : 0] : qy_up;
      le[v] = lm_c[v] + qx_prev[v] - qx[v] + qym - qy[v];
      if (!(colInt && I >= w.ei0 && I <= w.ei1)) {
        sxn[v] = axv[v] * lx_c[v];
        syn[v] = ayv[v] * ly_c[v];
      } else if (I >= w.di0 && I < w.di0 + w.m) {
        img1[v] = l_c[v];
      }
    }
    if (dom) {
      // imaging at interior model nodes, domain-node layout (aligned vectors)
      const size_t q = size_t(zl) * a.hstride + dnode(w, I0, J);
      T e1[V], e0[V];
      vldw(a.ek + q, e1); vldw(a.ekm1 + q, e0);
      const size_t dn = size_t(w.hld) * size_t(w.n);
      T* acc = a.acc + size_t(s) * a.astride + dnode(w, I0, J);
      T sE[V], cE[V], sS[V], cS[V];
      vldw(acc, sE); vldw(acc + 2 * dn, sS);
      if (a.kahan) { vldw(acc + dn, cE); vldw(acc + 3 * dn, cS); }
#pragma unroll
      for (int v = 0; v < V; ++v) {
        img2[v] = img1[v] * (e1[v] + e0[v]);
        img1[v] = img1[v] * (e1[v] - e0[v]);
        if (a.kahan) {
          kahan_add(&sE[v], &cE[v], img1[v]);
          kahan_add(&sS[v], &cS[v], img2[v]);
        } else {
          sE[v] += img1[v];
          sS[v] += img2[v];
        }
      }
      vst(acc, sE); vst(acc + 2 * dn, sS);
      if (a.kahan) { vst(acc + dn, cE); vst(acc + 3 * dn, cS); }
    }
    if (live) {
      vst(LB + k, le);
      if (anyBand) { vst(SxB + k, sxn); vst(SyB + k, syn); }
    }
#pragma unroll
    for (int v = 0; v < V; ++v) {
      qx_prev[v] = qx[v];
      l_c[v] = l_n[v]; px_c[v] = px_n[v]; py_c[v] = py_n[v]; lm_c[v] = lm_n[v]; lx_c[v] = lx_n[v];
      ly_c[v] = ly_n[v];
    }
  }
}

}  // namespace gj

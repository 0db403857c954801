// Temporally blocked forward Yee steps (w_solve.m:80-105, several steps per
// pass).  Each CTA owns a tile of TR x TC nodes of one shot and stages the
// tile plus a halo of D nodes on every side (RR = 32 G rows x RC columns,
// TR = RR - 2D, TC = RC - 2D) in shared memory: Ez, Hx, Hy at level n (and
// the split fields Ezx, Ezy in PML tiles).  It then runs up to D complete Yee
// steps in place on the staged region (new_H + new_H_pml, one barrier,
// new_Ez + source + new_Ez_pml, one barrier) and writes the owned tile at
// level n + D.  Each step's stencil reads one node further out than the
// previous one, so after d steps the staged values are exact on the region
// shrunk by d nodes per side, and after D steps on the owned tile; the halo
// cells are recomputed redundantly by the neighbouring tiles, so no tile
// waits on another.  Nodes outside the (NX+1) x (NY+1) grid are staged as
// zero and never updated, which is what they are in the padded storage.
//
// Receivers (w_solve.m:100) and the source current Jz (w_solve.m:104) are
// recorded from shared memory after every step by the tile that owns their
// node.  A pass reads the state once and writes it once for D steps: 24 B per
// node and pass in FP32 (Ez, Hx, Hy in and out) against 24 B per node and step
// for one step per pass, plus the interior coefficients Ceze, Cezhy that stay
// in registers across the D steps and the shots of the CTA.
//
// Interior tiles (PML = false: every updated node of the staged region is an
// interior Ez node, an interior Hx column and an interior Hy row, as the host
// classifies them) stage three fields; PML tiles stage five and read the strip
// and split-field coefficients per step (they are shared by all shots and stay
// in L2).  The arithmetic is k_step's, node for node.
#pragma once
#include "w_kernels.cuh"

namespace gj {

constexpr int TB_WARPS = 8;  // warps per CTA of the temporally blocked kernels

template <class T>
struct TbArgs {
  const T* A;            // state at level n, [shot][field][node], base one column in
  T* B;                  // state at level n + nd
  size_t fstride, sstride;
  int gn;                // shots in the launch
  int spb;               // shots per CTA (consecutive shots; the coefficients stay in registers)
  int it, nd;            // first step of the pass and steps in it (1..D)
  const long* src;       // per shot (absolute index) linear source node or -1
  const T* cezj;         // per shot
  const T* wav;          // [shot][nt]
  int nt;
  int shot0;             // absolute index of the launch's first shot (source tables)
  const int* rs;         // per shot of the launch: nrr x {column J, row I, receiver r}, sorted by column
  const int* nrs;        // per shot of the launch: receivers
  int nrr;
  T* d;                  // traces of the launch's shots, [shot][nrr][nt], or nullptr
  T* jz;                 // Ez at the source node, [shot][nt], or nullptr
};

// Tile (int2): x = first owned row r0, y = first owned column c0.
// Thread mapping: a lane keeps one staged row, 32 (warp % G) + lane, for the
// whole pass and handles the columns warp / G + CS q, q = 0..Q-1 (CS = warps
// / G), so every shared-memory and global access of a warp covers 32
// consecutive rows of one column.
template <class T, int D, int G, int RC, bool PML>
__global__ void __launch_bounds__(32 * TB_WARPS, 2) k_fwd_tb(const WDev<T> w, const TbArgs<T> a,
                                                          const int2* __restrict__ tiles) {
  constexpr int RR = 32 * G, TR = RR - 2 * D, TC = RC - 2 * D;
  constexpr int CS = TB_WARPS / G;  // column step between a lane's items
  constexpr int Q = RC / CS;        // items (columns) per lane
  constexpr int PLANE = RR * RC;
  static_assert(TR > 0 && TC > 0 && TB_WARPS % G == 0 && RC % CS == 0, "tile too small for its halo");
  extern __shared__ __align__(16) unsigned char tbsm[];
  T* sEz = reinterpret_cast<T*>(tbsm);
  T* sHx = sEz + PLANE;
  T* sHy = sEz + 2 * PLANE;
  T* sEx = sEz + 3 * PLANE;  // PML tiles only
  T* sEy = sEz + 4 * PLANE;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int2 tk = tiles[blockIdx.x];
  const int r0 = tk.x, c0 = tk.y;
  const int ld = w.ld, NX = w.NX, NY = w.NY;
  const size_t fs = a.fstride;
  const int row = 32 * (wid % G) + lane, col0 = wid / G;
  const int i = r0 - D + row;
  // row classes (fixed for the pass)
  const bool rIn = i >= 0 && i <= NX;
  const bool rHy = i >= 0 && i <= NX - 1 && row < RR - 1;
  const bool rE = i >= 1 && i <= NX - 1 && row >= 1;
  const bool rEint = i >= w.ei0 && i <= w.ei1;
  const bool rHyInt = i >= w.hyi0 && i <= w.hyi1;
  const bool rOwn = rIn && row >= D && row < RR - D;
  // column classes of item q (recomputed where used; registers hold only the
  // interior coefficients): bit 0 Hx updated, 1 Hy updated, 2 Ez updated,
  // 3 interior Ez node, 4 interior Hx column, 6 in the grid, 7 owned
  auto cls = [&](int q) -> unsigned {
    const int col = col0 + CS * q, j = c0 - D + col;
    const bool cIn = j >= 0 && j <= NY;
    unsigned c = 0;
    if (rIn && cIn) c |= 64u;
    if (rIn && j >= 0 && j <= NY - 1 && col < RC - 1) c |= 1u;
    if (rHy && cIn) c |= 2u;
    if (rE && j >= 1 && j <= NY - 1 && col >= 1) c |= 4u;
    if (rEint && j >= w.ej0 && j <= w.ej1) c |= 8u;
    if (j >= w.hxj0 && j <= w.hxj1) c |= 16u;
    if (rOwn && cIn && col >= D && col < RC - D) c |= 128u;
    return c;
  };
  T rce[PML ? 1 : Q], rch[PML ? 1 : Q];
  if (!PML) {
#pragma unroll
    for (int q = 0; q < Q; ++q) {
      rce[q] = T(0); rch[q] = T(0);
      if ((cls(q) & 12u) == 12u) {
        const size_t kk = nidx(i, c0 - D + col0 + CS * q, ld);
        rce[q] = __ldg(w.ce + kk);
        rch[q] = __ldg(w.chy + kk);
      }
    }
  }
  const T rxy = w.rxy, chx = w.chxez, chy = w.chyez;

  for (int z = 0; z < a.spb; ++z) {
    const int zl = blockIdx.y * a.spb + z;
    if (zl >= a.gn) break;  // uniform over the CTA
    const int s = a.shot0 + zl;
    const size_t off = size_t(zl) * a.sstride;
    const T* EzA = a.A + off;
    T* EzB = a.B + off;
    if (z > 0) __syncthreads();  // the previous shot's stores have read the staged region
    // stage level n
#pragma unroll
    for (int q = 0; q < Q; ++q) {
      const int col = col0 + CS * q;
      const int p = col * RR + row;
      T ez = T(0), hx = T(0), hy = T(0), ex = T(0), ey = T(0);
      if (cls(q) & 64u) {
        const size_t kk = nidx(i, c0 - D + col, ld);
        ez = EzA[kk]; hx = EzA[fs + kk]; hy = EzA[2 * fs + kk];
        if (PML) { ex = EzA[3 * fs + kk]; ey = EzA[4 * fs + kk]; }
      }
      sEz[p] = ez; sHx[p] = hx; sHy[p] = hy;
      if (PML) { sEx[p] = ex; sEy[p] = ey; }
    }
    const long src = a.src[s];
    const int srcI = src >= 0 ? int(src % ld) : -1, srcJ = src >= 0 ? int(src / ld) : -1;
    const T cz = src >= 0 ? a.cezj[s] : T(0);
    // receivers of this shot whose column lies in the owned columns
    int rlo = 0, rhi = 0;
    const int* rsz = a.rs + size_t(zl) * a.nrr * 3;
    if (a.d) {
      const int n = a.nrs[zl];
      int lo = 0, hi = n;
      while (lo < hi) { const int mid = (lo + hi) >> 1; if (rsz[3 * mid] < c0) lo = mid + 1; else hi = mid; }
      rlo = lo; hi = n;
      while (lo < hi) { const int mid = (lo + hi) >> 1; if (rsz[3 * mid] < c0 + TC) lo = mid + 1; else hi = mid; }
      rhi = lo;
    }
    const bool ownSrc = src >= 0 && srcI >= r0 && srcI < r0 + TR && srcJ >= c0 && srcJ < c0 + TC;
    const bool srcRow = src >= 0 && i == srcI;
    __syncthreads();
    for (int d = 0; d < a.nd; ++d) {
      const int itd = a.it + d;
      // new_H, new_H_pml (w_solve.m:85-89)
#pragma unroll
      for (int q = 0; q < Q; ++q) {
        const unsigned c = cls(q);
        if (!(c & 3u)) continue;
        const int col = col0 + CS * q;
        const int p = col * RR + row;
        const T ez = sEz[p];
        if (c & 1u) {
          T ha = T(1), hb = chx;
          if (PML && !(c & 16u)) {
            const size_t kk = nidx(i, c0 - D + col, ld);
            ha = __ldg(w.hxa + kk); hb = __ldg(w.hxb + kk);
          }
          sHx[p] = ha * sHx[p] + hb * (sEz[p + RR] - ez);
        }
        if (c & 2u) {
          T ha = T(1), hb = chy;
          if (PML && !rHyInt) {
            const size_t kk = nidx(i, c0 - D + col, ld);
            ha = __ldg(w.hya + kk); hb = __ldg(w.hyb + kk);
          }
          sHy[p] = ha * sHy[p] + hb * (sEz[p + 1] - ez);
        }
      }
      __syncthreads();
      // new_Ez + source + new_Ez_pml (w_solve.m:91-94)
      const T sval = srcRow ? cz * a.wav[size_t(s) * a.nt + itd] : T(0);
#pragma unroll
      for (int q = 0; q < Q; ++q) {
        const unsigned c = cls(q);
        if (!(c & 4u)) continue;
        const int col = col0 + CS * q, j = c0 - D + col;
        const int p = col * RR + row;
        const T dhy = sHy[p] - sHy[p - 1];
        const T dhx = sHx[p] - sHx[p - RR];
        T e;
        if (!PML || (c & 8u)) {
          T ce = rce[PML ? 0 : q], ch = rch[PML ? 0 : q];
          if (PML) {
            const size_t kk = nidx(i, j, ld);
            ce = __ldg(w.ce + kk); ch = __ldg(w.chy + kk);
          }
          e = ce * sEz[p] + ch * dhy + (rxy * ch) * dhx;
          if (srcRow && j == srcJ) e += sval;
        } else {
          const size_t kk = nidx(i, j, ld);
          const T ex = __ldg(w.ax + kk) * sEx[p] + __ldg(w.bx + kk) * dhy;
          const T ey = __ldg(w.ay + kk) * sEy[p] + __ldg(w.by + kk) * dhx;
          sEx[p] = ex; sEy[p] = ey;
          e = ex + ey;
        }
        sEz[p] = e;
      }
      __syncthreads();
      // receivers and Jz after the step (w_solve.m:100, 104)
      for (int r = rlo + int(threadIdx.x); r < rhi; r += 32 * TB_WARPS) {
        const int J = rsz[3 * r], I = rsz[3 * r + 1], rr = rsz[3 * r + 2];
        if (I >= r0 && I < r0 + TR)
          a.d[(size_t(zl) * a.nrr + rr) * a.nt + itd] = sEz[(J - c0 + D) * RR + (I - r0 + D)];
      }
      if (a.jz && ownSrc && threadIdx.x == 0)
        a.jz[size_t(zl) * a.nt + itd] = sEz[(srcJ - c0 + D) * RR + (srcI - r0 + D)];
    }
    // owned tile at level n + nd
#pragma unroll
    for (int q = 0; q < Q; ++q) {
      if (!(cls(q) & 128u)) continue;
      const int col = col0 + CS * q;
      const int p = col * RR + row;
      const size_t kk = nidx(i, c0 - D + col, ld);
      EzB[kk] = sEz[p]; EzB[fs + kk] = sHx[p]; EzB[2 * fs + kk] = sHy[p];
      if (PML) { EzB[3 * fs + kk] = sEx[p]; EzB[4 * fs + kk] = sEy[p]; }
    }
  }
}

// Tile shapes: index -> (G, RC).
constexpr int TB_NSHAPE = 3;
__host__ __device__ constexpr int tb_shape_G(int sh) { return sh == 2 ? 4 : 2; }
__host__ __device__ constexpr int tb_shape_RC(int sh) { return sh == 1 ? 64 : 32; }
inline size_t tb_smem(int shape, bool pml, size_t tsize) {
  return size_t(pml ? 5 : 3) * 32 * tb_shape_G(shape) * tb_shape_RC(shape) * tsize;
}

template <class T>
using TbKernel = void (*)(const WDev<T>, const TbArgs<T>, const int2*);

template <class T, int G, int RC, bool P>
TbKernel<T> tb_kernel_d(int D) {
  switch (D) {
    case 1: return k_fwd_tb<T, 1, G, RC, P>;
    case 2: return k_fwd_tb<T, 2, G, RC, P>;
    case 3: return k_fwd_tb<T, 3, G, RC, P>;
    default: return k_fwd_tb<T, 4, G, RC, P>;
  }
}
template <class T>
TbKernel<T> tb_kernel(int D, int shape, bool pml) {
  if (shape == 1) return pml ? tb_kernel_d<T, 2, 64, true>(D) : tb_kernel_d<T, 2, 64, false>(D);
  if (shape == 2) return pml ? tb_kernel_d<T, 4, 32, true>(D) : tb_kernel_d<T, 4, 32, false>(D);
  return pml ? tb_kernel_d<T, 2, 32, true>(D) : tb_kernel_d<T, 2, 32, false>(D);
}

}  // namespace gj

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
// classifies them, w_tblock_plan.h) stage three fields; PML tiles stage five
// and keep the strip and split-field coefficients of their nodes in registers
// for the pass (narrow tiles) or read them per step from L2 (wider tiles).
// The gradient's forward (when asked for) also writes the u history and the
// band history of the exact adjoint of every step.  The arithmetic is
// k_step's, node for node.  The streaming interior tasks (k_fwd_tbs, below)
// cover the interior of large grids; these tiles then cover the rest.
#pragma once
#include "w_kernels_ring.cuh"
#include "w_band.cuh"

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
  const long* src;       // per shot (shot0 + zl % spt) linear source node or -1
  const T* cezj;         // per launch shot (shot0 + zl)
  const T* wav;          // [shot][nt] (shot0 + zl % spt)
  int nt;
  int shot0;             // absolute index of the launch's first shot (source tables)
  const int* rs;         // per shot (zl % spt): nrr x {column J, row I, receiver r}, sorted by column
  const int* nrs;        // per shot (zl % spt): receivers
  int nrr;
  T* d;                  // traces of the launch's shots, [shot][nrr][nt], or nullptr
  T* jz;                 // Ez at the source node, [shot][nt], or nullptr
  // batches of models (the trial models of a step-length search): launch shot
  // zl is shot zl % spt of model zl / spt, whose coefficient arrays lie
  // (zl / spt) * cstride elements after the WDev ones; cezj is per launch shot
  int spt;
  size_t cstride;
  // gradient forward: the u history (domain-node layout, per shot hstride;
  // step it + d's slot at hist + d hslot) and the band history of the exact
  // adjoint (band frame, per shot w.bsz; step it + d's slot at band + d
  // bslot), the slots of step it + 1 given; nullptr when not kept
  T* hist; size_t hstride, hslot;
  T* band; size_t bslot;
};

// Tile (int4): owned rows [x, x + z), owned columns [y, y + w), z <= TR and
// w <= TC (tiles at the edge of a region are clipped).
// Thread mapping: a lane keeps one staged row, 32 (warp % G) + lane, for the
// whole pass and handles the columns warp / G + CS q, q = 0..Q-1 (CS = warps
// / G), so every shared-memory and global access of a warp covers 32
// consecutive rows of one column.
template <class T, int D, int G, int RC, bool PML>
__global__ void __launch_bounds__(32 * TB_WARPS, 2) k_fwd_tb(const WDev<T> w, const TbArgs<T> a,
                                                          const int4* __restrict__ tiles) {
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
  const int4 tk = tiles[blockIdx.x];
  const int r0 = tk.x, c0 = tk.y, tr = tk.z, tc = tk.w;
  const int ld = w.ld, NX = w.NX, NY = w.NY;
  const size_t fs = a.fstride;
  const int row = 32 * (wid % G) + lane, col0 = wid / G;
  const int i = r0 - D + row;
  // coefficients of the CTA's model (the host keeps a CTA's shots in one model)
  const size_t co = size_t(blockIdx.y * a.spb / a.spt) * a.cstride;
  // row classes (fixed for the pass)
  const bool rIn = i >= 0 && i <= NX;
  const bool rHy = i >= 0 && i <= NX - 1 && row < RR - 1;
  const bool rE = i >= 1 && i <= NX - 1 && row >= 1;
  const bool rEint = i >= w.ei0 && i <= w.ei1;
  const bool rHyInt = i >= w.hyi0 && i <= w.hyi1;
  const bool rOwn = rIn && row >= D && row < D + tr;
  // column classes of item q (recomputed where used; registers hold only the
  // interior coefficients): bit 0 Hx updated, 1 Hy updated, 2 Ez updated,
  // 3 interior Ez node, 4 interior Hx column, 6 in the grid, 7 owned
  auto cls_of = [&](int q) -> unsigned {
    const int col = col0 + CS * q, j = c0 - D + col;
    const bool cIn = j >= 0 && j <= NY;
    unsigned c = 0;
    if (rIn && cIn) c |= 64u;
    if (rIn && j >= 0 && j <= NY - 1 && col < RC - 1) c |= 1u;
    if (rHy && cIn) c |= 2u;
    if (rE && j >= 1 && j <= NY - 1 && col >= 1) c |= 4u;
    if (rEint && j >= w.ej0 && j <= w.ej1) c |= 8u;
    if (j >= w.hxj0 && j <= w.hxj1) c |= 16u;
    if (rOwn && cIn && col >= D && col < D + tc) c |= 128u;
    return c;
  };
  // the class bytes of the Q items, four per register
  unsigned clsw[(Q + 3) / 4];
#pragma unroll
  for (int k = 0; k < (Q + 3) / 4; ++k) clsw[k] = 0;
#pragma unroll
  for (int q = 0; q < Q; ++q) clsw[q >> 2] |= cls_of(q) << (8 * (q & 3));
  auto cls = [&](int q) -> unsigned { return (clsw[q >> 2] >> (8 * (q & 3))) & 0xffu; };
  T rce[PML ? 1 : Q], rch[PML ? 1 : Q];
  if (!PML) {
#pragma unroll
    for (int q = 0; q < Q; ++q) {
      rce[q] = T(0); rch[q] = T(0);
      if ((cls(q) & 12u) == 12u) {
        const size_t kk = nidx(i, c0 - D + col0 + CS * q, ld);
        rce[q] = __ldg(w.ce + co + kk);
        rch[q] = __ldg(w.chy + co + kk);
      }
    }
  }
  const T rxy = w.rxy, chx = w.chxez, chy = w.chyez;
  // PML tiles of the narrow shape keep every coefficient of their items in
  // registers for the pass (E: Ceze/Cezhy or ax, bx, ay, by; Hx and Hy
  // pairs); wider PML tiles read them per step (L2).
  constexpr bool CACHE = PML && Q <= 8;
  constexpr int QC = CACHE ? Q : 1;
  T kA[QC], kB[QC], kC[QC], kD[QC], kXa[QC], kXb[QC], kYa[QC], kYb[QC];
  if (CACHE) {
#pragma unroll
    for (int q = 0; q < QC; ++q) {
      const unsigned c = cls(q);
      kA[q] = kB[q] = kC[q] = kD[q] = T(0);
      kXa[q] = T(1); kXb[q] = chx; kYa[q] = T(1); kYb[q] = chy;
      if (!(c & 64u)) continue;
      const size_t kk = nidx(i, c0 - D + col0 + CS * q, ld);
      if (c & 4u) {
        if (c & 8u) { kA[q] = __ldg(w.ce + co + kk); kB[q] = __ldg(w.chy + co + kk); }
        else { kA[q] = __ldg(w.ax + co + kk); kB[q] = __ldg(w.bx + co + kk); kC[q] = __ldg(w.ay + co + kk); kD[q] = __ldg(w.by + co + kk); }
      }
      if ((c & 1u) && !(c & 16u)) { kXa[q] = __ldg(w.hxa + co + kk); kXb[q] = __ldg(w.hxb + co + kk); }
      if ((c & 2u) && !rHyInt) { kYa[q] = __ldg(w.hya + co + kk); kYb[q] = __ldg(w.hyb + co + kk); }
    }
  }

  for (int z = 0; z < a.spb; ++z) {
    const int zl = blockIdx.y * a.spb + z;
    if (zl >= a.gn) break;  // uniform over the CTA
    const int sp = zl % a.spt;  // shot of the model
    const int s = a.shot0 + sp;
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
    const T cz = src >= 0 ? a.cezj[a.shot0 + zl] : T(0);
    // receivers of this shot whose column lies in the owned columns
    int rlo = 0, rhi = 0;
    const int* rsz = a.rs + size_t(sp) * a.nrr * 3;
    if (a.d) {
      const int n = a.nrs[sp];
      int lo = 0, hi = n;
      while (lo < hi) { const int mid = (lo + hi) >> 1; if (rsz[3 * mid] < c0) lo = mid + 1; else hi = mid; }
      rlo = lo; hi = n;
      while (lo < hi) { const int mid = (lo + hi) >> 1; if (rsz[3 * mid] < c0 + tc) lo = mid + 1; else hi = mid; }
      rhi = lo;
    }
    const bool ownSrc = src >= 0 && srcI >= r0 && srcI < r0 + tr && srcJ >= c0 && srcJ < c0 + tc;
    const bool srcRow = src >= 0 && i == srcI;
    // thread t records receiver rlo + t of the owned tile (its shared-memory
    // offset and trace index kept for the pass); the rare receivers past the
    // first 32 TB_WARPS of the tile are read again at every step
    int myP = -1;
    size_t myD = 0;
    if (rlo + int(threadIdx.x) < rhi) {
      const int r = rlo + int(threadIdx.x);
      const int J = rsz[3 * r], I = rsz[3 * r + 1], rr = rsz[3 * r + 2];
      if (I >= r0 && I < r0 + tr) {
        myP = (J - c0 + D) * RR + (I - r0 + D);
        myD = (size_t(zl) * a.nrr + rr) * a.nt;
      }
    }
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
          if (CACHE) { ha = kXa[CACHE ? q : 0]; hb = kXb[CACHE ? q : 0]; }
          else if (PML && !(c & 16u)) {
            const size_t kk = nidx(i, c0 - D + col, ld);
            ha = __ldg(w.hxa + co + kk); hb = __ldg(w.hxb + co + kk);
          }
          sHx[p] = ha * sHx[p] + hb * (sEz[p + RR] - ez);
        }
        if (c & 2u) {
          T ha = T(1), hb = chy;
          if (CACHE) { ha = kYa[CACHE ? q : 0]; hb = kYb[CACHE ? q : 0]; }
          else if (PML && !rHyInt) {
            const size_t kk = nidx(i, c0 - D + col, ld);
            ha = __ldg(w.hya + co + kk); hb = __ldg(w.hyb + co + kk);
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
          if (CACHE) { ce = kA[CACHE ? q : 0]; ch = kB[CACHE ? q : 0]; }
          else if (PML) {
            const size_t kk = nidx(i, j, ld);
            ce = __ldg(w.ce + co + kk); ch = __ldg(w.chy + co + kk);
          }
          e = ce * sEz[p] + ch * dhy + (rxy * ch) * dhx;
          if (srcRow && j == srcJ) e += sval;
        } else {
          T ax_, bx_, ay_, by_;
          if (CACHE) { ax_ = kA[CACHE ? q : 0]; bx_ = kB[CACHE ? q : 0]; ay_ = kC[CACHE ? q : 0]; by_ = kD[CACHE ? q : 0]; }
          else {
            const size_t kk = nidx(i, j, ld);
            ax_ = __ldg(w.ax + co + kk); bx_ = __ldg(w.bx + co + kk); ay_ = __ldg(w.ay + co + kk); by_ = __ldg(w.by + co + kk);
          }
          const T ex = ax_ * sEx[p] + bx_ * dhy;
          const T ey = ay_ * sEy[p] + by_ * dhx;
          sEx[p] = ex; sEy[p] = ey;
          e = ex + ey;
        }
        sEz[p] = e;
      }
      __syncthreads();
      // receivers and Jz after the step (w_solve.m:100, 104)
      if (myP >= 0) a.d[myD + itd] = sEz[myP];
      for (int r = rlo + 32 * TB_WARPS + int(threadIdx.x); r < rhi; r += 32 * TB_WARPS) {
        const int J = rsz[3 * r], I = rsz[3 * r + 1], rr = rsz[3 * r + 2];
        if (I >= r0 && I < r0 + tr)
          a.d[(size_t(zl) * a.nrr + rr) * a.nt + itd] = sEz[(J - c0 + D) * RR + (I - r0 + D)];
      }
      if (a.jz && ownSrc && threadIdx.x == 0)
        a.jz[size_t(zl) * a.nt + itd] = sEz[(srcJ - c0 + D) * RR + (srcI - r0 + D)];
      // u history and band history of the step (owned nodes; as the ring kernels write them)
      if (a.hist || a.band) {
        const bool hrow = a.hist && drow(w, i);
        const bool brow = a.band && i < w.bRB;
#pragma unroll
        for (int q = 0; q < Q; ++q) {
          if (!(cls(q) & 128u)) continue;
          const int col = col0 + CS * q, j = c0 - D + col;
          const int p = col * RR + row;
          if (hrow && j >= w.dj0 && j < w.dj0 + w.n)
            a.hist[size_t(d) * a.hslot + size_t(zl) * a.hstride + dnode(w, i, j)] = sEz[p];
          if (brow) {
            T* bs = a.band + size_t(d) * a.bslot + size_t(zl) * w.bsz;
            const long oe = band_off_e(w, i, j, 0);
            if (oe >= 0) {
              const bool bn = PML && ez_bandnode(w, i, j);
              bs[oe] = bn ? sEx[p] : T(0);
              bs[oe + (i >= w.bR0 ? w.bBsz : w.bLsz)] = bn ? sEy[p] : T(0);
            }
            const long ox = band_off_hx(w, i, j);
            if (ox >= 0) bs[ox] = sHx[p];
            const long oy = band_off_hy(w, i, j);
            if (oy >= 0) bs[oy] = sHy[p];
            if (i == NX) {  // the frame's rows below the grid hold zeros (no tile owns them)
              for (int r2 = NX + 1; r2 < w.bRB; ++r2) {
                const long o2 = band_off_e(w, r2, j, 0);
                if (o2 >= 0) { bs[o2] = T(0); bs[o2 + (r2 >= w.bR0 ? w.bBsz : w.bLsz)] = T(0); }
                const long x2 = band_off_hx(w, r2, j);
                if (x2 >= 0) bs[x2] = T(0);
                const long y2 = band_off_hy(w, r2, j);
                if (y2 >= 0) bs[y2] = T(0);
              }
            }
          }
        }
      }
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

// --------------------------------------------------------------------------
// Streaming temporal blocking of the interior (k_fwd_tbs).  One warp per task
// (first loaded row R, output columns [c0, c1], shot): the lanes hold 32 V
// rows (V per lane, 16-byte vectors) and march along the columns with the
// level-0 data of the next S-1 columns in flight in a shared-memory ring
// (cp.async), as the one-step ring kernels do.  The D steps of a pass form a
// wavefront in registers: when column J arrives, step 1 updates column J,
// step 2 column J-1 (from step 1's outputs of columns J-1 and J and its own
// Hx of column J-2), ..., step D column J-D+1, which is stored.  Each level
// keeps its input columns and Ceze / Cezhy in registers, so a pass reads the
// state and the coefficients once and writes the state once for D steps.
// Row halos come only from the level-0 loads; a level's values are exact one
// row further in per step, so after D steps rows [R + D - 1, R + 32 V - D]
// are exact (from row 0 when R = 0: the grid above row 0 is zero at every
// level); the host spaces tasks so that their owned rows tile the region.
// Task (int4): x = R, y = c0 | c1 << 16, z = own_lo | own_hi << 16 (owned
// rows), w = shot in the launch | TBS_HAS_REC.  The streamed region
// is interior (no PML, no edge, no strip coefficient); the host covers the
// rest of the grid with clipped tiles of k_fwd_tb in the same pass.
// Receivers and the source are handled per level (time index it + d - 1).
// --------------------------------------------------------------------------
constexpr int TBS_WARPS = 4;  // warps (tasks) per CTA of k_fwd_tbs
constexpr int TBS_HAS_REC = 1 << 20;  // task flag: a receiver of the shot lies in the task's owned nodes
inline size_t tbs_smem(int S) { return size_t(TBS_WARPS) * S * RING_STAGE_FAST * 16; }

template <class T, int S, int D>
__global__ void __launch_bounds__(32 * TBS_WARPS) k_fwd_tbs(const WDev<T> w, const TbArgs<T> a,
                                                            const int4* __restrict__ tasks, int ntask) {
  constexpr int V = VT<T>::V;
  constexpr int SLOTS = RING_SLOTS_FAST, STAGE = RING_STAGE_FAST;
  static_assert(V * sizeof(T) == 16, "streaming tasks move 16 bytes per lane");
  extern __shared__ __align__(16) uint4 tbs_ring[];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const int t = blockIdx.x * TBS_WARPS + wib;
  if (t >= ntask) return;  // whole warp; no CTA barrier in this kernel
  const int4 tk = tasks[t];
  const int R = tk.x, c0 = tk.y & 0xffff, c1 = tk.y >> 16, zl = tk.w & (TBS_HAS_REC - 1);
  const int sp = zl % a.spt;                           // shot of the model
  const size_t co = size_t(zl / a.spt) * a.cstride;    // coefficients of the model
  const int ld = w.ld;
  const int I0 = R + lane * V;
  const bool upl = lane == 0, dnl = lane == 31;
  const size_t off = size_t(zl) * a.sstride, fs = a.fstride;
  const T* EzA = a.A + off;
  const T* HxA = EzA + fs;
  const T* HyA = EzA + 2 * fs;
  T* EzB = a.B + off;
  T* HxB = EzB + fs;
  T* HyB = EzB + 2 * fs;
  uint4* ring = tbs_ring + size_t(wib) * S * STAGE;
  const int s = a.shot0 + sp;
  const int own_lo = tk.z & 0xffff, own_hi = tk.z >> 16;
  unsigned own = 0;
#pragma unroll
  for (int v = 0; v < V; ++v)
    if (I0 + v >= own_lo && I0 + v < own_hi) own |= 1u << v;
  const long src = a.src[s];
  const int srcJ = src >= 0 ? int(src / ld) : -1, srcI = src >= 0 ? int(src % ld) : -1;
  const bool srcLane = srcI >= I0 && srcI < I0 + V;
  T sv[D];
#pragma unroll
  for (int d = 0; d < D; ++d) sv[d] = srcLane ? a.cezj[a.shot0 + zl] * a.wav[size_t(s) * a.nt + a.it + d] : T(0);
  const T chx = w.chxez, chy = w.chyez, rxy = w.rxy;
  const int Js = c0 - D + 1, Je = c1 + D - 1;
  auto issue = [&](int J, int stg) {
    uint4* Rg = ring + size_t(stg) * STAGE;
    uint4* L = Rg + lane;
    const size_t k = nidx(I0, J, ld);
    cp16(L + RF_EZN * 32, EzA + k + ld);
    cp16(L + RF_HX * 32, HxA + k);
    cp16(L + RF_HY * 32, HyA + k);
    cp16(L + RF_CE * 32, w.ce + co + k);
    cp16(L + RF_CH * 32, w.chy + co + k);
    uint4* H = Rg + SLOTS * 32;
    if (dnl) cp16(H + HF_EZDN, EzA + nidx(I0 + V, J, ld));
    if (upl && I0 >= 1) {
      const size_t ku = nidx(I0 - V, J, ld);
      cp16(H + HF_EZUP, EzA + ku);
      cp16(H + HF_HYUP, HyA + ku);
    }
    cp_commit();
  };
  for (int p = 0; p < S - 1; ++p) {
    if (Js + p <= Je) issue(Js + p, p);
    else cp_commit();
  }
  // level 1: Ez(Js) and Hx_new(Js - 1) from global memory
  T ez_c[V], hx1[V];
  vldw(EzA + nidx(I0, Js, ld), ez_c);
  {
    T ezm[V], hxo[V];
    vldw(EzA + nidx(I0, Js - 1, ld), ezm);
    vldw(HxA + nidx(I0, Js - 1, ld), hxo);
#pragma unroll
    for (int v = 0; v < V; ++v) hx1[v] = T(1) * hxo[v] + chx * (ez_c[v] - ezm[v]);
  }
  // levels 2..D: the previous column's outputs of the level below, own Hx of
  // the previous column; Ceze / Cezhy of the last D columns (index d - 1:
  // the column of level d)
  T pE[D][V], pHx[D][V], pHy[D][V], hxp[D][V], ceq[D][V], chq[D][V];
#pragma unroll
  for (int d = 0; d < D; ++d) {
    vzero<T, V>(pE[d]); vzero<T, V>(pHx[d]); vzero<T, V>(pHy[d]); vzero<T, V>(hxp[d]);
    vzero<T, V>(ceq[d]); vzero<T, V>(chq[d]);
  }
  // receivers (tasks flagged by the host as holding some): a window of the
  // shot's column-sorted list from the first one at a column >= c0, lane q
  // holding entry q; per level the index of its next receiver and that
  // receiver's column (entries past the window are read from global memory)
  const int* rsl = a.rs + size_t(sp) * 3 * a.nrr;
  const int rn = (a.d && (tk.w & TBS_HAS_REC)) ? a.nrs[sp] : 0;
  const int rp0 = rn ? rec_first(rsl, rn, c0) : 0;
  int wJ = 0x7fffffff, wI = 0, wR = 0;
  if (rp0 + lane < rn) { wJ = rsl[3 * (rp0 + lane)]; wI = rsl[3 * (rp0 + lane) + 1]; wR = rsl[3 * (rp0 + lane) + 2]; }
  int rq[D], nJ[D];
#pragma unroll
  for (int d = 0; d < D; ++d) { rq[d] = 0; nJ[d] = __shfl_sync(0xffffffffu, wJ, 0); }
  auto record = [&](int d, int K, const T (&E)[V]) {
    while (nJ[d] == K && K <= c1) {  // warp-uniform
      const int q = rq[d];
      int I, r;
      if (q < 32) { I = __shfl_sync(0xffffffffu, wI, q); r = __shfl_sync(0xffffffffu, wR, q); }
      else { I = rsl[3 * (rp0 + q) + 1]; r = rsl[3 * (rp0 + q) + 2]; }
      if (I >= I0 && I < I0 + V && ((own >> (I - I0)) & 1u)) {
        T val = T(0);
#pragma unroll
        for (int v = 0; v < V; ++v)
          if (I == I0 + v) val = E[v];
        a.d[(size_t(zl) * a.nrr + r) * a.nt + a.it + d] = val;
      }
      rq[d] = q + 1;
      if (q + 1 < 32) nJ[d] = __shfl_sync(0xffffffffu, wJ, q + 1);
      else nJ[d] = rp0 + q + 1 < rn ? rsl[3 * (rp0 + q + 1)] : 0x7fffffff;
    }
    // Jz = Ez at the source node after the step (w_solve.m:104)
    if (a.jz && K == srcJ && K >= c0 && K <= c1 && srcLane && ((own >> (srcI - I0)) & 1u)) {
      T val = T(0);
#pragma unroll
      for (int v = 0; v < V; ++v)
        if (srcI == I0 + v) val = E[v];
      a.jz[size_t(zl) * a.nt + a.it + d] = val;
    }
  };
  // u history of level d at column K (owned rows; the layout's rows as the ring kernels write them)
  const bool hlane = a.hist && own && drow(w, I0);
  auto hist_store = [&](int d, int K, const T (&E)[V]) {
    if (!hlane || K < c0 || K > c1 || K < w.dj0 || K >= w.dj0 + w.n) return;
    T* hp = a.hist + size_t(d) * a.hslot + size_t(zl) * a.hstride + dnode(w, I0, K);
    if (own == (1u << V) - 1u) {
      vst(hp, E);
    } else {
#pragma unroll
      for (int v = 0; v < V; ++v)
        if ((own >> v) & 1u) hp[v] = E[v];
    }
  };
  for (int J = Js; J <= Je; ++J) {
    const int it = J - Js;
    if (J + S - 1 <= Je) issue(J + S - 1, (it + S - 1) % S);
    else cp_commit();
    cp_wait<S - 1>();
    const uint4* Rg = ring + size_t(it % S) * STAGE;
    const uint4* L = Rg + lane;
    const uint4* H = Rg + SLOTS * 32;
    T ez_n[V], hxo[V], hyo[V];
    sld(L + RF_EZN * 32, ez_n); sld(L + RF_HX * 32, hxo); sld(L + RF_HY * 32, hyo);
    sld(L + RF_CE * 32, ceq[0]); sld(L + RF_CH * 32, chq[0]);
    // ---- level 1, column J
    T E[V], HX[V], HY[V];
    {
      T nxt = __shfl_down_sync(0xffffffffu, ez_c[0], 1);
      if (dnl) nxt = sfirst<T>(H + HF_EZDN);
#pragma unroll
      for (int v = 0; v < V; ++v) {
        HX[v] = T(1) * hxo[v] + chx * (ez_n[v] - ez_c[v]);
        const T edn = (v < V - 1) ? ez_c[v < V - 1 ? v + 1 : v] : nxt;
        HY[v] = T(1) * hyo[v] + chy * (edn - ez_c[v]);
      }
      T hy_up = __shfl_up_sync(0xffffffffu, HY[V - 1], 1);
      if (upl) {
        hy_up = T(0);
        if (I0 >= 1) hy_up = T(1) * slast<T>(H + HF_HYUP) + chy * (ez_c[0] - slast<T>(H + HF_EZUP));
      }
#pragma unroll
      for (int v = 0; v < V; ++v) {
        const T dhy = HY[v] - (v > 0 ? HY[v > 0 ? v - 1 : 0] : hy_up);
        const T dhx = HX[v] - hx1[v];
        E[v] = ceq[0][v] * ez_c[v] + chq[0][v] * dhy + (rxy * chq[0][v]) * dhx;
      }
      if (J == srcJ && srcLane) {
#pragma unroll
        for (int v = 0; v < V; ++v)
          if (srcI == I0 + v) E[v] += sv[0];
      }
      record(0, J, E);
      hist_store(0, J, E);
#pragma unroll
      for (int v = 0; v < V; ++v) { hx1[v] = HX[v]; ez_c[v] = ez_n[v]; }
    }
    // ---- levels 2..D, column J - d + 1
#pragma unroll
    for (int d = 1; d < D; ++d) {
      const int K = J - d;
      T E2[V], HX2[V], HY2[V];
      T nxt = __shfl_down_sync(0xffffffffu, pE[d][0], 1);
      if (dnl) nxt = T(0);  // below the task: not exact at this level (rows not owned)
#pragma unroll
      for (int v = 0; v < V; ++v) {
        HX2[v] = T(1) * pHx[d][v] + chx * (E[v] - pE[d][v]);
        const T edn = (v < V - 1) ? pE[d][v < V - 1 ? v + 1 : v] : nxt;
        HY2[v] = T(1) * pHy[d][v] + chy * (edn - pE[d][v]);
      }
      T hy_up = __shfl_up_sync(0xffffffffu, HY2[V - 1], 1);
      if (upl) hy_up = T(0);  // row R - 1: zero above the grid (R = 0), else not owned
#pragma unroll
      for (int v = 0; v < V; ++v) {
        const T dhy = HY2[v] - (v > 0 ? HY2[v > 0 ? v - 1 : 0] : hy_up);
        const T dhx = HX2[v] - hxp[d][v];
        E2[v] = ceq[d][v] * pE[d][v] + chq[d][v] * dhy + (rxy * chq[d][v]) * dhx;
      }
      if (K == srcJ && srcLane) {
#pragma unroll
        for (int v = 0; v < V; ++v)
          if (srcI == I0 + v) E2[v] += sv[d];
      }
      record(d, K, E2);
      hist_store(d, K, E2);
#pragma unroll
      for (int v = 0; v < V; ++v) {
        hxp[d][v] = HX2[v];
        pE[d][v] = E[v]; pHx[d][v] = HX[v]; pHy[d][v] = HY[v];
        E[v] = E2[v]; HX[v] = HX2[v]; HY[v] = HY2[v];
      }
    }
    // ---- level D output, column J - D + 1
    const int KD = J - D + 1;
    if (KD >= c0 && KD <= c1 && own) {
      const size_t k = nidx(I0, KD, ld);
      if (own == (1u << V) - 1u) {
        vst(EzB + k, E); vst(HxB + k, HX); vst(HyB + k, HY);
      } else {
#pragma unroll
        for (int v = 0; v < V; ++v)
          if ((own >> v) & 1u) { EzB[k + v] = E[v]; HxB[k + v] = HX[v]; HyB[k + v] = HY[v]; }
      }
    }
#pragma unroll
    for (int d = D - 1; d > 0; --d)
#pragma unroll
      for (int v = 0; v < V; ++v) { ceq[d][v] = ceq[d - 1][v]; chq[d][v] = chq[d - 1][v]; }
  }
  cp_wait<0>();
}

template <class T>
using TbsKernel = void (*)(const WDev<T>, const TbArgs<T>, const int4*, int);
// Ring stages of the streaming tasks: 3 (two columns in flight) or 6.
template <class T, int S>
TbsKernel<T> tbs_kernel_s(int D) {
  switch (D) {
    case 1: return k_fwd_tbs<T, S, 1>;
    case 2: return k_fwd_tbs<T, S, 2>;
    case 3: return k_fwd_tbs<T, S, 3>;
    default: return k_fwd_tbs<T, S, 4>;
  }
}
template <class T>
TbsKernel<T> tbs_kernel(int D, int S) {
  return S >= 6 ? tbs_kernel_s<T, 6>(D) : tbs_kernel_s<T, 3>(D);
}

// Tile shapes: index -> (G, RC).
constexpr int TB_NSHAPE = 3;
__host__ __device__ constexpr int tb_shape_G(int sh) { return sh == 2 ? 4 : 2; }
__host__ __device__ constexpr int tb_shape_RC(int sh) { return sh == 1 ? 64 : 32; }
inline size_t tb_smem(int shape, bool pml, size_t tsize) {
  return size_t(pml ? 5 : 3) * 32 * tb_shape_G(shape) * tb_shape_RC(shape) * tsize;
}

template <class T>
using TbKernel = void (*)(const WDev<T>, const TbArgs<T>, const int4*);

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

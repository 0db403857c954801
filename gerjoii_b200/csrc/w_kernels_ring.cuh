// Warp-task ring kernels.  Each warp runs one task: a block of 32*V rows
// (V rows per lane, 16-byte vectors) of one shot, marching along a chunk of
// columns [j0, j1].  Warps are independent (no CTA barrier): every lane
// streams the data of its own rows for the next S-1 columns into a per-warp
// shared-memory ring with cp.async (16-byte copies, one commit group per
// column), and lanes 0 and 31 stream the 16-byte vectors just above and
// below the block (the i-halo) the same way, so no load in the loop waits on
// global memory.
//
// Two code paths per column: the general one (every row class, the PML band
// and the grid edges, arithmetic of k_stepv<T, 0> / k_adj_stepv<T>), and a
// branch-free one taken when the whole task block is interior rows and the
// column is interior (scalar H coefficients, Ceze/Cezhy arrays, no split
// fields).  The free-top layout stores Ceze = 1, Cezhy = 0 on the Ez = 0 row,
// so blocks that start at row 0 take the fast path too (Ez there stays 0 and
// its adjoint is cleared).  Tasks are listed by the host, general-path
// blocks first with shorter column chunks.
//
// The exact adjoint stores the adjoint field of the interior model nodes into
// a ring of Kd slots; k_image applies the imaging condition
// S1 += l (E^k - E^{k-1}), S2 += l (E^k + E^{k-1}) over those slots in one
// streaming pass.
#pragma once
#include "w_kernels_vec.cuh"
#include "w_band.cuh"

namespace gj {

__device__ __forceinline__ unsigned smem_addr(const void* p) {
  return static_cast<unsigned>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void cp16(void* dst, const void* src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(smem_addr(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}
__device__ __forceinline__ void sld(const uint4* p, float (&r)[4]) {
  const float4 x = *reinterpret_cast<const float4*>(p);
  r[0] = x.x; r[1] = x.y; r[2] = x.z; r[3] = x.w;
}
__device__ __forceinline__ void sld(const uint4* p, double (&r)[2]) {
  const double2 x = *reinterpret_cast<const double2*>(p);
  r[0] = x.x; r[1] = x.y;
}
// First / last element of a 16-byte halo vector.
template <class T> __device__ __forceinline__ T sfirst(const uint4* p) { return *reinterpret_cast<const T*>(p); }
template <class T> __device__ __forceinline__ T slast(const uint4* p) {
  return reinterpret_cast<const T*>(p)[16 / sizeof(T) - 1];
}

constexpr int RING_SLOTS = 15;  // 16-byte entries per lane per column
constexpr int RING_HALO = 16;   // 16-byte halo entries per warp per column
constexpr int RING_STAGE = RING_SLOTS * 32 + RING_HALO;  // uint4 per warp per stage
// The fast-only variants keep 5 entries per lane and 5 halo entries.
constexpr int RING_SLOTS_FAST = 5;
constexpr int RING_STAGE_FAST = RING_SLOTS_FAST * 32 + 5;
template <bool FAST> struct RingShape {
  static constexpr int slots = FAST ? RING_SLOTS_FAST : RING_SLOTS;
  static constexpr int stage = FAST ? RING_STAGE_FAST : RING_STAGE;
};

// Forward slots for column J.
enum { RF_EZN = 0, RF_HX, RF_HY, RF_CE, RF_CH, RF_HXA, RF_HXB, RF_HYA, RF_HYB, RF_AX, RF_BX, RF_AY, RF_BY,
       RF_EX, RF_EY };
// Forward halo: below the block (lane 31) and above it (lane 0), column J.
enum { HF_EZDN = 0, HF_EZUP, HF_HYUP, HF_HYAUP, HF_HYBUP };
// Adjoint slots: data of column J+1 (p-values) and of column J (H-like half).
enum { RA_LN = 0, RA_CE, RA_CH, RA_AX, RA_BX, RA_AY, RA_BY, RA_SX, RA_SY, RA_LX, RA_LY, RA_HXA, RA_HXB,
       RA_HYA, RA_HYB };
// Adjoint halo, column J: p-value inputs below (lane 31) and above (lane 0).
enum { HA_LDN = 0, HA_SXDN, HA_CHDN, HA_BXDN, HA_LUP, HA_SXUP, HA_CHUP, HA_BXUP, HA_LYUP, HA_HYBUP };

// Receivers of the launch's shots for the fused record (forward) and
// injection (exact adjoint): per shot nrr entries {column J, row I, receiver r}
// sorted by column, `nrs` valid.  Traces are [shot in launch][r][t].
template <class T>
struct RecArgs {
  const int* rs;   // first shot of the launch
  const int* nrs;  // first shot of the launch
  int nrr, nt;
  T* d; int it;          // forward: d(r, it) = Ez after the step (k_record), when d
  const T* e; int kinj;  // adjoint: output += e(r, kinj) (k_inject_add of the next step), when kinj >= 0
};

// First receiver of a shot's column-sorted list at column >= j0.
__device__ __forceinline__ int rec_first(const int* rs, int n, int j0) {
  int lo = 0, hi = n;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (rs[3 * mid] < j0) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

// Shared memory of a launch with `warps` warps per CTA and S stages.
inline size_t ring_smem(int warps, int S, bool fast) {
  return size_t(warps) * S * (fast ? RING_STAGE_FAST : RING_STAGE) * 16;
}

// Task of one warp (int4): x = first row r0, y, z = first and last column,
// w = (shot within the launch << 1) | fast, fast = 1 when every row of
// [r0, r0+32V-1] is an interior Ez row (or the free-top Ez = 0 row) and a Hy
// interior row, and the halo rows r0-1 (when r0 > 0) and r0+32V are
// interior Ez and Hy rows.  FAST kernels run only tasks of fast blocks
// restricted to interior columns (forward [ej0, ej1], adjoint [ej0, ej1-1])
// and keep only the fast path.

// --------------------------------------------------------------------------
// Forward Yee step (w_solve.m:85-105): new_H, new_H_pml, new_Ez, source,
// new_Ez_pml; history of the domain Ez (domain-node layout) when a.hist.
// Grid: x = tasks / warps per CTA.
// --------------------------------------------------------------------------
template <class T, int S, bool FAST>
__global__ void __launch_bounds__(128) k_fwdw(const WDev<T> w, const StepArgs<T> a, const int4* __restrict__ tasks,
                                              int ntask, const RecArgs<T> ra) {
  constexpr int SLOTS = RingShape<FAST>::slots, STAGE = RingShape<FAST>::stage;
  constexpr int V = VT<T>::V;
  static_assert(V * sizeof(T) == 16, "ring kernels move 16 bytes per lane");
  extern __shared__ __align__(16) uint4 smem[];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const int t = blockIdx.x * (blockDim.x >> 5) + wib;
  if (t >= ntask) return;  // whole warp; the kernel has no CTA barrier
  const int4 tk = tasks[t];
  const int ld = w.ld, NX = w.NX, NY = w.NY;
  // split task (general kernel, bottom block): lanes 0-15 run shot z, lanes
  // 16-31 shot z+1 over the same 64 rows; a half's first lane loads its own
  // up-halo (second half: halo entries shifted by 5, past the first half's
  // five), its last lane reads the zero padding below NX
  const bool split = !FAST && ((tk.w >> 1) & 1);
  const int half = split ? (lane >> 4) : 0;
  const int hl = split ? (lane & 15) : lane;
  const bool upl = hl == 0, dnl = split ? hl == 15 : lane == 31;
  const int hoff = half ? 5 : 0;
  const int I0 = tk.x + hl * V;
  const int j0 = tk.y, j1 = tk.z;
  const bool fastRows = (tk.w & 1) != 0;
  const bool live = I0 <= NX;
  const int zl = (tk.w >> 2) + half;
  const int s = a.shot0 + zl;
  const size_t off = size_t(zl) * a.sstride, fs = a.fstride;
  const T* EzA = a.A + off;
  const T* HxA = EzA + fs;
  const T* HyA = EzA + 2 * fs;
  const T* ExA = EzA + 3 * fs;
  const T* EyA = EzA + 4 * fs;
  T* EzB = a.B + off;
  T* HxB = EzB + fs;
  T* HyB = EzB + 2 * fs;
  T* ExB = EzB + 3 * fs;
  T* EyB = EzB + 4 * fs;
  uint4* ring = smem + size_t(wib) * S * STAGE;
  const long src = a.src[s];
  T sval = T(0);
  if (src >= 0) sval = a.cezj[s] * a.wav[size_t(s) * a.nt + a.it];
  const int srcJ = src >= 0 ? int(src / ld) : -1, srcI = src >= 0 ? int(src % ld) : -1;
  bool hyStrip = false, rowBandAny = false, rowIntAny = false;
#pragma unroll
  for (int v = 0; v < V; ++v) {
    const int I = I0 + v;
    const bool rint = I >= w.ei0 && I <= w.ei1;
    rowIntAny = rowIntAny || rint;
    if (I <= NX - 1 && !(I >= w.hyi0 && I <= w.hyi1)) hyStrip = true;
    if (I >= 1 && I <= NX - 1 && !rint) rowBandAny = true;
  }
  const int Iup = I0 - 1;  // lane 0's halo row
  const bool upStrip = Iup >= 0 && Iup <= NX - 1 && !(Iup >= w.hyi0 && Iup <= w.hyi1);
  // row classes of this lane's V rows as bit masks (the general path selects
  // per row instead of branching): Hx row, Hy row, Hy interior row, updated
  // Ez row, interior Ez row
  unsigned mHx = 0, mHy = 0, mHyInt = 0, mE = 0, mEint = 0;
#pragma unroll
  for (int v = 0; v < V; ++v) {
    const int I = I0 + v;
    if (I <= NX) mHx |= 1u << v;
    if (I <= NX - 1) mHy |= 1u << v;
    if (I >= w.hyi0 && I <= w.hyi1) mHyInt |= 1u << v;
    if (I >= 1 && I <= NX - 1) mE |= 1u << v;
    if (I >= w.ei0 && I <= w.ei1) mEint |= 1u << v;
  }
  auto colInt = [&](int J) { return J >= w.ej0 && J <= w.ej1; };
  auto colE = [&](int J) { return J >= 1 && J <= NY - 1; };
  auto hxStrip = [&](int J) { return !(J >= w.hxj0 && J <= w.hxj1); };
  auto needInt = [&](int J) { return colInt(J) && rowIntAny; };
  auto needBand = [&](int J) { return colE(J) && (rowBandAny || (!colInt(J) && rowIntAny)); };
  auto issue = [&](int J, int stg) {
    uint4* R = ring + size_t(stg) * STAGE;
    if (FAST) {
      uint4* L = R + lane;
      const size_t k = nidx(I0, J, ld);
      cp16(L + RF_EZN * 32, EzA + k + ld);
      cp16(L + RF_HX * 32, HxA + k);
      cp16(L + RF_HY * 32, HyA + k);
      cp16(L + RF_CE * 32, w.ce + k);
      cp16(L + RF_CH * 32, w.chy + k);
      uint4* H = R + SLOTS * 32;
      if (dnl) cp16(H + HF_EZDN, EzA + nidx(I0 + V, J, ld));
      if (upl && I0 >= 1) {
        const size_t ku = nidx(I0 - V, J, ld);
        cp16(H + HF_EZUP, EzA + ku);
        cp16(H + HF_HYUP, HyA + ku);
      }
    } else if (live) {
      uint4* L = R + lane;
      const size_t k = nidx(I0, J, ld);
      cp16(L + RF_EZN * 32, EzA + k + ld);
      cp16(L + RF_HX * 32, HxA + k);
      cp16(L + RF_HY * 32, HyA + k);
      if (needInt(J)) { cp16(L + RF_CE * 32, w.ce + k); cp16(L + RF_CH * 32, w.chy + k); }
      if (hxStrip(J)) { cp16(L + RF_HXA * 32, w.hxa + k); cp16(L + RF_HXB * 32, w.hxb + k); }
      if (hyStrip) { cp16(L + RF_HYA * 32, w.hya + k); cp16(L + RF_HYB * 32, w.hyb + k); }
      if (needBand(J)) {
        cp16(L + RF_AX * 32, w.ax + k); cp16(L + RF_BX * 32, w.bx + k);
        cp16(L + RF_AY * 32, w.ay + k); cp16(L + RF_BY * 32, w.by + k);
        cp16(L + RF_EX * 32, ExA + k); cp16(L + RF_EY * 32, EyA + k);
      }
      uint4* H = R + SLOTS * 32 + hoff;
      if (dnl && I0 + V <= NX) cp16(H + HF_EZDN, EzA + nidx(I0 + V, J, ld));
      if (upl && I0 >= 1) {
        const size_t ku = nidx(I0 - V, J, ld);
        cp16(H + HF_EZUP, EzA + ku);
        cp16(H + HF_HYUP, HyA + ku);
        if (upStrip) { cp16(H + HF_HYAUP, w.hya + ku); cp16(H + HF_HYBUP, w.hyb + ku); }
      }
    }
    cp_commit();
  };
  for (int p = 0; p < S - 1; ++p) {
    if (j0 + p <= j1) issue(j0 + p, p);
    else cp_commit();
  }
  // Ez(j0) and Hx_new(j0-1) from global memory (once per task)
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
  // receiver window (fused k_record): lane q holds receiver rp + q of this
  // shot's column-sorted list, from the first one at column >= j0
  const int* rsl = ra.rs + size_t(zl) * 3 * ra.nrr;
  const int rn = (ra.d && !split) ? ra.nrs[zl] : 0;  // split tasks hold no receivers
  int rp = rn ? rec_first(rsl, rn, j0) : 0;
  int wJ = 0x7fffffff, wI = 0, wR = 0, widx = 0;
  auto rec_window = [&]() {
    const int q = rp + lane;
    wJ = 0x7fffffff;
    if (q < rn) { wJ = rsl[3 * q]; wI = rsl[3 * q + 1]; wR = rsl[3 * q + 2]; }
    widx = 0;
  };
  if (rn) rec_window();
  int rJ = __shfl_sync(0xffffffffu, wJ, 0);
  for (int J = j0; J <= j1; ++J) {
    const int it = J - j0;
    if (J + S - 1 <= j1) issue(J + S - 1, (it + S - 1) % S);
    else cp_commit();
    cp_wait<S - 1>();
    const uint4* R = ring + size_t(it % S) * STAGE;
    const uint4* L = R + lane;
    const uint4* H = R + SLOTS * 32 + hoff;
    const size_t k = nidx(I0, J, ld);
    T ez_n[V], hxo[V], hyo[V], hx_new[V], hy_new[V], e_new[V];
    if (FAST || (fastRows && J >= w.ej0 && J <= w.ej1)) {
      // ---- interior block, interior column: no PML, no edges
      T ce_[V], ch_[V];
      sld(L + RF_EZN * 32, ez_n); sld(L + RF_HX * 32, hxo); sld(L + RF_HY * 32, hyo);
      sld(L + RF_CE * 32, ce_); sld(L + RF_CH * 32, ch_);
      T nxt = __shfl_down_sync(0xffffffffu, ez_c[0], 1);
      if (dnl) nxt = sfirst<T>(H + HF_EZDN);
#pragma unroll
      for (int v = 0; v < V; ++v) {
        hx_new[v] = T(1) * hxo[v] + w.chxez * (ez_n[v] - ez_c[v]);
        const T edn = (v < V - 1) ? ez_c[v < V - 1 ? v + 1 : v] : nxt;
        hy_new[v] = T(1) * hyo[v] + w.chyez * (edn - ez_c[v]);
      }
      vst(HxB + k, hx_new); vst(HyB + k, hy_new);
      T hy_up = __shfl_up_sync(0xffffffffu, hy_new[V - 1], 1);
      if (upl) {
        hy_up = T(0);
        if (I0 >= 1) hy_up = T(1) * slast<T>(H + HF_HYUP) + w.chyez * (ez_c[0] - slast<T>(H + HF_EZUP));
      }
#pragma unroll
      for (int v = 0; v < V; ++v) {
        const T dhy = hy_new[v] - (v > 0 ? hy_new[v > 0 ? v - 1 : 0] : hy_up);
        const T dhx = hx_new[v] - hx_prev[v];
        e_new[v] = ce_[v] * ez_c[v] + ch_[v] * dhy + (w.rxy * ch_[v]) * dhx;
      }
      if (J == srcJ && srcI >= I0 && srcI < I0 + V) {
#pragma unroll
        for (int v = 0; v < V; ++v)
          if (srcI == I0 + v) e_new[v] += sval;
      }
      vst(EzB + k, e_new);
    } else if constexpr (!FAST) {
      // ---- general path (w_solve.m:136-268 with every row class)
      vzero<T, V>(ez_n); vzero<T, V>(hxo); vzero<T, V>(hyo);
      if (live) { sld(L + RF_EZN * 32, ez_n); sld(L + RF_HX * 32, hxo); sld(L + RF_HY * 32, hyo); }
      const bool hxs = hxStrip(J);
      T hxa_[V], hxb_[V], hya_[V], hyb_[V];
      if (live && hxs) { sld(L + RF_HXA * 32, hxa_); sld(L + RF_HXB * 32, hxb_); }
      else {
#pragma unroll
        for (int v = 0; v < V; ++v) { hxa_[v] = T(1); hxb_[v] = w.chxez; }
      }
      vzero<T, V>(hya_); vzero<T, V>(hyb_);
      if (live && hyStrip) { sld(L + RF_HYA * 32, hya_); sld(L + RF_HYB * 32, hyb_); }
      T nxt = __shfl_down_sync(0xffffffffu, ez_c[0], 1);
      if (dnl) nxt = (I0 + V <= NX) ? sfirst<T>(H + HF_EZDN) : T(0);
      const bool hxCol = J <= NY - 1;
#pragma unroll
      for (int v = 0; v < V; ++v) {
        const T hxv = hxa_[v] * hxo[v] + hxb_[v] * (ez_n[v] - ez_c[v]);
        hx_new[v] = (hxCol && ((mHx >> v) & 1u)) ? hxv : T(0);
        const T edn = (v < V - 1) ? ez_c[v < V - 1 ? v + 1 : v] : nxt;
        const bool hin = (mHyInt >> v) & 1u;
        const T ha = hin ? T(1) : hya_[v], hb = hin ? w.chyez : hyb_[v];
        const T hyv = ha * hyo[v] + hb * (edn - ez_c[v]);
        hy_new[v] = ((mHy >> v) & 1u) ? hyv : T(0);
      }
      if (live) { vst(HxB + k, hx_new); vst(HyB + k, hy_new); }
      T hy_up = __shfl_up_sync(0xffffffffu, hy_new[V - 1], 1);
      if (upl) {
        hy_up = T(0);
        if (live && I0 >= 1 && Iup <= NX - 1) {
          T ha = T(1), hb = w.chyez;
          if (upStrip) { ha = slast<T>(H + HF_HYAUP); hb = slast<T>(H + HF_HYBUP); }
          hy_up = ha * slast<T>(H + HF_HYUP) + hb * (ez_c[0] - slast<T>(H + HF_EZUP));
        }
      }
      const bool cE = colE(J);
      const bool cInt = colInt(J);
      const bool anyInt = needInt(J);
      const bool anyBand = needBand(J);
      T ce_[V], ch_[V], ax_[V], bx_[V], ay_[V], by_[V], exo[V], eyo[V];
      if (live && anyInt) { sld(L + RF_CE * 32, ce_); sld(L + RF_CH * 32, ch_); }
      else { vzero<T, V>(ce_); vzero<T, V>(ch_); }
      if (live && anyBand) {
        sld(L + RF_AX * 32, ax_); sld(L + RF_BX * 32, bx_); sld(L + RF_AY * 32, ay_); sld(L + RF_BY * 32, by_);
        sld(L + RF_EX * 32, exo); sld(L + RF_EY * 32, eyo);
      } else {
        vzero<T, V>(ax_); vzero<T, V>(bx_); vzero<T, V>(ay_); vzero<T, V>(by_); vzero<T, V>(exo); vzero<T, V>(eyo);
      }
      const bool srcCol = J == srcJ;
#pragma unroll
      for (int v = 0; v < V; ++v) {
        const bool rE = cE && ((mE >> v) & 1u);
        const bool rI = rE && cInt && ((mEint >> v) & 1u);
        const bool rB = rE && !rI;
        const T dhy = hy_new[v] - (v > 0 ? hy_new[v > 0 ? v - 1 : 0] : hy_up);
        const T dhx = hx_new[v] - hx_prev[v];
        T ei = ce_[v] * ez_c[v] + ch_[v] * dhy + (w.rxy * ch_[v]) * dhx;
        if (srcCol && I0 + v == srcI) ei += sval;
        const T exn = ax_[v] * exo[v] + bx_[v] * dhy;
        const T eyn = ay_[v] * eyo[v] + by_[v] * dhx;
        e_new[v] = rI ? ei : (rB ? exn + eyn : ez_c[v]);
        exo[v] = rB ? exn : exo[v];
        eyo[v] = rB ? eyn : eyo[v];
      }
      if (live) {
        vst(EzB + k, e_new);
        if (anyBand) { vst(ExB + k, exo); vst(EyB + k, eyo); }
      }
      // band history of the exact adjoint (w_band.cuh): the split fields at
      // the band nodes (zero elsewhere) and the strip H fields after the step
      if (a.band && live && I0 < w.bRB) {
        T* bs = a.band + size_t(zl) * w.bsz;
        const long oe = band_off_e(w, I0, J, 0);
        if (oe >= 0) { vst(bs + oe, exo); vst(bs + oe + (I0 >= w.bR0 ? w.bBsz : w.bLsz), eyo); }
        const long ox = band_off_hx(w, I0, J);
        if (ox >= 0) vst(bs + ox, hx_new);
        const long oy = band_off_hy(w, I0, J);
        if (oy >= 0) vst(bs + oy, hy_new);
      }
    }
    if (live && a.hist && J >= w.dj0 && J < w.dj0 + w.n && drow(w, I0))
      vst(a.hist + size_t(zl) * a.hstride + dnode(w, I0, J), e_new);
    while (rJ == J) {  // d(it, r) = Ez(receiver) after the step (w_solve.m:100)
      const int I = __shfl_sync(0xffffffffu, wI, widx), r = __shfl_sync(0xffffffffu, wR, widx);
      if (I >= I0 && I < I0 + V) {
        T val = T(0);
#pragma unroll
        for (int v = 0; v < V; ++v)
          if (I == I0 + v) val = e_new[v];
        ra.d[(size_t(zl) * ra.nrr + r) * ra.nt + ra.it] = val;
      }
      if (++widx == 32) { rp += 32; rec_window(); }
      rJ = __shfl_sync(0xffffffffu, wJ, widx);
    }
#pragma unroll
    for (int v = 0; v < V; ++v) { hx_prev[v] = hx_new[v]; ez_c[v] = ez_n[v]; }
  }
  cp_wait<0>();
}

// Per-lane row predicates of the adjoint's p-values (adj_pv).
struct AdjRows {
  bool eAny, inAny, outAny;  // some row in [1, NX-1]; of those, some interior / some band
};

// p-values of V nodes of column J from ring data (same arithmetic as adj_pv),
// selecting per row by the lane's row masks.
template <class T, int V>
__device__ __forceinline__ void adj_pv_ring(const WDev<T>& w, int J, bool live, const AdjRows& rr, unsigned mE,
                                            unsigned mEint, const uint4* L, const T (&l)[V], T (&px)[V],
                                            T (&py)[V], T (&lm)[V], T (&lx)[V], T (&ly)[V], T (&axn)[V],
                                            T (&ayn)[V]) {
  const bool colE = J >= 1 && J <= w.NY - 1;
  const bool colInt = J >= w.ej0 && J <= w.ej1;
  const bool anyInt = colE && colInt && rr.inAny;
  const bool anyBand = colE && (colInt ? rr.outAny : rr.eAny);
  T ce_[V], ch_[V], bx_[V], by_[V], sx[V], sy[V];
  if (live && anyInt) { sld(L + RA_CE * 32, ce_); sld(L + RA_CH * 32, ch_); }
  else { vzero<T, V>(ce_); vzero<T, V>(ch_); }
  if (live && anyBand) {
    sld(L + RA_AX * 32, axn); sld(L + RA_BX * 32, bx_); sld(L + RA_AY * 32, ayn); sld(L + RA_BY * 32, by_);
    sld(L + RA_SX * 32, sx); sld(L + RA_SY * 32, sy);
  } else {
    vzero<T, V>(bx_); vzero<T, V>(by_); vzero<T, V>(sx); vzero<T, V>(sy);
  }
#pragma unroll
  for (int v = 0; v < V; ++v) {
    const bool rE = colE && ((mE >> v) & 1u);
    const bool rI = rE && colInt && ((mEint >> v) & 1u);
    const bool rB = rE && !rI;
    const T lxv = sx[v] + l[v], lyv = sy[v] + l[v];
    px[v] = rI ? ch_[v] * l[v] : (rB ? bx_[v] * lxv : T(0));
    py[v] = rI ? (w.rxy * ch_[v]) * l[v] : (rB ? by_[v] * lyv : T(0));
    lm[v] = rI ? ce_[v] * l[v] : T(0);
    lx[v] = rB ? lxv : T(0);
    ly[v] = rB ? lyv : T(0);
  }
}

// Node class of (I, J) for the adjoint's p-value: 1 interior, 2 band, 0 none.
template <class T>
__device__ __forceinline__ int adj_class(const WDev<T>& w, int I, int J) {
  if (I >= w.ei0 && I <= w.ei1 && J >= w.ej0 && J <= w.ej1) return 1;
  if (I >= 1 && I <= w.NX - 1 && J >= 1 && J <= w.NY - 1) return 2;
  return 0;
}
// px of a halo node from its adjoint l, split adjoint sx and coefficients.
template <class T>
__device__ __forceinline__ T halo_px(int cls, T l, T sx, T ch, T bx) {
  if (cls == 1) return ch * l;
  if (cls == 2) return bx * (sx + l);
  return T(0);
}

// --------------------------------------------------------------------------
// Exact adjoint step (transpose of k_fwdw), adjoint field of the interior
// model nodes into a.lout (domain-node layout; zero elsewhere in the model
// columns) for k_image.  Grid: x = tasks / warps per CTA.
// --------------------------------------------------------------------------
template <class T>
struct AdjRingArgs {
  const T* A; T* B; size_t fstride, sstride;
  int shot0;
  T* lout; size_t hstride;
  T* band;  // adjoint band slot of this step (w.bsz per shot, w_band.cuh), or nullptr
};

template <class T, int S, bool FAST>
__global__ void __launch_bounds__(128) k_adjw(const WDev<T> w, const AdjRingArgs<T> a, const int4* __restrict__ tasks,
                                              int ntask, const RecArgs<T> ra) {
  constexpr int SLOTS = RingShape<FAST>::slots, STAGE = RingShape<FAST>::stage;
  constexpr int V = VT<T>::V;
  static_assert(V * sizeof(T) == 16, "ring kernels move 16 bytes per lane");
  extern __shared__ __align__(16) uint4 smem[];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const int t = blockIdx.x * (blockDim.x >> 5) + wib;
  if (t >= ntask) return;
  const int4 tk = tasks[t];
  const int ld = w.ld, NX = w.NX, NY = w.NY;
  // split task (general kernel, bottom block): lanes 0-15 run shot z, lanes
  // 16-31 shot z+1 (see k_fwdw); the second half's halo entries are shifted
  // by 6.  Its down-halo entries (6-9) would overlap the first half's up-halo
  // ones, but a split task's last lanes have Idn > NX and load no down-halo.
  const bool split = !FAST && ((tk.w >> 1) & 1);
  const int half = split ? (lane >> 4) : 0;
  const int hl = split ? (lane & 15) : lane;
  const bool upl = hl == 0, dnl = split ? hl == 15 : lane == 31;
  const int hoff = half ? 6 : 0;
  const int I0 = tk.x + hl * V;
  const int j0 = tk.y, j1 = tk.z;
  const bool fastRows = (tk.w & 1) != 0;
  const bool live = I0 <= NX;
  const int zl = (tk.w >> 2) + half;
  const size_t off = size_t(zl) * a.sstride, fs = a.fstride;
  const T* LA = a.A + off;
  const T* LxA = LA + fs;
  const T* LyA = LA + 2 * fs;
  const T* SxA = LA + 3 * fs;
  const T* SyA = LA + 4 * fs;
  T* LB = a.B + off;
  T* LxB = LB + fs;
  T* LyB = LB + 2 * fs;
  T* SxB = LB + 3 * fs;
  T* SyB = LB + 4 * fs;
  uint4* ring = smem + size_t(wib) * S * STAGE;
  bool hyStrip = false;
  AdjRows rr{false, false, false};
  unsigned dmask = 0;  // model rows of this lane
#pragma unroll
  for (int v = 0; v < V; ++v) {
    const int I = I0 + v;
    if (I <= NX - 1 && !(I >= w.hyi0 && I <= w.hyi1)) hyStrip = true;
    if (I >= 1 && I <= NX - 1) {
      rr.eAny = true;
      if (I >= w.ei0 && I <= w.ei1) rr.inAny = true;
      else rr.outAny = true;
    }
    if (I >= w.di0 && I < w.di0 + w.m) dmask |= 1u << v;
  }
  const int Idn = I0 + V, Iup = I0 - 1;  // halo rows of lanes 31 and 0
  const bool upStrip = Iup >= 0 && Iup <= NX - 1 && !(Iup >= w.hyi0 && Iup <= w.hyi1);
  // row classes as bit masks (see k_fwdw)
  unsigned mHx = 0, mHy = 0, mHyInt = 0, mE = 0, mEint = 0;
#pragma unroll
  for (int v = 0; v < V; ++v) {
    const int I = I0 + v;
    if (I <= NX) mHx |= 1u << v;
    if (I <= NX - 1) mHy |= 1u << v;
    if (I >= w.hyi0 && I <= w.hyi1) mHyInt |= 1u << v;
    if (I >= 1 && I <= NX - 1) mE |= 1u << v;
    if (I >= w.ei0 && I <= w.ei1) mEint |= 1u << v;
  }
  auto pvNeed = [&](int J, bool& anyInt, bool& anyBand) {
    const bool colE = J >= 1 && J <= NY - 1;
    const bool colInt = J >= w.ej0 && J <= w.ej1;
    anyInt = colE && colInt && rr.inAny;
    anyBand = colE && (colInt ? rr.outAny : rr.eAny);
  };
  auto issue = [&](int J, int stg) {
    uint4* R = ring + size_t(stg) * STAGE;
    if (FAST) {
      uint4* L = R + lane;
      const size_t k = nidx(I0, J, ld), kn = k + ld;
      cp16(L + RF_EZN * 32, LA + kn);       // slot 0: l(J+1)
      cp16(L + RF_HX * 32, LxA + k);        // slot 1: lx(J)
      cp16(L + RF_HY * 32, LyA + k);        // slot 2: ly(J)
      cp16(L + RF_CE * 32, w.ce + kn);      // slot 3: Ceze(J+1)
      cp16(L + RF_CH * 32, w.chy + kn);     // slot 4: Cezhy(J+1)
      uint4* H = R + SLOTS * 32;
      if (dnl) {
        const size_t kd = nidx(Idn, J, ld);
        cp16(H + 0, LA + kd);
        cp16(H + 1, w.chy + kd);
      }
      if (upl && I0 >= 1) {
        const size_t ku = nidx(I0 - V, J, ld);
        cp16(H + 2, LA + ku);
        cp16(H + 3, w.chy + ku);
        cp16(H + 4, LyA + ku);
      }
    } else if (live) {
      uint4* L = R + lane;
      const size_t k = nidx(I0, J, ld), kn = k + ld;
      cp16(L + RA_LN * 32, LA + kn);
      bool ai, ab;
      pvNeed(J + 1, ai, ab);
      if (ai) { cp16(L + RA_CE * 32, w.ce + kn); cp16(L + RA_CH * 32, w.chy + kn); }
      if (ab) {
        cp16(L + RA_AX * 32, w.ax + kn); cp16(L + RA_BX * 32, w.bx + kn);
        cp16(L + RA_AY * 32, w.ay + kn); cp16(L + RA_BY * 32, w.by + kn);
        cp16(L + RA_SX * 32, SxA + kn); cp16(L + RA_SY * 32, SyA + kn);
      }
      cp16(L + RA_LX * 32, LxA + k);
      cp16(L + RA_LY * 32, LyA + k);
      if (!(J >= w.hxj0 && J <= w.hxj1)) { cp16(L + RA_HXA * 32, w.hxa + k); cp16(L + RA_HXB * 32, w.hxb + k); }
      if (hyStrip) { cp16(L + RA_HYA * 32, w.hya + k); cp16(L + RA_HYB * 32, w.hyb + k); }
      uint4* H = R + SLOTS * 32 + hoff;
      if (dnl && Idn <= NX) {
        const size_t kd = nidx(Idn, J, ld);
        const int cls = adj_class(w, Idn, J);
        if (cls) cp16(H + HA_LDN, LA + kd);
        if (cls == 1) cp16(H + HA_CHDN, w.chy + kd);
        if (cls == 2) { cp16(H + HA_SXDN, SxA + kd); cp16(H + HA_BXDN, w.bx + kd); }
      }
      if (upl && I0 >= 1) {
        const size_t ku = nidx(I0 - V, J, ld);
        const int cls = adj_class(w, Iup, J);
        if (cls) cp16(H + HA_LUP, LA + ku);
        if (cls == 1) cp16(H + HA_CHUP, w.chy + ku);
        if (cls == 2) { cp16(H + HA_SXUP, SxA + ku); cp16(H + HA_BXUP, w.bx + ku); }
        cp16(H + HA_LYUP, LyA + ku);
        if (upStrip) cp16(H + HA_HYBUP, w.hyb + ku);
      }
    }
    cp_commit();
  };
  for (int p = 0; p < S - 1; ++p) {
    if (j0 + p <= j1) issue(j0 + p, p);
    else cp_commit();
  }
  // column j0 and the H-like q of column j0-1 from global memory (once per task)
  T l_c[V], px_c[V], py_c[V], lm_c[V], lx_c[V], ly_c[V], ax_c[V], ay_c[V];
  vzero<T, V>(l_c); vzero<T, V>(ax_c); vzero<T, V>(ay_c);
  {
    const size_t k = nidx(I0, j0, ld);
    if (live) vldw(LA + k, l_c);
    adj_pv<T, V>(w, I0, j0, k, live, l_c, SxA, SyA, px_c, py_c, lm_c, lx_c, ly_c);
    bool ai, ab;
    pvNeed(j0, ai, ab);
    if (live && ab) { vld(w.ax + k, ax_c); vld(w.ay + k, ay_c); }
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
  // receiver window (fused injection of the next step's adjoint source):
  // lane q holds receiver rp + q of this shot's column-sorted list and its e
  const int* rsl = ra.rs + size_t(zl) * 3 * ra.nrr;
  const int rn = (ra.kinj >= 0 && !split) ? ra.nrs[zl] : 0;  // split tasks hold no receivers
  int rp = rn ? rec_first(rsl, rn, j0) : 0;
  int wJ = 0x7fffffff, wI = 0, widx = 0;
  T wE = T(0);
  auto rec_window = [&]() {
    const int q = rp + lane;
    wJ = 0x7fffffff;
    if (q < rn) {
      wJ = rsl[3 * q]; wI = rsl[3 * q + 1];
      wE = ra.e[(size_t(zl) * ra.nrr + rsl[3 * q + 2]) * ra.nt + ra.kinj];
    }
    widx = 0;
  };
  if (rn) rec_window();
  int rJ = __shfl_sync(0xffffffffu, wJ, 0);
  // output += e(receiver, kinj) at the receivers of column J (k_inject_add)
  auto inject = [&](int J, T (&le)[V]) {
    while (rJ == J) {
      const int I = __shfl_sync(0xffffffffu, wI, widx);
      const T ev = __shfl_sync(0xffffffffu, wE, widx);
      if (I >= I0 && I < I0 + V) {
#pragma unroll
        for (int v = 0; v < V; ++v)
          if (I == I0 + v) le[v] += ev;
      }
      if (++widx == 32) { rp += 32; rec_window(); }
      rJ = __shfl_sync(0xffffffffu, wJ, widx);
    }
  };
  for (int J = j0; J <= j1; ++J) {
    const int it = J - j0;
    if (J + S - 1 <= j1) issue(J + S - 1, (it + S - 1) % S);
    else cp_commit();
    cp_wait<S - 1>();
    const uint4* R = ring + size_t(it % S) * STAGE;
    const uint4* L = R + lane;
    const uint4* H = R + SLOTS * 32 + hoff;
    const size_t k = nidx(I0, J, ld);
    T l_n[V], px_n[V], py_n[V], lm_n[V], lx_n[V], ly_n[V], ax_n[V], ay_n[V], lxo[V], lyo[V];
    T lxn[V], lyn[V], qx[V], le[V], img[V];
    if (FAST || (fastRows && J >= w.ej0 && J + 1 <= w.ej1)) {
      // ---- interior block, interior columns J and J+1
      T ce_[V], ch_[V];
      T ldn, chdn, lup = T(0), chup = T(0), lyup = T(0);
      if (FAST) {
        sld(L + RF_EZN * 32, l_n); sld(L + RF_HX * 32, lxo); sld(L + RF_HY * 32, lyo);
        sld(L + RF_CE * 32, ce_); sld(L + RF_CH * 32, ch_);
        ldn = sfirst<T>(H + 0); chdn = sfirst<T>(H + 1);
        if (I0 >= 1) { lup = slast<T>(H + 2); chup = slast<T>(H + 3); lyup = slast<T>(H + 4); }
      } else {
        sld(L + RA_LN * 32, l_n); sld(L + RA_LX * 32, lxo); sld(L + RA_LY * 32, lyo);
        sld(L + RA_CE * 32, ce_); sld(L + RA_CH * 32, ch_);
        ldn = sfirst<T>(H + HA_LDN); chdn = sfirst<T>(H + HA_CHDN);
        if (I0 >= 1) { lup = slast<T>(H + HA_LUP); chup = slast<T>(H + HA_CHUP); lyup = slast<T>(H + HA_LYUP); }
      }
#pragma unroll
      for (int v = 0; v < V; ++v) {
        px_n[v] = ch_[v] * l_n[v]; py_n[v] = (w.rxy * ch_[v]) * l_n[v]; lm_n[v] = ce_[v] * l_n[v];
        lx_n[v] = ly_n[v] = ax_n[v] = ay_n[v] = T(0);
      }
      T px_dn = __shfl_down_sync(0xffffffffu, px_c[0], 1);
      T px_up = __shfl_up_sync(0xffffffffu, px_c[V - 1], 1);
      if (dnl) px_dn = chdn * ldn;
      if (upl) px_up = (I0 >= 1) ? chup * lup : T(0);
      T qy[V];
#pragma unroll
      for (int v = 0; v < V; ++v) {
        const T lt = lxo[v] + py_c[v] - py_n[v];
        lxn[v] = T(1) * lt;
        qx[v] = w.chxez * lt;
        const T pdn = (v < V - 1) ? px_c[v < V - 1 ? v + 1 : v] : px_dn;
        const T lt2 = lyo[v] + px_c[v] - pdn;
        lyn[v] = T(1) * lt2;
        qy[v] = w.chyez * lt2;
      }
      vst(LxB + k, lxn); vst(LyB + k, lyn);
      T qy_up = __shfl_up_sync(0xffffffffu, qy[V - 1], 1);
      if (upl) qy_up = (I0 >= 1) ? w.chyez * (lyup + px_up - px_c[0]) : T(0);
#pragma unroll
      for (int v = 0; v < V; ++v) {
        const T qym = (v > 0) ? qy[v > 0 ? v - 1 : 0] : qy_up;
        le[v] = lm_c[v] + qx_prev[v] - qx[v] + qym - qy[v];
        img[v] = ((dmask >> v) & 1u) ? l_c[v] : T(0);
      }
      if (I0 == 0) le[0] = T(0);  // the Ez = 0 row of a free top is not a state
      inject(J, le);
      vst(LB + k, le);
    } else if constexpr (!FAST) {
      // ---- general path
      vzero<T, V>(l_n); vzero<T, V>(lxo); vzero<T, V>(lyo); vzero<T, V>(ax_n); vzero<T, V>(ay_n);
      if (live) { sld(L + RA_LN * 32, l_n); sld(L + RA_LX * 32, lxo); sld(L + RA_LY * 32, lyo); }
      adj_pv_ring<T, V>(w, J + 1, live, rr, mE, mEint, L, l_n, px_n, py_n, lm_n, lx_n, ly_n, ax_n, ay_n);
      const bool hxs = !(J >= w.hxj0 && J <= w.hxj1);
      T hxa_[V], hxb_[V], hya_[V], hyb_[V];
      if (live && hxs) { sld(L + RA_HXA * 32, hxa_); sld(L + RA_HXB * 32, hxb_); }
      else {
#pragma unroll
        for (int v = 0; v < V; ++v) { hxa_[v] = T(1); hxb_[v] = w.chxez; }
      }
      vzero<T, V>(hya_); vzero<T, V>(hyb_);
      if (live && hyStrip) { sld(L + RA_HYA * 32, hya_); sld(L + RA_HYB * 32, hyb_); }
      T px_dn = __shfl_down_sync(0xffffffffu, px_c[0], 1);
      T px_up = __shfl_up_sync(0xffffffffu, px_c[V - 1], 1);
      if (dnl) {
        px_dn = T(0);
        if (live && Idn <= NX) {
          const int cls = adj_class(w, Idn, J);
          if (cls) px_dn = halo_px<T>(cls, sfirst<T>(H + HA_LDN), sfirst<T>(H + HA_SXDN), sfirst<T>(H + HA_CHDN),
                                      sfirst<T>(H + HA_BXDN));
        }
      }
      if (upl) {
        px_up = T(0);
        if (live && I0 >= 1) {
          const int cls = adj_class(w, Iup, J);
          if (cls) px_up = halo_px<T>(cls, slast<T>(H + HA_LUP), slast<T>(H + HA_SXUP), slast<T>(H + HA_CHUP),
                                      slast<T>(H + HA_BXUP));
        }
      }
      T qy[V], ltx[V], lty[V];
      const bool hxCol = J <= NY - 1;
#pragma unroll
      for (int v = 0; v < V; ++v) {
        const bool rx = hxCol && ((mHx >> v) & 1u);
        const T lt = lxo[v] + py_c[v] - py_n[v];
        lxn[v] = rx ? hxa_[v] * lt : T(0);
        qx[v] = rx ? hxb_[v] * lt : T(0);
        ltx[v] = rx ? lt : T(0);
        const bool ry = (mHy >> v) & 1u, hin = (mHyInt >> v) & 1u;
        const T ha = hin ? T(1) : hya_[v], hb = hin ? w.chyez : hyb_[v];
        const T pdn = (v < V - 1) ? px_c[v < V - 1 ? v + 1 : v] : px_dn;
        const T lt2 = lyo[v] + px_c[v] - pdn;
        lyn[v] = ry ? ha * lt2 : T(0);
        qy[v] = ry ? hb * lt2 : T(0);
        lty[v] = ry ? lt2 : T(0);
      }
      // adjoint band values (w_band.cuh): lx, ly at the band nodes, the
      // transposed strip H values
      if (a.band && live && I0 < w.bRB) {
        T* bs = a.band + size_t(zl) * w.bsz;
        const long oe = band_off_e(w, I0, J, 0);
        if (oe >= 0) { vst(bs + oe, lx_c); vst(bs + oe + (I0 >= w.bR0 ? w.bBsz : w.bLsz), ly_c); }
        const long ox = band_off_hx(w, I0, J);
        if (ox >= 0) vst(bs + ox, ltx);
        const long oy = band_off_hy(w, I0, J);
        if (oy >= 0) vst(bs + oy, lty);
      }
      if (live) { vst(LxB + k, lxn); vst(LyB + k, lyn); }
      T qy_up = __shfl_up_sync(0xffffffffu, qy[V - 1], 1);
      if (upl) {
        qy_up = T(0);
        if (live && I0 >= 1) {
          const T hb = upStrip ? slast<T>(H + HA_HYBUP) : w.chyez;
          qy_up = hb * (slast<T>(H + HA_LYUP) + px_up - px_c[0]);
        }
      }
      const bool colE = J >= 1 && J <= NY - 1;
      const bool colInt = J >= w.ej0 && J <= w.ej1;
      bool anyInt, anyBand;
      pvNeed(J, anyInt, anyBand);
      T sxn[V], syn[V];
#pragma unroll
      for (int v = 0; v < V; ++v) {
        const bool rE = colE && ((mE >> v) & 1u);
        const bool rI = rE && colInt && ((mEint >> v) & 1u);
        const bool rB = rE && !rI;
        const T qym = (v > 0) ? qy[v > 0 ? v - 1 : 0] : qy_up;
        const T lev = lm_c[v] + qx_prev[v] - qx[v] + qym - qy[v];
        le[v] = rE ? lev : T(0);
        sxn[v] = rB ? ax_c[v] * lx_c[v] : T(0);
        syn[v] = rB ? ay_c[v] * ly_c[v] : T(0);
        img[v] = (rI && ((dmask >> v) & 1u)) ? l_c[v] : T(0);
      }
      inject(J, le);
      if (live) {
        vst(LB + k, le);
        if (anyBand) { vst(SxB + k, sxn); vst(SyB + k, syn); }
      }
    }
    if (live && J >= w.dj0 && J < w.dj0 + w.n && drow(w, I0))
      vst(a.lout + size_t(zl) * a.hstride + dnode(w, I0, J), img);
#pragma unroll
    for (int v = 0; v < V; ++v) {
      qx_prev[v] = qx[v];
      l_c[v] = l_n[v]; px_c[v] = px_n[v]; py_c[v] = py_n[v]; lm_c[v] = lm_n[v]; lx_c[v] = lx_n[v];
      ly_c[v] = ly_n[v]; ax_c[v] = ax_n[v]; ay_c[v] = ay_n[v];
    }
  }
  cp_wait<0>();
}

// --------------------------------------------------------------------------
// Imaging over a window of adjoint steps.  Slot r of the l ring holds the
// adjoint field of step k = kA - r; the history slot of E^k is Ek0 - r*hsl
// (consecutive steps are consecutive history slots, hsl elements apart).
//   S1 += sum_r l_r (E^k - E^{k-1}),  S2 += sum_r l_r (E^k + E^{k-1})
// summed in T over the window, then added to the accumulators (compensated
// when kahan).  Only the V-row groups that meet the model rows are visited.
// Grid: x = row groups x model columns (grid-stride), y = shots of the group.
// --------------------------------------------------------------------------
template <class T>
__global__ void __launch_bounds__(256) k_image(const WDev<T> w, const T* lring, size_t lsl, const T* Ek0,
                                               size_t hsl, int cnt, size_t hstride, T* acc, size_t astride,
                                               int shot0, int kahan) {
  constexpr int V = VT<T>::V;
  const int zl = blockIdx.y;
  const int s = shot0 + zl;
  const int g0 = w.di0 / V, g1 = (w.di0 + w.m - 1) / V;  // row groups meeting the model
  const int ng = g1 - g0 + 1;
  const size_t total = size_t(ng) * w.n;
  const size_t dn = size_t(w.hld) * size_t(w.n);
  for (size_t t = threadIdx.x + size_t(blockIdx.x) * blockDim.x; t < total; t += size_t(blockDim.x) * gridDim.x) {
    const int gi = int(t % ng), b = int(t / ng);
    const size_t q = size_t(b) * w.hld + size_t((g0 + gi) * V - w.hr0);
    const T* L = lring + size_t(zl) * hstride + q;
    const T* E = Ek0 + size_t(zl) * hstride + q;
    T eh[V], s1[V], s2[V];
    vldw(E, eh);
    vzero<T, V>(s1); vzero<T, V>(s2);
#pragma unroll 4
    for (int r = 0; r < cnt; ++r) {
      T l[V], el[V];
      vldw(L + size_t(r) * lsl, l);
      vldw(E - size_t(r + 1) * hsl, el);
#pragma unroll
      for (int v = 0; v < V; ++v) {
        s1[v] += l[v] * (eh[v] - el[v]);
        s2[v] += l[v] * (eh[v] + el[v]);
        eh[v] = el[v];
      }
    }
    T* A = acc + size_t(s) * astride + q;
    T sE[V], cE[V], sS[V], cS[V];
    vldw(A, sE); vldw(A + 2 * dn, sS);
    if (kahan) {
      vldw(A + dn, cE); vldw(A + 3 * dn, cS);
#pragma unroll
      for (int v = 0; v < V; ++v) { kahan_add(&sE[v], &cE[v], s1[v]); kahan_add(&sS[v], &cS[v], s2[v]); }
      vst(A + dn, cE); vst(A + 3 * dn, cS);
    } else {
#pragma unroll
      for (int v = 0; v < V; ++v) { sE[v] += s1[v]; sS[v] += s2[v]; }
    }
    vst(A, sE); vst(A + 2 * dn, sS);
  }
}

// --------------------------------------------------------------------------
// Reference imaging (w_grad.m:86-87 with differentiate_cube.m:33-51) over a
// window of adjoint steps.  Slot r of the ring holds the adjoint Ez after the
// step of history index k = kA - r (1..nt); history slot k sits at
// H + (k - base) * hsl (slot k: E after forward step k-1).  Per step:
//   S1 -= (c0 u[k0] + c1 u[k1] + c2 u[k2]) l,  S2 -= u[k] l
// with differentiate_cube's stencil (one-sided at k = 1 and k = nt), summed in
// T over the window and then added to the accumulators (compensated when kahan).
// --------------------------------------------------------------------------
template <class T>
__global__ void __launch_bounds__(256) k_image_ref(const WDev<T> w, const T* lring, size_t lsl, const T* H,
                                                   long base, size_t hsl, int kA, int cnt, int nt, T idt,
                                                   size_t hstride, T* acc, size_t astride, int shot0, int kahan) {
  constexpr int V = VT<T>::V;
  const int zl = blockIdx.y;
  const int s = shot0 + zl;
  const int g0 = w.di0 / V, g1 = (w.di0 + w.m - 1) / V;
  const int ng = g1 - g0 + 1;
  const size_t total = size_t(ng) * w.n;
  const size_t dn = size_t(w.hld) * size_t(w.n);
  for (size_t t = threadIdx.x + size_t(blockIdx.x) * blockDim.x; t < total; t += size_t(blockDim.x) * gridDim.x) {
    const int gi = int(t % ng), b = int(t / ng);
    const size_t q = size_t(b) * w.hld + size_t((g0 + gi) * V - w.hr0);
    const T* L = lring + size_t(zl) * hstride + q;
    const T* U = H + size_t(zl) * hstride + q;
    T s1[V], s2[V];
    vzero<T, V>(s1); vzero<T, V>(s2);
    for (int r = 0; r < cnt; ++r) {
      const int k = kA - r;
      int k0, k1, k2;
      T c0, c1, c2;
      if (k == 1) { k0 = 1; k1 = 2; k2 = 3; c0 = T(-1.5) * idt; c1 = T(2.0) * idt; c2 = T(-0.5) * idt; }
      else if (k == nt) { k0 = nt - 2; k1 = nt - 1; k2 = nt; c0 = T(0.5) * idt; c1 = T(-2.0) * idt; c2 = T(1.5) * idt; }
      else { k0 = k - 1; k1 = k; k2 = k + 1; c0 = T(-0.5) * idt; c1 = T(0); c2 = T(0.5) * idt; }
      T l[V], u0[V], u1[V], u2[V], uk[V];
      vldw(L + size_t(r) * lsl, l);
      vldw(U + size_t(k0 - base) * hsl, u0);
      vldw(U + size_t(k1 - base) * hsl, u1);
      vldw(U + size_t(k2 - base) * hsl, u2);
      vldw(U + size_t(k - base) * hsl, uk);
#pragma unroll
      for (int v = 0; v < V; ++v) {
        const T du = c0 * u0[v] + c1 * u1[v] + c2 * u2[v];
        s1[v] -= du * l[v];
        s2[v] -= uk[v] * l[v];
      }
    }
    T* A = acc + size_t(s) * astride + q;
    T sE[V], cE[V], sS[V], cS[V];
    vldw(A, sE); vldw(A + 2 * dn, sS);
    if (kahan) {
      vldw(A + dn, cE); vldw(A + 3 * dn, cS);
#pragma unroll
      for (int v = 0; v < V; ++v) { kahan_add(&sE[v], &cE[v], s1[v]); kahan_add(&sS[v], &cS[v], s2[v]); }
      vst(A + dn, cE); vst(A + 3 * dn, cS);
    } else {
#pragma unroll
      for (int v = 0; v < V; ++v) { sE[v] += s1[v]; sS[v] += s2[v]; }
    }
    vst(A, sE); vst(A + 2 * dn, sS);
  }
}

}  // namespace gj

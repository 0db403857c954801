// 2.5D DC-resistivity kernels for sm_100a.
//
// One "system" is the operator Lk of one (source, ky) pair (dc_Lk.m:809):
//   Lk = -L + ky^2 diag(sigma), L the 5-point finite-volume operator with
//   harmonic-mean face conductances, a Neumann top and Robin sides/bottom.
// The off-diagonals are shared by all systems; the diagonal carries ky^2 sigma
// and the source- and ky-dependent Robin ghost terms.
//
// Unknowns are ordered with the shorter grid direction fastest, so the matrix
// is banded with half-bandwidth b = min(n, m).  The preconditioner is the
// LDL^T factor of that band (FP64 by default, FP32 on request; complete within
// the band), computed by one CTA per system, blocked, with the active band
// columns in shared memory.  CG runs in FP64 with that preconditioner.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace gj {

// Grid and ordering.  Node (l, h): l lateral in [0, n), h depth in [0, m)
// (the reference's (l, h) minus one); vectorised reference index l + h*n.
struct DcGrid {
  int n, m, N;      // nodes per direction, total
  int b;            // half-bandwidth = min(n, m)
  int depth_fast;   // 1: band index q = h + l*m (b = m); 0: q = l + h*n (b = n)
  double DX, DZ;    // DELTAS(:,:,1), DELTAS(:,:,2) as the reference computes them
  int nb;           // compact Robin entries per system: 2(m-2) + (n-2) + 4
  int wp, nq;       // factor layout: column stride (16-byte multiple), columns (N rounded up to 32)
};

__device__ __forceinline__ int dc_q(const DcGrid& G, int l, int h) {
  return G.depth_fast ? h + l * G.m : l + h * G.n;
}

// Face conductances of Lk (shared): ox(l,h) = Lk((l,h),(l+1,h)) = H*DZ/DX,
// oz(l,h) = Lk((l,h),(l,h+1)) = H*DX/DZ, H = 2 s_i s_j / (s_i + s_j)
// (dc_Lk.m:112-155 with -Lk), and dbase = -(sum of the node's offdiagonals).
__global__ void k_dc_faces(const DcGrid G, const double* sig, double* ox, double* oz, double* dbase) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= G.n * G.m) return;
  const int l = t % G.n, h = t / G.n;  // reference layout (lateral fastest)
  const double s = sig[t];
  double d = 0;
  if (l + 1 < G.n) {
    const double s2 = sig[t + 1];
    const double v = 2.0 * s * s2 / (s + s2) * (G.DZ / G.DX);
    ox[t] = v; d -= v;
  } else ox[t] = 0;
  if (l >= 1) {
    const double s2 = sig[t - 1];
    d -= 2.0 * s * s2 / (s + s2) * (G.DZ / G.DX);
  }
  if (h + 1 < G.m) {
    const double s2 = sig[t + G.n];
    const double v = 2.0 * s * s2 / (s + s2) * (G.DX / G.DZ);
    oz[t] = v; d -= v;
  } else oz[t] = 0;
  if (h >= 1) {
    const double s2 = sig[t - G.n];
    d -= 2.0 * s * s2 / (s + s2) * (G.DX / G.DZ);
  }
  dbase[t] = d;
}

// Robin ghost coefficient "face * alpha" of node (l, h) for one system, from
// the compact array [left h=1..m-2 | bottom l=1..n-2 | right h=1..m-2 |
// c11 c21 c12 c22] (dc_Lk.m:236-520, alphas :945-960).  MM5 = -sigma * this.
__device__ __forceinline__ double dc_robin_fa(const DcGrid& G, const double* al, int l, int h) {
  const int n = G.n, m = G.m;
  if (h >= 1 && h <= m - 2) {
    if (l == 0) return G.DZ * al[h - 1];
    if (l == n - 1) return G.DZ * al[(m - 2) + (n - 2) + (h - 1)];
    return 0.0;
  }
  if (h == m - 1) {
    const int c = 2 * (m - 2) + (n - 2);
    if (l >= 1 && l <= n - 2) return G.DX * al[(m - 2) + (l - 1)];
    if (l == 0) return G.DZ * al[c + 0] + G.DX * al[c + 1];
    if (l == n - 1) return G.DZ * al[c + 2] + G.DX * al[c + 3];
  }
  return 0.0;
}

// Diagonal of Lk at node (l, h) for one system.
__device__ __forceinline__ double dc_diag(const DcGrid& G, const double* dbase, const double* sig,
                                          const double* al, double ky2, int l, int h) {
  const int t = l + h * G.n;
  return dbase[t] - sig[t] * dc_robin_fa(G, al, l, h) + ky2 * sig[t];
}

// Band entry A(q, q-off) for off in {1, b}: the coupling to the previous node
// along the fast direction (off = 1) or the slow direction (off = b).
__device__ __forceinline__ double dc_sub(const DcGrid& G, const double* ox, const double* oz, int q, int off) {
  if (G.depth_fast) {
    const int l = q / G.m, h = q % G.m;
    if (off == 1) return h >= 1 ? oz[l + (h - 1) * G.n] : 0.0;
    return l >= 1 ? ox[(l - 1) + h * G.n] : 0.0;
  }
  const int l = q % G.n, h = q / G.n;
  if (off == 1) return l >= 1 ? ox[(l - 1) + h * G.n] : 0.0;
  return h >= 1 ? oz[l + (h - 1) * G.n] : 0.0;
}

__device__ __forceinline__ void dc_lh(const DcGrid& G, int q, int& l, int& h) {
  if (G.depth_fast) { l = q / G.m; h = q % G.m; }
  else { l = q % G.n; h = q / G.n; }
}

// Band LDL^T of every system (TF = double by default, float on request): one
// CTA of 256 threads per system, blocked right-looking with panels of DC_NB
// columns.  The window holds the M = b + DC_NB band columns of the current
// block as S[c mod M][r mod Mr] = A(r, c), r = c .. c+b, with Mr = b + 1
// rounded up to 4 so that four rows starting at a multiple of 4 are contiguous.
// Per block of pivots q .. q+DC_NB-1:
//   panel: thread t holds row q+t of the DC_NB panel columns in registers.
//     Warp 0 holds the pivot rows and runs the DC_NB pivots with shuffles
//     (d = A(c0, c0), l = A(r, c0) / d, rank-1 update of the later panel
//     columns), publishing d, 1 / d and the l of the pivot rows; after one
//     barrier every other row applies the same DC_NB steps from those values.
//     The l are written out; the rows below the panel also go to U[p][r'] = l
//     and Ud[p][r'] = l d (r' = row - q - DC_NB, zero outside the band).
//     Three barriers per block.
//   trailing: the b x b lower triangle of columns q+DC_NB .. takes the
//     rank-DC_NB update A(r, c) -= sum_p Ud[p][r'] U[p][c'], one register tile
//     of 4 rows x TC columns per thread and pass (host-built tile list,
//     column-major, so the lanes of a warp share the U operand and read
//     contiguous rows of one column); TC = 4 by default (351 tiles, two passes
//     at b = 101), TC = 8 covers b = 101 in one pass of 182 tiles but spills;
//   the DC_NB columns entering the window (original entries: diagonal,
//     A(c+1, c), A(c+b, c), fetched during the panel by the last DC_NB threads)
//     take the panel's slots.
// Pivots past N belong to an identity padding up to a multiple of DC_NB.
// Output per system: G.nq columns of G.wp entries, column q = [1 / d_q,
// l_{q+1,q}, ..., l_{q+b,q}, padding] (l = 0 past N); the columns N .. nq-1
// are zero.
constexpr int DC_NB = 8;
constexpr int DC_FACTOR_THREADS = 256;
static_assert(DC_FACTOR_THREADS == 32 * DC_NB, "one warp per entering column");

struct DcFactorShape {
  int M, Mr, BP, BPU, ntiles;
};

__host__ __device__ inline DcFactorShape dc_factor_shape(int b) {
  DcFactorShape f;
  f.M = b + DC_NB;
  f.Mr = (b + 1 + 3) / 4 * 4;
  f.BP = (b + 3) / 4 * 4;
  f.BPU = (f.BP + 7) / 8 * 8;  // row stride of U, Ud: whole 8-column tiles
  const int nt = f.BP / 4;
  f.ntiles = nt * (nt + 1) / 2;
  return f;
}

template <class TF>
__host__ __device__ inline size_t dc_factor_smem(int b) {
  const DcFactorShape f = dc_factor_shape(b);
  return (size_t(f.M) * f.Mr + 2 * size_t(DC_NB) * f.BPU + DC_NB * DC_NB + 5 * DC_NB) * sizeof(TF) +
         size_t(f.ntiles) * sizeof(unsigned);
}

__device__ __forceinline__ void dc_ld4(const double* p, double v[4]) {
  const double2 a = *reinterpret_cast<const double2*>(p), c = *reinterpret_cast<const double2*>(p + 2);
  v[0] = a.x; v[1] = a.y; v[2] = c.x; v[3] = c.y;
}
__device__ __forceinline__ void dc_ld4(const float* p, float v[4]) {
  const float4 a = *reinterpret_cast<const float4*>(p);
  v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w;
}
__device__ __forceinline__ void dc_st4(double* p, const double v[4]) {
  *reinterpret_cast<double2*>(p) = make_double2(v[0], v[1]);
  *reinterpret_cast<double2*>(p + 2) = make_double2(v[2], v[3]);
}
__device__ __forceinline__ void dc_st4(float* p, const float v[4]) {
  *reinterpret_cast<float4*>(p) = make_float4(v[0], v[1], v[2], v[3]);
}
// Four entries at p in the order (2h, 2h+1, 2-2h, 3-2h), h = 0 or 1: two
// 16-byte halves, the one at p + 2h first (FP64); FP32 entries are one
// 16-byte vector and h = 0.
__device__ __forceinline__ void dc_ld4h(const double* p, int h, double v[4]) {
  const double2 a = *reinterpret_cast<const double2*>(p + 2 * h);
  const double2 c = *reinterpret_cast<const double2*>(p + 2 - 2 * h);
  v[0] = a.x; v[1] = a.y; v[2] = c.x; v[3] = c.y;
}
__device__ __forceinline__ void dc_ld4h(const float* p, int, float v[4]) { dc_ld4(p, v); }
__device__ __forceinline__ void dc_st4h(double* p, int h, const double v[4]) {
  *reinterpret_cast<double2*>(p + 2 * h) = make_double2(v[0], v[1]);
  *reinterpret_cast<double2*>(p + 2 - 2 * h) = make_double2(v[2], v[3]);
}
__device__ __forceinline__ void dc_st4h(float* p, int, const float v[4]) { dc_st4(p, v); }
// 16 bytes of entries to a 16-byte aligned address
__device__ __forceinline__ void dc_st16(double* p, const double (&v)[2]) {
  *reinterpret_cast<double2*>(p) = make_double2(v[0], v[1]);
}
__device__ __forceinline__ void dc_st16(float* p, const float (&v)[4]) {
  *reinterpret_cast<float4*>(p) = make_float4(v[0], v[1], v[2], v[3]);
}

template <class TF, int TC>
__global__ void __launch_bounds__(DC_FACTOR_THREADS, 2) k_dc_factor(const DcGrid G, const double* ox, const double* oz,
                                                                 const double* dbase, const double* sig,
                                                                 const double* alpha, const double* ky2,
                                                                 const unsigned* tiles, int ntiles, int sys0, TF* fac,
                                                                 int* status) {
  extern __shared__ __align__(16) unsigned char shraw[];
  const int N = G.N, b = G.b, wp = G.wp;
  const DcFactorShape fs = dc_factor_shape(b);
  static_assert(TC == 4 || TC == 8, "trailing tiles of 4 rows x 4 or 8 columns");
  const int M = fs.M, Mr = fs.Mr, BP = fs.BP, BPU = fs.BPU;
  TF* S = reinterpret_cast<TF*>(shraw);
  TF* U = S + size_t(M) * Mr;  // [DC_NB][BPU]
  TF* Ud = U + DC_NB * BPU;    // [DC_NB][BPU]
  TF* pd = Ud + DC_NB * BPU;   // pivots d of the block
  TF* pdinv = pd + DC_NB;      // 1 / d
  TF* pl = pdinv + DC_NB;      // [DC_NB][DC_NB]: l of the panel's own rows, pl[p][c] = L(q+c, q+p)
  TF* stg = pl + DC_NB * DC_NB;  // [3][DC_NB]: entering columns' diagonal, A(c+1, c), A(c+b, c)
  unsigned* tab = reinterpret_cast<unsigned*>(stg + 3 * DC_NB);
  const int sys = blockIdx.x, tid = threadIdx.x, nth = DC_FACTOR_THREADS;
  const double* al = alpha + size_t(sys0 + sys) * G.nb;
  const double k2 = ky2[sys0 + sys];
  TF* F = fac + size_t(sys) * size_t(G.nq) * wp;
  // original band entries of column c (identity past N)
  auto entering = [&](int c, TF& dg, TF& s1, TF& s2) {
    dg = TF(1); s1 = TF(0); s2 = TF(0);
    if (c < N) {
      int l, h;
      dc_lh(G, c, l, h);
      dg = TF(dc_diag(G, dbase, sig, al, k2, l, h));
      if (c + 1 < N) s1 = TF(dc_sub(G, ox, oz, c + 1, 1));
      if (c + b < N) s2 = TF(dc_sub(G, ox, oz, c + b, b));
    }
  };
  auto column_value = [&](int c, int k, TF dg, TF s1, TF s2) {  // row slot k of column c
    const int r0 = c % Mr;
    int r1 = r0 + 1, rb = r0 + b;
    if (r1 >= Mr) r1 -= Mr;
    if (rb >= Mr) rb -= Mr;
    return k == r0 ? dg : (k == r1 ? s1 : (k == rb ? s2 : TF(0)));
  };
  // ntiles (the host list's length, at most fs.ntiles, the 4 x 4 count that
  // sizes tab) tiles of 4 rows x TC columns
  for (int e = tid; e < ntiles; e += nth) tab[e] = tiles[e];
  for (int e = tid; e < M * Mr; e += nth) {  // columns 0 .. M-1
    const int c = e / Mr, k = e % Mr;
    TF dg, s1, s2;
    entering(c, dg, s1, s2);
    S[e] = column_value(c, k, dg, s1, s2);
  }
  const int Nn = (N + DC_NB - 1) / DC_NB * DC_NB;
  int sq = 0, rq = 0;  // q mod M, q mod Mr
  __syncthreads();
  for (int q = 0; q < Nn; q += DC_NB) {
    if (tid >= nth - DC_NB) {  // entering columns of this block
      const int t = tid - (nth - DC_NB);
      TF dg, s1, s2;
      entering(q + M + t, dg, s1, s2);
      stg[t] = dg; stg[DC_NB + t] = s1; stg[2 * DC_NB + t] = s2;
    }
    // ---- panel: thread t owns row q+t of the panel columns (t < DC_NB + BP) in registers
    const bool row = tid < DC_NB + BP;
    TF a[DC_NB];
    {
      const int pos = (rq + tid) % Mr;
#pragma unroll
      for (int c = 0; c < DC_NB; ++c) {
        int sc = sq + c;
        if (sc >= M) sc -= M;
        a[c] = (row && tid >= c && tid - c <= b) ? S[sc * Mr + pos] : TF(0);
      }
    }
    if (tid < 32) {  // warp 0 holds the pivot rows (lanes 0 .. DC_NB-1): the pivots by shuffles
#pragma unroll
      for (int p = 0; p < DC_NB; ++p) {
        const TF dp = __shfl_sync(0xffffffffu, a[p], p);
        const TF dinv = TF(1) / dp;
        const TF l = tid > p ? a[p] * dinv : TF(0);
        const TF ld = l * dp;
        if (tid == 0) { pd[p] = dp; pdinv[p] = dinv; }
#pragma unroll
        for (int c = p + 1; c < DC_NB; ++c) {
          const TF lc_ = __shfl_sync(0xffffffffu, l, c);
          if (tid == 0) pl[p * DC_NB + c] = lc_;
          a[c] -= ld * lc_;
        }
        a[p] = l;
      }
    }
    __syncthreads();  // pivots published
    if (tid >= 32 && row) {
#pragma unroll
      for (int p = 0; p < DC_NB; ++p) {
        const TF l = a[p] * pdinv[p];
        const TF ld = l * pd[p];
#pragma unroll
        for (int c = p + 1; c < DC_NB; ++c) a[c] -= ld * pl[p * DC_NB + c];
        a[p] = l;
      }
    }
    if (row && tid >= DC_NB) {  // a[p] = l of row q+t for pivot q+p, rows below the panel
#pragma unroll
      for (int p = 0; p < DC_NB; ++p) {
        U[p * BPU + tid - DC_NB] = a[p];
        Ud[p * BPU + tid - DC_NB] = a[p] * pd[p];
      }
    }
    if (tid < DC_NB && q + tid < N) {
      const TF d = pd[tid];
      if (!(d != TF(0)) || !isfinite(d)) atomicExch(status + sys0 + sys, 1);
    }
    __syncthreads();
    // ---- factor columns q .. q+DC_NB-1: warp p writes column q+p,
    // [1 / d, l_{q+p+1,q+p} .. l_{q+p+b,q+p}] (0 for rows at or past N and in
    // the padding past b), 16 bytes per lane, from the published pivots, the
    // panel rows' l (pl) and the rows below the panel (U); the stores overlap
    // the trailing update.  wp is a multiple of the entries per store, so the
    // last store of a column ends inside it.
    {
      const int p = tid >> 5, lane = tid & 31;
      const int c0 = q + p;
      if (c0 < N) {
        TF* Fc = F + size_t(c0) * wp;
        constexpr int EV = 16 / int(sizeof(TF));
        for (int v = lane; v * EV <= b; v += 32) {
          TF e[EV];
#pragma unroll
          for (int u = 0; u < EV; ++u) {
            const int i = v * EV + u;
            e[u] = i == 0 ? pdinv[p]
                 : (i > b || c0 + i >= N) ? TF(0)
                 : (i < DC_NB - p ? pl[p * DC_NB + p + i] : U[p * BPU + i + p - DC_NB]);
          }
          dc_st16(Fc + v * EV, e);
        }
      }
    }
    // ---- trailing rank-DC_NB update.  A lane's 4 rows are 32 bytes (FP64),
    // and the lanes of a warp hold consecutive row blocks of one column, so a
    // 16-byte load of the same half by every lane spans 1 KB with every
    // second 16 bytes unused (two shared wavefronts per 128 bytes).  Lanes
    // with bit 2 set take their second half first (rows 2, 3, 0, 1): each 8
    // lanes then cover all 32 banks once.  The lane keeps that row order for
    // its accumulators, the Ud rows and the stores, so nothing moves between
    // lanes.  FP32 rows are 16 bytes, contiguous across lanes already.
    const int hs = sizeof(TF) == 8 ? (tid >> 2) & 1 : 0;  // row pair first in this lane's order
    int sqn = sq + DC_NB, rqn = (rq + DC_NB) % Mr;
    if (sqn >= M) sqn -= M;
    for (int e = tid; e < ntiles; e += nth) {
      const unsigned tv = tab[e];
      const int rt = int(tv & 0xffffu), ct = int(tv >> 16);
      int rbase = rqn + 4 * rt;
      if (rbase >= Mr) rbase -= Mr;
      TF acc[TC][4];
      int sc[TC];
#pragma unroll
      for (int kc = 0; kc < TC; ++kc) {
        int s_ = sqn + TC * ct + kc;  // TC * ct + kc < BPU <= M
        if (s_ >= M) s_ -= M;
        sc[kc] = s_;
        dc_ld4h(S + s_ * Mr + rbase, hs, acc[kc]);
      }
#pragma unroll
      for (int p = 0; p < DC_NB; ++p) {
        TF av[4], bv[TC];
        dc_ld4h(Ud + p * BPU + 4 * rt, hs, av);
#pragma unroll
        for (int h = 0; h < TC / 4; ++h) dc_ld4(U + p * BPU + TC * ct + 4 * h, bv + 4 * h);
#pragma unroll
        for (int kc = 0; kc < TC; ++kc)
#pragma unroll
          for (int kr = 0; kr < 4; ++kr) acc[kc][kr] -= av[kr] * bv[kc];
      }
      if (4 * rt > TC * ct + TC - 1 && 4 * rt + 3 < b) {  // strictly below the diagonal, inside the band
#pragma unroll
        for (int kc = 0; kc < TC; ++kc) dc_st4h(S + sc[kc] * Mr + rbase, hs, acc[kc]);
      } else {
#pragma unroll
        for (int kc = 0; kc < TC; ++kc)
#pragma unroll
          for (int kr = 0; kr < 4; ++kr) {
            const int rr = kr ^ (2 * hs);  // the row of slot kr
            const int rp = 4 * rt + rr, cp = TC * ct + kc;
            if (rp >= cp && rp < b) S[sc[kc] * Mr + rbase + rr] = acc[kc][kr];
          }
      }
    }
    // ---- entering columns q+M .. q+M+DC_NB-1 into the panel's slots: warp t
    // zeroes slot column t with 16-byte stores, then writes its three entries
    // (diagonal, A(c+1, c), A(c+b, c))
    {
      const int t = tid >> 5, lane = tid & 31;
      int s_ = sq + t;
      if (s_ >= M) s_ -= M;
      TF* col = S + s_ * Mr;
      const int nvec = Mr * int(sizeof(TF)) / 16;
      for (int v = lane; v < nvec; v += 32) reinterpret_cast<uint4*>(col)[v] = make_uint4(0u, 0u, 0u, 0u);
      __syncwarp();
      if (lane < 3) {
        const int c = q + M + t, r0 = c % Mr;
        int k = r0 + (lane == 0 ? 0 : (lane == 1 ? 1 : b));
        if (k >= Mr) k -= Mr;
        // b = 1 makes lanes 1 and 2 write the same entry, the same value
        col[k] = stg[lane * DC_NB + t];
      }
    }
    sq = sqn;
    rq = rqn;
    __syncthreads();
  }
  for (size_t e = size_t(N) * wp + tid; e < size_t(G.nq) * wp; e += nth) F[e] = TF(0);
}

// z = (L D L^T)^{-1} r and rz = r.z for every system; one warp (one CTA) per
// system.  r, z are FP64 vectors in the reference layout [sys][l + h*n].
// Factor columns stream through a shared-memory ring of NST chunks of CH
// columns (16-byte cp.async, NST - 1 chunks ahead); a ring of 4 x 8 columns
// (26.6 KB for b = 101 in FP64) lets 8 systems share an SM, where 4 x 16
// columns allowed 4.  The substitution window
// lives in registers: within the 32-step sub-block starting at band index qs,
// slot u of lane t holds position qs + 32u + t (mod 32R), so slot 0 holds the
// sub-block's own positions; the slots rotate by one between sub-blocks and
// every register index is a compile-time constant.
//   forward  L y = r, column form: y_q = w_q, then w_{q+i} -= l_{q+i,q} y_q for
//            i = 1..b, and z_q = y_q / d_q (the factor stores 1 / d_q);
//   backward L^T x = z, row form: x_q = z_q - sum_i l_{q+i,q} x_{q+i}.  Lanes
//            sum the terms i >= DC_NEAR over their slots and the warp reduces
//            them; the DC_NEAR - 1 nearest terms come from registers, so the
//            reduction of step q waits only for x_{q+DC_NEAR}, which enters the
//            window DC_NEAR steps after it is computed.
constexpr int DC_NEAR = 4;

template <class TF>
__host__ __device__ inline size_t dc_precond_smem(int wp, int ch, int nst) {
  return size_t(nst) * ch * wp * sizeof(TF);
}

__device__ __forceinline__ unsigned dc_smem_addr(const void* p) {
  return static_cast<unsigned>(__cvta_generic_to_shared(p));
}

// Copies factor chunk c (columns c*CH ..) into ring slot c mod NST as one
// commit group (an empty group when c is outside [0, nch)).
template <class TF, int CH, int NST>
__device__ __forceinline__ void dc_chunk_async(TF* ring, const TF* F, int c, int nch, int wp, int lane) {
  if (c >= 0 && c < nch) {
    const int pieces = CH * wp * int(sizeof(TF)) / 16;
    const char* src = reinterpret_cast<const char*>(F + size_t(c) * CH * wp);
    const unsigned dst = dc_smem_addr(ring + (c & (NST - 1)) * CH * wp);
    for (int p = lane; p < pieces; p += 32)
      asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(dst + 16u * unsigned(p)),
                   "l"(src + 16 * size_t(p))
                   : "memory");
  }
  asm volatile("cp.async.commit_group;\n" ::: "memory");
}

template <class TF, int R, int CH, int NST>
__global__ void __launch_bounds__(32) k_dc_precond(const DcGrid G, const TF* fac, const double* r, double* z,
                                                   double* rz, int nsys, const int* done) {
  extern __shared__ __align__(16) unsigned char shpraw[];
  TF* ring = reinterpret_cast<TF*>(shpraw);
  constexpr int WIN = 32 * R;
  const int sys = blockIdx.x, lane = threadIdx.x & 31;
  if (sys >= nsys || (done && done[sys])) return;
  const int N = G.N, b = G.b, wp = G.wp, nq = G.nq;
  static_assert((CH == 4 || CH == 8 || CH == 16) && (NST == 4 || NST == 8), "power-of-two ring shapes");
  const int nch = nq / CH;
  const TF* F = fac + size_t(sys) * nq * wp;
  const double* Rv = r + size_t(sys) * N;
  double* Z = z + size_t(sys) * N;
  auto ref = [&](int q) { int l, h; dc_lh(G, q, l, h); return l + h * G.n; };
  auto rld = [&](const double* v, int a) { return (a >= 0 && a < N) ? v[ref(a)] : 0.0; };
  auto chunk_wait = [&](int c_issue) {
    __syncwarp();  // every lane is done with the slot being refilled
    dc_chunk_async<TF, CH, NST>(ring, F, c_issue, nch, wp, lane);
    asm volatile("cp.async.wait_group %0;\n" ::"n"(NST - 1) : "memory");
    __syncwarp();
  };
  auto column = [&](int q) { return ring + (((q / CH) & (NST - 1)) * CH + (q & (CH - 1))) * wp; };
  // ---- forward sweep
  TF w[R];
#pragma unroll
  for (int u = 0; u < R; ++u) w[u] = TF(rld(Rv, 32 * u + lane));
  double rn = rld(Rv, WIN + lane);  // refills of the sub-block's slot 0
  for (int c = 0; c < NST - 1; ++c) dc_chunk_async<TF, CH, NST>(ring, F, c, nch, wp, lane);
  for (int qs = 0; qs < nq; qs += 32) {
    const double rnn = rld(Rv, qs + 32 + WIN + lane);
    TF zv = TF(0);
#pragma unroll
    for (int j = 0; j < 32; ++j) {
      if ((j & (CH - 1)) == 0) chunk_wait((qs + j) / CH + NST - 1);
      const TF* col = column(qs + j);
      const TF y = __shfl_sync(0xffffffffu, w[0], j);
      if (lane == j) { zv = y * col[0]; w[0] = TF(rn); }
#pragma unroll
      for (int u = 0; u < R; ++u) {
        const int i = (32 * u + lane - j + WIN) & (WIN - 1);
        if (i >= 1 && i <= b) w[u] -= col[i] * y;
      }
    }
    if (qs + lane < N) Z[ref(qs + lane)] = double(zv);
    const TF w0 = w[0];
#pragma unroll
    for (int u = 0; u + 1 < R; ++u) w[u] = w[u + 1];
    w[R - 1] = w0;
    rn = rnn;
  }
  asm volatile("cp.async.wait_group 0;\n" ::: "memory");
  __syncwarp();
  // ---- backward sweep
#pragma unroll
  for (int u = 0; u < R; ++u) w[u] = TF(0);
  TF nx[DC_NEAR];  // nx[k] = x_{q+1+k}
#pragma unroll
  for (int k = 0; k < DC_NEAR; ++k) nx[k] = TF(0);
  for (int c = 0; c < NST - 1; ++c) dc_chunk_async<TF, CH, NST>(ring, F, nch - 1 - c, nch, wp, lane);
  double zc = rld(Z, nq - 32 + lane), rc = rld(Rv, nq - 32 + lane);
  double acc = 0.0;
  for (int qs = nq - 32; qs >= 0; qs -= 32) {
    const double zn = rld(Z, qs - 32 + lane), rnx = rld(Rv, qs - 32 + lane);
    TF xv = TF(0);
#pragma unroll
    for (int j = 31; j >= 0; --j) {
      if ((j & (CH - 1)) == CH - 1) chunk_wait((qs + j) / CH - (NST - 1));
      const TF* col = column(qs + j);
      if (j + DC_NEAR < 32) { if (lane == j + DC_NEAR) w[0] = nx[DC_NEAR - 1]; }
      else if (lane == j + DC_NEAR - 32) w[1] = nx[DC_NEAR - 1];
      TF part = TF(0);
#pragma unroll
      for (int u = 0; u < R; ++u) {
        const int i = (32 * u + lane - j + WIN) & (WIN - 1);
        if (i >= DC_NEAR && i <= b) part += col[i] * w[u];
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
      TF x = TF(__shfl_sync(0xffffffffu, zc, j)) - part;
#pragma unroll
      for (int k = DC_NEAR - 2; k >= 0; --k) x -= col[k + 1] * nx[k];
#pragma unroll
      for (int k = DC_NEAR - 1; k > 0; --k) nx[k] = nx[k - 1];
      nx[0] = x;
      if (lane == j) xv = x;
    }
    if (qs + lane < N) {
      Z[ref(qs + lane)] = double(xv);
      acc += rc * double(xv);
    }
    const TF wl = w[R - 1];
#pragma unroll
    for (int u = R - 1; u > 0; --u) w[u] = w[u - 1];
    w[0] = wl;
    zc = zn;
    rc = rnx;
  }
  asm volatile("cp.async.wait_group 0;\n" ::: "memory");
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if (lane == 0) rz[sys] = acc;
}

// --------------------------------------------------------------------------
// FP32 incomplete-Cholesky preconditioner IC(0) in red-black ordering (the
// option beside the band factor).  With the nodes coloured by (l + h) & 1 the
// 5-point operator is A = [Dr B; B' Db] (no red-red or black-black
// couplings), and IC(0), which keeps only A's own pattern, is
//   L = [Dr^1/2, 0; B' Dr^-1/2, Sb^1/2],  Sb = diag(Db - B' Dr^-1 B),
// so M^-1 r takes two sweeps:
//   black: z_b = (r_b - sum_red A(b, r) r_r / D_r) / Sb_b
//   red:   z_r = (r_r - sum_black A(r, b) z_b) / D_r.
// dinv[sys][t] holds 1 / D_r at the red nodes and 1 / Sb at the black ones,
// in FP32; the sweeps run in FP32 and return z in FP64 for the FP64 flexible
// CG, whose iteration refines the FP32-preconditioned solve to the FP64
// tolerance.
// --------------------------------------------------------------------------
__global__ void k_dc_ic0_setup(const DcGrid G, const double* ox, const double* oz, const double* dbase,
                               const double* sig, const double* alpha, const double* ky2, int sys0, int nsys,
                               float* dinv, int* status) {
  const int sys = blockIdx.y;
  if (sys >= nsys) return;
  const double* al = alpha + size_t(sys0 + sys) * G.nb;
  const double k2 = ky2[sys0 + sys];
  float* Dv = dinv + size_t(sys) * G.N;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < G.N; t += blockDim.x * gridDim.x) {
    const int l = t % G.n, h = t / G.n;
    double d = dc_diag(G, dbase, sig, al, k2, l, h);
    if ((l + h) & 1) {  // black: Schur diagonal over the red neighbours
      if (l + 1 < G.n) d -= ox[t] * ox[t] / dc_diag(G, dbase, sig, al, k2, l + 1, h);
      if (l >= 1) d -= ox[t - 1] * ox[t - 1] / dc_diag(G, dbase, sig, al, k2, l - 1, h);
      if (h + 1 < G.m) d -= oz[t] * oz[t] / dc_diag(G, dbase, sig, al, k2, l, h + 1);
      if (h >= 1) d -= oz[t - G.n] * oz[t - G.n] / dc_diag(G, dbase, sig, al, k2, l, h - 1);
    }
    if (!(d > 0.0) || !isfinite(d)) atomicExch(status + sys0 + sys, 1);
    Dv[t] = float(1.0 / d);
  }
}

// Black sweep: z_b, and r.z over the black nodes into rz[sys].
__global__ void k_dc_ic0_black(const DcGrid G, const float* dinv, const double* ox, const double* oz,
                               const double* r, double* z, double* rz, int nsys, const int* done) {
  const int sys = blockIdx.y;
  if (sys >= nsys || (done && done[sys])) return;
  const size_t o = size_t(sys) * G.N;
  const float* Dv = dinv + o;
  const double* R = r + o;
  double part = 0;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < G.N; t += blockDim.x * gridDim.x) {
    const int l = t % G.n, h = t / G.n;
    if (!((l + h) & 1)) continue;
    float v = float(R[t]);
    if (l + 1 < G.n) v -= float(ox[t]) * (float(R[t + 1]) * Dv[t + 1]);
    if (l >= 1) v -= float(ox[t - 1]) * (float(R[t - 1]) * Dv[t - 1]);
    if (h + 1 < G.m) v -= float(oz[t]) * (float(R[t + G.n]) * Dv[t + G.n]);
    if (h >= 1) v -= float(oz[t - G.n]) * (float(R[t - G.n]) * Dv[t - G.n]);
    const double zb = double(v * Dv[t]);
    z[o + t] = zb;
    part += R[t] * zb;
  }
  for (int off = 16; off > 0; off >>= 1) part += __shfl_down_sync(0xffffffffu, part, off);
  if ((threadIdx.x & 31) == 0) atomicAdd(rz + sys, part);
}

// Red sweep after the black one: z_r, and r.z over the red nodes into rz[sys].
__global__ void k_dc_ic0_red(const DcGrid G, const float* dinv, const double* ox, const double* oz,
                             const double* r, double* z, double* rz, int nsys, const int* done) {
  const int sys = blockIdx.y;
  if (sys >= nsys || (done && done[sys])) return;
  const size_t o = size_t(sys) * G.N;
  const float* Dv = dinv + o;
  const double* R = r + o;
  const double* Z = z + o;
  double part = 0;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < G.N; t += blockDim.x * gridDim.x) {
    const int l = t % G.n, h = t / G.n;
    if ((l + h) & 1) continue;
    float v = float(R[t]);
    if (l + 1 < G.n) v -= float(ox[t]) * float(Z[t + 1]);
    if (l >= 1) v -= float(ox[t - 1]) * float(Z[t - 1]);
    if (h + 1 < G.m) v -= float(oz[t]) * float(Z[t + G.n]);
    if (h >= 1) v -= float(oz[t - G.n]) * float(Z[t - G.n]);
    const double zr = double(v * Dv[t]);
    z[o + t] = zr;
    part += R[t] * zr;
  }
  for (int off = 16; off > 0; off >>= 1) part += __shfl_down_sync(0xffffffffu, part, off);
  if ((threadIdx.x & 31) == 0) atomicAdd(rz + sys, part);
}

// y = Lk x for every system (FP64), optional dot x.y into dot[sys].
__global__ void k_dc_apply(const DcGrid G, const double* ox, const double* oz, const double* dbase,
                           const double* sig, const double* alpha, const double* ky2, int sys0,
                           const double* x, double* y, double* dot, int nsys, const int* done) {
  const int sys = blockIdx.y;
  if (sys >= nsys || (done && done[sys])) return;
  const double* al = alpha + size_t(sys0 + sys) * G.nb;
  const double k2 = ky2[sys0 + sys];
  const double* X = x + size_t(sys) * G.N;
  double* Y = y + size_t(sys) * G.N;
  double part = 0;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < G.N; t += blockDim.x * gridDim.x) {
    const int l = t % G.n, h = t / G.n;
    double v = dc_diag(G, dbase, sig, al, k2, l, h) * X[t];
    if (l + 1 < G.n) v += ox[t] * X[t + 1];
    if (l >= 1) v += ox[t - 1] * X[t - 1];
    if (h + 1 < G.m) v += oz[t] * X[t + G.n];
    if (h >= 1) v += oz[t - G.n] * X[t - G.n];
    Y[t] = v;
    part += v * X[t];
  }
  if (dot) {
    for (int o = 16; o > 0; o >>= 1) part += __shfl_down_sync(0xffffffffu, part, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(dot + sys, part);
  }
}

// CG update: alpha = rz/pAp; x += alpha p; r -= alpha Ap; rr = r.r and
// rzo = r_new . z_old (for the flexible Polak-Ribiere beta, since the FP32
// preconditioner is only symmetric to rounding).
__global__ void k_dc_cg_xr(int N, const double* rz, const double* pap, double* x, double* r, const double* p,
                           const double* ap, const double* z, double* rr, double* rzo, int nsys, const int* done) {
  const int sys = blockIdx.y;
  if (sys >= nsys || (done && done[sys])) return;
  const double den = pap[sys];
  const double a = (den != 0.0) ? rz[sys] / den : 0.0;
  const size_t o = size_t(sys) * N;
  double part = 0, part2 = 0;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < N; t += blockDim.x * gridDim.x) {
    x[o + t] += a * p[o + t];
    const double v = r[o + t] - a * ap[o + t];
    r[o + t] = v;
    part += v * v;
    part2 += v * z[o + t];
  }
  for (int off = 16; off > 0; off >>= 1) {
    part += __shfl_down_sync(0xffffffffu, part, off);
    part2 += __shfl_down_sync(0xffffffffu, part2, off);
  }
  if ((threadIdx.x & 31) == 0) { atomicAdd(rr + sys, part); atomicAdd(rzo + sys, part2); }
}

// p = z + beta p, beta = (r.z_new - r.z_old) / rz_old (flexible CG); p = z when first.
__global__ void k_dc_cg_p(int N, const double* rz_new, const double* rz_old, const double* rzo, const double* z,
                          double* p, int first, int nsys, const int* done) {
  const int sys = blockIdx.y;
  if (sys >= nsys || (done && done[sys])) return;
  double beta = 0.0;
  if (!first && rz_old[sys] != 0.0) beta = (rz_new[sys] - (rzo ? rzo[sys] : 0.0)) / rz_old[sys];
  const size_t o = size_t(sys) * N;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < N; t += blockDim.x * gridDim.x)
    p[o + t] = z[o + t] + beta * p[o + t];
}

// r = b - y (FP64), rr = r.r, bb = b.b
__global__ void k_dc_residual(int N, const double* bvec, const double* y, double* r, double* rr, double* bb,
                              int nsys) {
  const int sys = blockIdx.y;
  if (sys >= nsys) return;
  const size_t o = size_t(sys) * N;
  double p1 = 0, p2 = 0;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < N; t += blockDim.x * gridDim.x) {
    const double v = bvec[o + t] - y[o + t];
    r[o + t] = v;
    p1 += v * v;
    p2 += bvec[o + t] * bvec[o + t];
  }
  for (int off = 16; off > 0; off >>= 1) {
    p1 += __shfl_down_sync(0xffffffffu, p1, off);
    p2 += __shfl_down_sync(0xffffffffu, p2, off);
  }
  if ((threadIdx.x & 31) == 0) { atomicAdd(rr + sys, p1); if (bb) atomicAdd(bb + sys, p2); }
}

// Sensitivity of one system (dc_Sk.m with dc_gradient2_5d.m:37-38):
// g += (2/pi) w [ sum_faces ratio 2 (s_j/(s_i+s_j))^2 (U_i-U_j)(a_i-a_j)
//                 + face*alpha U_i a_i - ky^2 U_i a_i ].
__global__ void k_dc_sens(const DcGrid G, const double* sig, const double* alpha, const double* ky2,
                          const double* wts, int sys0, int nky, const double* U, const double* A, double* g,
                          int nsys) {
  const int sys = blockIdx.y;
  if (sys >= nsys) return;
  const int gs = sys0 + sys;
  const double* al = alpha + size_t(gs) * G.nb;
  const double k2 = ky2[gs];
  const double wq = (2.0 / 3.14159265358979323846) * wts[gs];
  const double* Us = U + size_t(sys) * G.N;
  const double* As = A + size_t(sys) * G.N;
  double* gg = g + size_t(gs / nky) * G.N;  // one gradient per source
  const double rx = G.DZ / G.DX, rzz = G.DX / G.DZ;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < G.N; t += blockDim.x * gridDim.x) {
    const int l = t % G.n, h = t / G.n;
    const double si = sig[t], ui = Us[t], ai = As[t];
    double v = 0;
    if (l + 1 < G.n) { const double sj = sig[t + 1]; const double q = sj / (si + sj);
      v += rx * 2 * q * q * (ui - Us[t + 1]) * (ai - As[t + 1]); }
    if (l >= 1) { const double sj = sig[t - 1]; const double q = sj / (si + sj);
      v += rx * 2 * q * q * (ui - Us[t - 1]) * (ai - As[t - 1]); }
    if (h + 1 < G.m) { const double sj = sig[t + G.n]; const double q = sj / (si + sj);
      v += rzz * 2 * q * q * (ui - Us[t + G.n]) * (ai - As[t + G.n]); }
    if (h >= 1) { const double sj = sig[t - G.n]; const double q = sj / (si + sj);
      v += rzz * 2 * q * q * (ui - Us[t - G.n]) * (ai - As[t - G.n]); }
    v += dc_robin_fa(G, al, l, h) * ui * ai;
    v -= k2 * ui * ai;
    atomicAdd(gg + t, wq * v);
  }
}

}  // namespace gj

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
// the band), computed by one CTA per system with a rolling window of b+1 band
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

// Band LDL^T of every system (TF = double by default, float on request): one CTA per system.  Output per system:
// N columns of (b+1) floats: [d_q, l_{q+1,q}, ..., l_{q+b,q}].
// Shared memory: (b+1)^2 floats (rolling window, circular in both indices)
// + (b+1) floats (current column).  The b(b+1)/2 updates of each step are
// split into equal contiguous runs over all threads (row-major packed order),
// and the next band row's entries are fetched from global memory while the
// update runs.
// Band LDL^T of every system (TF = double by default, float on request): one
// CTA per system.  The trailing window holds the b+1 band columns c = q..q+b
// as cw[slot][k] = A(c + k, c), k = 0..b, in slots c mod (b+1).  At pivot q:
//   1. (every 64 pivots) stage the entries of the columns entering at the next
//      64 pivots (diagonal, A(c+1, c), A(c+b, c)), double-buffered;
//   2. column q+b enters the slot that pivot q-1 freed;
//   3. d = A(q, q), l_i = A(q+i, q) / d, output F[q] = {d, l_1 .. l_b};
//   4. rank-1 update A(q+j+k, q+j) -= (l_{j+k} d) l_j over the packed
//      elements (j in 1..b, k in 0..b-j) of the host-built table `jk`,
//      interleaved over the threads so neighbouring threads touch neighbouring
//      entries of one column.
// Two barriers per pivot.
constexpr int DC_STAGE = 64;

template <class TF>
__host__ __device__ inline size_t dc_factor_smem(int b) {
  const size_t W = size_t(b) + 1, T = size_t(b) * (b + 1) / 2;
  return (W * W + 2 * W + 6 * DC_STAGE) * sizeof(TF) + T * sizeof(unsigned);
}

template <class TF>
__global__ void __launch_bounds__(256) k_dc_factor(const DcGrid G, const double* ox, const double* oz,
                                                   const double* dbase, const double* sig, const double* alpha,
                                                   const double* ky2, const unsigned* jk, int sys0, TF* fac,
                                                   int* status) {
  extern __shared__ __align__(16) unsigned char shraw[];
  const int N = G.N, b = G.b, W = b + 1;
  const int T = b * (b + 1) / 2;
  TF* cw = reinterpret_cast<TF*>(shraw);
  TF* lc = cw + W * W;        // l_i, i = 1..b
  TF* lcd = lc + W;           // l_i d
  TF* stg = lcd + W;          // [2][3][DC_STAGE]: diag | A(c+1, c) | A(c+b, c)
  unsigned* tab = reinterpret_cast<unsigned*>(stg + 6 * DC_STAGE);
  const int sys = blockIdx.x;
  const double* al = alpha + size_t(sys0 + sys) * G.nb;
  const double k2 = ky2[sys0 + sys];
  TF* F = fac + size_t(sys) * size_t(N) * W;
  const int nth = blockDim.x, tid = threadIdx.x;
  auto diag = [&](int c) {
    int l, h;
    dc_lh(G, c, l, h);
    return TF(dc_diag(G, dbase, sig, al, k2, l, h));
  };
  for (int e = tid; e < T; e += nth) tab[e] = jk[e];
  for (int e = tid; e < W * W; e += nth) {  // columns 0..b
    const int c = e / W, k = e % W;
    TF v = TF(0);
    if (c < N && c + k < N) {
      if (k == 0) v = diag(c);
      else if (k == 1) v = TF(dc_sub(G, ox, oz, c + 1, 1));
      else if (k == b) v = TF(dc_sub(G, ox, oz, c + b, b));
    }
    cw[e] = v;
  }
  for (int q = 0; q < N; ++q) {
    const int p0 = q % W;
    if (q % DC_STAGE == 0) {  // 1. columns entering after pivots q .. q+63
      TF* sb = stg + ((q / DC_STAGE) & 1) * 3 * DC_STAGE;
      for (int t = tid; t < DC_STAGE; t += nth) {
        const int c = q + W + t;
        TF d = TF(0), s1 = TF(0), s2 = TF(0);
        if (c < N) {
          d = diag(c);
          if (c + 1 < N) s1 = TF(dc_sub(G, ox, oz, c + 1, 1));
          if (c + b < N) s2 = TF(dc_sub(G, ox, oz, c + b, b));
        }
        sb[t] = d; sb[DC_STAGE + t] = s1; sb[2 * DC_STAGE + t] = s2;
      }
    }
    if (q >= 1) {  // 2. column q-1+W into slot (q-1) mod W
      const int qq = q - 1;
      const TF* sb = stg + ((qq / DC_STAGE) & 1) * 3 * DC_STAGE;
      const int t = qq % DC_STAGE;
      TF* col = cw + (qq % W) * W;
      for (int k = tid; k < W; k += nth)
        col[k] = k == 0 ? sb[t] : (k == 1 ? sb[DC_STAGE + t] : (k == b ? sb[2 * DC_STAGE + t] : TF(0)));
    }
    __syncthreads();  // stage 1 of pivot q-64.. and 2 visible; previous update complete
    // 3. pivot
    const TF* pc = cw + p0 * W;
    const TF d = pc[0];
    if (tid == 0) {
      F[size_t(q) * W] = d;
      if (!(d != TF(0)) || !isfinite(d)) atomicExch(status + sys0 + sys, 1);
    }
    for (int i = tid + 1; i <= b; i += nth) {
      const TF li = (q + i < N) ? pc[i] / d : TF(0);
      lc[i] = li;
      lcd[i] = li * d;
      F[size_t(q) * W + i] = li;
    }
    __syncthreads();
    // 4. rank-1 update of columns q+1 .. q+b
    for (int e = tid; e < T; e += nth) {
      const unsigned jkv = tab[e];
      const int j = int(jkv >> 16), k = int(jkv & 0xffffu);
      int slot = p0 + j;
      if (slot >= W) slot -= W;
      cw[slot * W + k] -= lcd[j + k] * lc[j];
    }
  }
}

// z = (L D L^T)^{-1} r for every system, one warp per system, and rz = r.z.
// r, z are FP64 vectors in the reference layout [sys][l + h*n].  The rolling
// window (b+1 values) lives in shared memory per warp; factor columns stream
// through a per-warp ring of DC_RING columns with cp.async (issued DC_RING - 1
// pivots ahead), r / z values 32 steps at a time (one per lane).
constexpr int DC_RING = 16;

template <class TF>
__host__ __device__ inline size_t dc_precond_smem(int b, int warps) {
  return size_t(warps) * (size_t(b) + 1) * (DC_RING + 1) * sizeof(TF);
}

__device__ __forceinline__ unsigned dc_smem_addr(const void* p) {
  return static_cast<unsigned>(__cvta_generic_to_shared(p));
}

// Copies factor column q (b+1 entries) into a ring slot, one commit group.
template <class TF>
__device__ __forceinline__ void dc_col_async(TF* dst, const TF* F, int q, int N, int W, int lane) {
  if (q >= 0 && q < N) {
    const TF* src = F + size_t(q) * W;
    for (int i = lane; i < W; i += 32)
      asm volatile("cp.async.ca.shared.global [%0], [%1], %2;\n" ::"r"(dc_smem_addr(dst + i)), "l"(src + i),
                   "n"(int(sizeof(TF)))
                   : "memory");
  }
  asm volatile("cp.async.commit_group;\n" ::: "memory");
}

template <class TF>
__global__ void k_dc_precond(const DcGrid G, const TF* fac, const double* r, double* z, double* rz,
                             int nsys, const int* done) {
  extern __shared__ __align__(16) unsigned char shpraw[];
  TF* shp = reinterpret_cast<TF*>(shpraw);
  const int W = G.b + 1;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int sys = blockIdx.x * (blockDim.x >> 5) + warp;
  if (sys >= nsys || (done && done[sys])) return;
  TF* win = shp + size_t(warp) * W * (DC_RING + 1);
  TF* ring = win + W;  // DC_RING columns of W entries
  const TF* F = fac + size_t(sys) * size_t(G.N) * W;
  const double* R = r + size_t(sys) * G.N;
  double* Z = z + size_t(sys) * G.N;
  const int N = G.N, b = G.b;
  constexpr int MAXI = 8;  // b <= 256 -> at most 8 entries of a column per lane
  auto ref = [&](int q) { int l, h; dc_lh(G, q, l, h); return l + h * G.n; };
  auto wait_ring = [&]() { asm volatile("cp.async.wait_group %0;\n" ::"n"(DC_RING - 1) : "memory"); __syncwarp(); };
  // forward: L y = r
  for (int i = lane; i < W; i += 32) win[i] = (i < N) ? TF(R[ref(i)]) : TF(0);
  for (int p = 0; p < DC_RING - 1; ++p) dc_col_async(ring + (p % DC_RING) * W, F, p, N, W, lane);
  __syncwarp();
  double rpre = 0.0;
  for (int q = 0; q < N; ++q) {
    if ((q & 31) == 0) {  // r values entering the window over the next 32 steps
      const int nq = q + W + lane;
      rpre = (nq < N) ? R[ref(nq)] : 0.0;
    }
    dc_col_async(ring + ((q + DC_RING - 1) % DC_RING) * W, F, q + DC_RING - 1, N, W, lane);
    wait_ring();
    const TF* col = ring + (q % DC_RING) * W;
    const TF dq = col[0];
    const int p0 = q % W;
    const TF y = win[p0];
#pragma unroll
    for (int u = 0; u < MAXI; ++u) {
      const int i = lane + 1 + 32 * u;
      if (i <= b && q + i < N) { int pi = p0 + i; if (pi >= W) pi -= W; win[pi] -= col[i] * y; }
    }
    const double rin = __shfl_sync(0xffffffffu, rpre, q & 31);
    __syncwarp();
    if (lane == 0) {
      Z[ref(q)] = double(y / dq);
      win[p0] = (q + W < N) ? TF(rin) : TF(0);
    }
    __syncwarp();  // the ring slot of column q is refilled at pivot q+1
  }
  asm volatile("cp.async.wait_group 0;\n" ::: "memory");
  __threadfence_block();
  // backward: L^T x = z, x_q = z_q - sum_i l_{q+i,q} x_{q+i}
  for (int i = lane; i < W; i += 32) win[i] = TF(0);
  __syncwarp();
  for (int p = 0; p < DC_RING - 1; ++p) dc_col_async(ring + (p % DC_RING) * W, F, N - 1 - p, N, W, lane);
  double acc = 0.0;
  double zpre = 0.0, rpre2 = 0.0;
  for (int q = N - 1; q >= 0; --q) {
    const int s_ = N - 1 - q;  // step of the backward sweep
    const int k = s_ & 31;
    if (k == 0) {  // z and r values of the next 32 steps (descending)
      const int qq = q - lane;
      zpre = (qq >= 0) ? Z[ref(qq)] : 0.0;
      rpre2 = (qq >= 0) ? R[ref(qq)] : 0.0;
    }
    dc_col_async(ring + ((s_ + DC_RING - 1) % DC_RING) * W, F, q - (DC_RING - 1), N, W, lane);
    wait_ring();
    const TF* col = ring + (s_ % DC_RING) * W;
    TF sum = TF(0);
#pragma unroll
    for (int u = 0; u < MAXI; ++u) {
      const int i = lane + 1 + 32 * u;
      if (i <= b && q + i < N) { int pi = q % W + i; if (pi >= W) pi -= W; sum += col[i] * win[pi]; }
    }
    for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
    const double zq = __shfl_sync(0xffffffffu, zpre, k);
    const double rq = __shfl_sync(0xffffffffu, rpre2, k);
    if (lane == 0) {
      const TF x = TF(zq) - sum;
      win[q % W] = x;
      Z[ref(q)] = double(x);
      acc += rq * double(x);
    }
    __syncwarp();
  }
  asm volatile("cp.async.wait_group 0;\n" ::: "memory");
  if (lane == 0) rz[sys] = acc;
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

// 2.5D DC-resistivity forward and sensitivity: host driver of dc_kernels.cuh.
//
// For every (source, ky) system: Lk u_k = 0.5 s (dc_fwd_k.m:40-43), then
// u = (2/pi) sum_k w_k u_k and d = M u (dc_fwd2_5d.m:50-54); for the gradient,
// Lk a_k = M' e (dc_adjoint.m:10, Lk is symmetric), g_k = Sk(u_k) a_k and
// g = (2/pi) sum_k w_k g_k trimmed of the Robin padding (dc_gradient2_5d.m).
// All systems of a batch of sources are solved together by FP64 CG
// preconditioned with the band LDL^T factor of each system (FP64 by default,
// FP32 on request), or, as an option, with the FP32 red-black IC(0)
// preconditioner (k_dc_ic0_*).
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "dc_kernels.cuh"
#include "gj_internal.h"

namespace gj {

// Columns of the factor's trailing-update register tiles (4 rows x 4 columns
// by default; GJ_DC_TILE=8 selects 4 x 8, which spills at 128 registers).
static int dc_tile_cols() {
  const char* e = getenv("GJ_DC_TILE");
  return (e && atoi(e) == 8) ? 8 : 4;
}
// Shape of the substitution's shared-memory ring: chunks of `ch` factor
// columns, `nst` chunks (8 x 4 by default; GJ_DC_RING=CHxNST picks 4x4, 4x8,
// 8x4 or 16x4).
struct DcRing { int ch = 8, nst = 4; };
static DcRing dc_ring() {
  DcRing r;
  if (const char* e = getenv("GJ_DC_RING")) {
    int a = 0, b = 0;
    if (sscanf(e, "%dx%d", &a, &b) == 2 &&
        ((a == 4 && (b == 4 || b == 8)) || (a == 8 && b == 4) || (a == 16 && b == 4))) { r.ch = a; r.nst = b; }
  }
  return r;
}
// The substitution kernel of a window of 32 R band positions and a ring shape.
template <class TF>
static void (*dc_precond_kernel(int b, DcRing r))(const DcGrid, const TF*, const double*, double*, double*, int,
                                                   const int*) {
  const bool wide = b >= 128;
  if (r.ch == 4 && r.nst == 4) return wide ? k_dc_precond<TF, 8, 4, 4> : k_dc_precond<TF, 4, 4, 4>;
  if (r.ch == 4) return wide ? k_dc_precond<TF, 8, 4, 8> : k_dc_precond<TF, 4, 4, 8>;
  if (r.ch == 16) return wide ? k_dc_precond<TF, 8, 16, 4> : k_dc_precond<TF, 4, 16, 4>;
  return wide ? k_dc_precond<TF, 8, 8, 4> : k_dc_precond<TF, 4, 8, 4>;
}

namespace {

__global__ void k_dc_rhs_src(int N, const long* ab, const double* cur, int nky, int sys0, int nsys, double* b) {
  const int sys = blockIdx.x * blockDim.x + threadIdx.x;
  if (sys >= nsys) return;
  const int src = (sys0 + sys) / nky;
  double* B = b + size_t(sys) * N;
  // 0.5 * s with s = +I at A, -I at B (dc_electrodes.m:54-55, dc_fwd_k.m:40)
  B[ab[2 * src]] += 0.5 * cur[src];
  B[ab[2 * src + 1]] -= 0.5 * cur[src];
}

// d[src][j] = (2/pi) sum_k w_k (u_k(M_j) - u_k(N_j)) for the sources of a batch.
__global__ void k_dc_data(int N, int nky, int src0, int nsrc_b, const long* mn_off, const long* mn, const double* wts,
                          const double* uk, double* d) {
  const int sb = blockIdx.y;
  if (sb >= nsrc_b) return;
  const int src = src0 + sb;
  const long o0 = mn_off[src], o1 = mn_off[src + 1];
  for (long j = o0 + threadIdx.x + long(blockIdx.x) * blockDim.x; j < o1; j += long(blockDim.x) * gridDim.x) {
    double v = 0;
    for (int k = 0; k < nky; ++k) {
      const double* U = uk + (size_t(sb) * nky + k) * N;
      v += wts[size_t(src) * nky + k] * (U[mn[2 * j]] - U[mn[2 * j + 1]]);
    }
    d[j] = (2.0 / 3.14159265358979323846) * v;
  }
}

// Adjoint right-hand side M' e for every ky of a source (dc_adjoint.m:10).
__global__ void k_dc_rhs_adj(int N, int nky, int src0, int nsrc_b, const long* mn_off, const long* mn,
                             const double* e, double* b) {
  const int sb = blockIdx.y;
  if (sb >= nsrc_b) return;
  const int src = src0 + sb;
  const long o0 = mn_off[src], o1 = mn_off[src + 1];
  for (long j = o0 + threadIdx.x; j < o1; j += blockDim.x)
    for (int k = 0; k < nky; ++k) {
      double* B = b + (size_t(sb) * nky + k) * N;
      atomicAdd(B + mn[2 * j], e[j]);
      atomicAdd(B + mn[2 * j + 1], -e[j]);
    }
}

// u[src] = (2/pi) sum_k w_k u_k (dc_fwd2_5d.m:51).
__global__ void k_dc_stack(int N, int nky, int src0, int nsrc_b, const double* wts, const double* uk, double* u) {
  const int sb = blockIdx.y;
  if (sb >= nsrc_b) return;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < N; t += blockDim.x * gridDim.x) {
    double v = 0;
    for (int k = 0; k < nky; ++k) v += wts[size_t(src0 + sb) * nky + k] * uk[(size_t(sb) * nky + k) * N + t];
    u[size_t(sb) * N + t] = (2.0 / 3.14159265358979323846) * v;
  }
}

}  // namespace

struct DcPlan {
  DcGrid G{};
  int nky = 0, nsrc = 0, robin = 0;
  DevBuf sig, faces, ky2, wts, alpha, ab, cur, mnoff, mnbuf, dots, done, status, gbuf, dbuf, ebuf, ubuf;
  DevBuf tiles;  // the factor's trailing-update tiles, (ct << 16) | rt, column-major
  int ntiles = 0;
  std::vector<long> off;
};

template <class TF>
static gj_status pcg(Err& err, Ctx& c, DcPlan& P, int sys0, int nsys, double* B, double* X, double tol, int maxit,
                     int& iters, double& relmax, cudaStream_t st, bool ic0 = false) {
  const DcGrid& G = P.G;
  const int N = G.N;
  const size_t vn = size_t(nsys) * N;
  double* R = X + vn;
  double* Z = R + vn;
  double* Pv = Z + vn;
  double* AP = Pv + vn;
  double* d = P.dots.as<double>();
  double* rzA = d; double* rzB = d + nsys; double* pap = d + 2 * nsys; double* rr = d + 3 * nsys;
  double* bb = d + 4 * nsys;
  double* rzo = d + 5 * nsys;
  int* done = P.done.as<int>();
  const double* ox = P.faces.as<double>();
  const double* oz = ox + N;
  const double* db = oz + N;
  const double* sg = P.sig.as<double>();
  const double* al = P.alpha.as<double>();
  const double* k2 = P.ky2.as<double>();
  const TF* F = c.dc_fac.as<TF>();
  const dim3 gv((N + 255) / 256 < 64 ? (N + 255) / 256 : 64, nsys);
  const DcRing ring = dc_ring();
  const size_t shp = dc_precond_smem<TF>(G.wp, ring.ch, ring.nst);
  const auto kpre = dc_precond_kernel<TF>(G.b, ring);
  auto precond = [&](double* rzv) {  // one warp per system; window of 32R >= b + 1 positions
    const bool tm = c.timer.begin(KK_DC_PRECOND, st, nsys);
    if (ic0) {  // two FP32 sweeps of the red-black IC(0) factor
      cudaMemsetAsync(rzv, 0, nsys * sizeof(double), st);
      const float* Dv = c.dc_fac.as<float>();
      k_dc_ic0_black<<<gv, 256, 0, st>>>(G, Dv, ox, oz, R, Z, rzv, nsys, done);
      k_dc_ic0_red<<<gv, 256, 0, st>>>(G, Dv, ox, oz, R, Z, rzv, nsys, done);
      c.launches += 1;
    } else {
      kpre<<<nsys, 32, shp, st>>>(G, F, R, Z, rzv, nsys, done);
    }
    c.timer.end(tm, st);
  };
  GJ_CUDA(err, cudaMemsetAsync(X, 0, vn * sizeof(double), st));
  GJ_CUDA(err, cudaMemcpyAsync(R, B, vn * sizeof(double), cudaMemcpyDeviceToDevice, st));
  GJ_CUDA(err, cudaMemsetAsync(done, 0, nsys * sizeof(int), st));
  GJ_CUDA(err, cudaMemsetAsync(bb, 0, nsys * sizeof(double), st));
  GJ_CUDA(err, cudaMemsetAsync(rr, 0, nsys * sizeof(double), st));
  k_dc_residual<<<gv, 256, 0, st>>>(N, B, X, R, rr, bb, nsys);  // r = b (x = 0)
  precond(rzA);
  k_dc_cg_p<<<gv, 256, 0, st>>>(N, rzA, rzA, nullptr, Z, Pv, 1, nsys, done);
  c.launches += 3;
  std::vector<double> hbb(nsys), hrr(nsys);
  std::vector<int> hdone(nsys, 0);
  GJ_CUDA(err, cudaMemcpyAsync(hbb.data(), bb, nsys * sizeof(double), cudaMemcpyDeviceToHost, st));
  iters = 0;
  for (int it = 0; it < maxit; ++it) {
    GJ_CUDA(err, cudaMemsetAsync(pap, 0, nsys * sizeof(double), st));
    GJ_CUDA(err, cudaMemsetAsync(rr, 0, nsys * sizeof(double), st));
    GJ_CUDA(err, cudaMemsetAsync(rzo, 0, nsys * sizeof(double), st));
    k_dc_apply<<<gv, 256, 0, st>>>(G, ox, oz, db, sg, al, k2, sys0, Pv, AP, pap, nsys, done);
    k_dc_cg_xr<<<gv, 256, 0, st>>>(N, rzA, pap, X, R, Pv, AP, Z, rr, rzo, nsys, done);
    precond(rzB);
    k_dc_cg_p<<<gv, 256, 0, st>>>(N, rzB, rzA, rzo, Z, Pv, 0, nsys, done);
    c.launches += 4;
    std::swap(rzA, rzB);
    GJ_CUDA(err, cudaMemcpyAsync(hrr.data(), rr, nsys * sizeof(double), cudaMemcpyDeviceToHost, st));
    GJ_CUDA(err, cudaStreamSynchronize(st));
    iters = it + 1;
    bool all = true;
    for (int s = 0; s < nsys; ++s) {
      if (hdone[s]) continue;
      const double rel = hbb[s] > 0 ? std::sqrt(hrr[s] / hbb[s]) : 0.0;
      if (rel <= tol) hdone[s] = 1;
      else all = false;
    }
    GJ_CUDA(err, cudaMemcpyAsync(done, hdone.data(), nsys * sizeof(int), cudaMemcpyHostToDevice, st));
    if (all) break;
  }
  // true FP64 residual of the final iterate
  GJ_CUDA(err, cudaMemsetAsync(rr, 0, nsys * sizeof(double), st));
  k_dc_apply<<<gv, 256, 0, st>>>(G, ox, oz, db, sg, al, k2, sys0, X, AP, nullptr, nsys, nullptr);
  k_dc_residual<<<gv, 256, 0, st>>>(N, B, AP, R, rr, nullptr, nsys);
  c.launches += 2;
  GJ_CUDA(err, cudaMemcpyAsync(hrr.data(), rr, nsys * sizeof(double), cudaMemcpyDeviceToHost, st));
  GJ_CUDA(err, cudaStreamSynchronize(st));
  relmax = 0;
  for (int s = 0; s < nsys; ++s) relmax = std::max(relmax, hbb[s] > 0 ? std::sqrt(hrr[s] / hbb[s]) : 0.0);
  GJ_CUDA(err, cudaGetLastError());
  return GJ_OK;
}

template <class TF>
static gj_status dc_run_t(Ctx& c, const gj_dc_grid& gg, const double* sigma, const gj_dc_src* srcs, int nsrc,
                          bool grad, const gj_dc_opts& o, double* d_out, double* e_out, double* u_out, double* g_out,
                          double* misfit_out, gj_dc_stats* stats, double* uk_out) {
  Err& err = c.err;
  if (!sigma || !srcs || nsrc < 1) return err.set(GJ_EINVAL, "null sigma/sources or nsrc < 1");
  if (gg.n < 3 || gg.m < 3 || gg.n_ky < 1 || gg.robin < 0 || 2 * gg.robin >= gg.n || gg.robin >= gg.m)
    return err.set(GJ_EINVAL, "bad DC grid (n, m >= 3, n_ky >= 1, robin padding smaller than the grid)");
  if (!(gg.dx != 0 && gg.dz != 0)) return err.set(GJ_EINVAL, "dx and dz must be nonzero");
  DcPlan P;
  DcGrid& G = P.G;
  G.n = gg.n; G.m = gg.m; G.N = gg.n * gg.m;
  G.depth_fast = gg.m <= gg.n ? 1 : 0;
  G.b = std::min(gg.n, gg.m);
  G.DX = gg.dx; G.DZ = gg.dz;
  G.nb = 2 * (gg.m - 2) + (gg.n - 2) + 4;
  {
    const int per16 = 16 / int(sizeof(TF));  // factor columns start on 16-byte boundaries
    G.wp = (G.b + 1 + per16 - 1) / per16 * per16;
    G.nq = (G.N + 31) / 32 * 32;
  }
  {
    int dev = 0, maxsm = 0;
    GJ_CUDA(err, cudaGetDevice(&dev));
    GJ_CUDA(err, cudaDeviceGetAttribute(&maxsm, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    if (G.b > DC_FACTOR_THREADS - DC_NB - 1 || dc_factor_smem<TF>(G.b) > size_t(maxsm) ||
        dc_precond_smem<TF>(G.wp, dc_ring().ch, dc_ring().nst) > size_t(maxsm))
      return err.set(GJ_EUNSUPPORTED, "band width min(n, m) = %d: the factor window needs %zu bytes of shared memory "
                                      "(limit %d)", G.b, dc_factor_smem<TF>(G.b), maxsm);
  }
  P.nky = gg.n_ky; P.nsrc = nsrc; P.robin = gg.robin;
  const int N = G.N, nky = P.nky, nsys_all = nsrc * nky;
  cudaStream_t st = 0;
  Marks marks;
  c.timer.cur = &marks;
  struct Unset { Ctx& c; ~Unset() { c.timer.cur = nullptr; } } unset{c};
  // ---- inputs
  std::vector<double> hky2(nsys_all), hw(nsys_all), hal(size_t(nsys_all) * G.nb), hcur(nsrc);
  std::vector<long> hab(2 * nsrc), hmn;
  P.off.assign(nsrc + 1, 0);
  for (int s = 0; s < nsrc; ++s) {
    const gj_dc_src& q = srcs[s];
    if (q.a < 0 || q.a >= N || q.b < 0 || q.b >= N) return err.set(GJ_EINVAL, "source %d: electrode outside the grid", s);
    if (!q.ky || !q.w || !q.alpha) return err.set(GJ_EINVAL, "source %d: null ky/w/alpha", s);
    if (q.nd < 0 || (q.nd > 0 && !q.mn)) return err.set(GJ_EINVAL, "source %d: bad receivers", s);
    if (grad && q.nd > 0 && !q.d_obs) return err.set(GJ_EINVAL, "source %d: gradient needs d_obs", s);
    hab[2 * s] = q.a; hab[2 * s + 1] = q.b; hcur[s] = q.current;
    for (int k = 0; k < nky; ++k) {
      hky2[s * nky + k] = q.ky[k] * q.ky[k];
      hw[s * nky + k] = q.w[k];
      for (int e = 0; e < G.nb; ++e) hal[(size_t(s) * nky + k) * G.nb + e] = q.alpha[size_t(k) * G.nb + e];
    }
    for (int j = 0; j < 2 * q.nd; ++j) {
      if (q.mn[j] < 0 || q.mn[j] >= N) return err.set(GJ_EINVAL, "source %d: receiver node outside the grid", s);
      hmn.push_back(q.mn[j]);
    }
    P.off[s + 1] = P.off[s] + q.nd;
  }
  const long ndat = P.off[nsrc];
  GJ_TRY(P.sig.alloc(err, N * sizeof(double)));
  GJ_TRY(P.faces.alloc(err, 3 * size_t(N) * sizeof(double)));
  GJ_TRY(P.ky2.alloc(err, nsys_all * sizeof(double)));
  GJ_TRY(P.wts.alloc(err, nsys_all * sizeof(double)));
  GJ_TRY(P.alpha.alloc(err, hal.size() * sizeof(double)));
  GJ_TRY(P.ab.alloc(err, hab.size() * sizeof(long)));
  GJ_TRY(P.cur.alloc(err, nsrc * sizeof(double)));
  GJ_TRY(P.mnoff.alloc(err, (nsrc + 1) * sizeof(long)));
  GJ_TRY(P.mnbuf.alloc(err, std::max<size_t>(hmn.size(), 2) * sizeof(long)));
  GJ_TRY(P.dbuf.alloc(err, std::max<long>(ndat, 1) * sizeof(double)));
  GJ_TRY(P.ebuf.alloc(err, std::max<long>(ndat, 1) * sizeof(double)));
  GJ_TRY(P.status.alloc(err, nsys_all * sizeof(int)));
  GJ_CUDA(err, cudaMemcpy(P.sig.p, sigma, N * sizeof(double), cudaMemcpyHostToDevice));
  GJ_CUDA(err, cudaMemcpy(P.ky2.p, hky2.data(), nsys_all * sizeof(double), cudaMemcpyHostToDevice));
  GJ_CUDA(err, cudaMemcpy(P.wts.p, hw.data(), nsys_all * sizeof(double), cudaMemcpyHostToDevice));
  GJ_CUDA(err, cudaMemcpy(P.alpha.p, hal.data(), hal.size() * sizeof(double), cudaMemcpyHostToDevice));
  GJ_CUDA(err, cudaMemcpy(P.ab.p, hab.data(), hab.size() * sizeof(long), cudaMemcpyHostToDevice));
  GJ_CUDA(err, cudaMemcpy(P.cur.p, hcur.data(), nsrc * sizeof(double), cudaMemcpyHostToDevice));
  GJ_CUDA(err, cudaMemcpy(P.mnoff.p, P.off.data(), (nsrc + 1) * sizeof(long), cudaMemcpyHostToDevice));
  if (!hmn.empty()) GJ_CUDA(err, cudaMemcpy(P.mnbuf.p, hmn.data(), hmn.size() * sizeof(long), cudaMemcpyHostToDevice));
  GJ_CUDA(err, cudaMemset(P.status.p, 0, nsys_all * sizeof(int)));
  double* ox = P.faces.as<double>();
  k_dc_faces<<<(N + 255) / 256, 256, 0, st>>>(G, P.sig.as<double>(), ox, ox + N, ox + 2 * N);
  ++c.launches;
  if (grad) {
    GJ_TRY(P.gbuf.alloc(err, size_t(nsrc) * N * sizeof(double)));
    GJ_CUDA(err, cudaMemset(P.gbuf.p, 0, size_t(nsrc) * N * sizeof(double)));
  }
  if (u_out) GJ_TRY(P.ubuf.alloc(err, size_t(nsrc) * N * sizeof(double)));
  // ---- batch size from the memory budget: FP32 factor + 7 FP64 vectors + u_k per system
  size_t free_b = 0, total_b = 0;
  GJ_CUDA(err, cudaMemGetInfo(&free_b, &total_b));
  const size_t reusable = c.dc_fac.bytes + c.dc_vec.bytes;  // this context's DC buffers from earlier calls
  const size_t budget = o.mem_budget_bytes ? o.mem_budget_bytes : size_t(0.7 * double(free_b + reusable));
  const bool ic0 = o.precond == 1;
  const size_t fac_sys = ic0 ? size_t(N) * sizeof(float) : size_t(G.nq) * G.wp * sizeof(TF);
  const size_t per_sys = fac_sys + size_t(N) * 8 * sizeof(double) + 64;
  int srcs_per_batch = int(std::min<size_t>(nsrc, std::max<size_t>(1, budget / (per_sys * nky))));
  if (o.sources_per_batch > 0) srcs_per_batch = std::min(srcs_per_batch, o.sources_per_batch);
  const int nsys_b = srcs_per_batch * nky;
  GJ_TRY(c.dc_fac.alloc(err, size_t(nsys_b) * fac_sys));
  GJ_TRY(c.dc_vec.alloc(err, size_t(nsys_b) * N * 7 * sizeof(double)));  // B, X, R, Z, P, AP, U
  GJ_TRY(P.dots.alloc(err, 6 * size_t(nsys_b) * sizeof(double)));
  GJ_TRY(P.done.alloc(err, nsys_b * sizeof(int)));
  const double tol = o.tol > 0 ? o.tol : 1e-10;
  const int maxit = o.max_iter > 0 ? o.max_iter : (ic0 ? 20000 : 50);
  int it_max = 0;
  double rel_max = 0;
  const size_t smem_f = dc_factor_smem<TF>(G.b);
  const int tc = dc_tile_cols();
  const auto kfac = tc == 8 ? k_dc_factor<TF, 8> : k_dc_factor<TF, 4>;
  GJ_CUDA(err, cudaFuncSetAttribute(kfac, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem_f)));
  {
    const DcRing ring = dc_ring();
    GJ_CUDA(err, cudaFuncSetAttribute(dc_precond_kernel<TF>(G.b, ring), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      int(dc_precond_smem<TF>(G.wp, ring.ch, ring.nst))));
  }
  {
    // tiles of 4 rows x tc columns on or below the diagonal, column-major
    const DcFactorShape fs = dc_factor_shape(G.b);
    const int nt = fs.BP / 4, nct = (tc == 8 ? fs.BPU : fs.BP) / tc;
    std::vector<unsigned> ht;
    for (int ct = 0; ct < nct; ++ct)
      for (int rt = tc * ct / 4; rt < nt; ++rt) ht.push_back((unsigned(ct) << 16) | unsigned(rt));
    if (ht.size() > size_t(fs.ntiles)) return err.set(GJ_EINVAL, "factor tile list longer than its shared-memory table");
    P.ntiles = int(ht.size());
    GJ_TRY(P.tiles.alloc(err, ht.size() * sizeof(unsigned)));
    GJ_CUDA(err, cudaMemcpy(P.tiles.p, ht.data(), ht.size() * sizeof(unsigned), cudaMemcpyHostToDevice));
  }
  double* V = c.dc_vec.as<double>();
  for (int s0 = 0; s0 < nsrc; s0 += srcs_per_batch) {
    const int nsb = std::min(srcs_per_batch, nsrc - s0);
    const int nsys = nsb * nky, sys0 = s0 * nky;
    const size_t vn = size_t(nsys) * N;
    double* B = V;
    double* X = B + vn;  // X, R, Z, P, AP follow (pcg layout)
    double* U = X + 5 * vn;
    // factor (band LDL^T), or the IC(0) diagonals
    {
      const bool tm = c.timer.begin(KK_DC_FACTOR, st, nsys);
      if (ic0) {
        const dim3 gv((N + 255) / 256 < 64 ? (N + 255) / 256 : 64, nsys);
        k_dc_ic0_setup<<<gv, 256, 0, st>>>(G, ox, ox + N, ox + 2 * N, P.sig.as<double>(), P.alpha.as<double>(),
                                           P.ky2.as<double>(), sys0, nsys, c.dc_fac.as<float>(),
                                           P.status.as<int>());
      } else {
        kfac<<<nsys, DC_FACTOR_THREADS, smem_f, st>>>(G, ox, ox + N, ox + 2 * N, P.sig.as<double>(),
                                                      P.alpha.as<double>(), P.ky2.as<double>(),
                                                      P.tiles.as<unsigned>(), P.ntiles, sys0, c.dc_fac.as<TF>(),
                                                      P.status.as<int>());
      }
      c.timer.end(tm, st);
      ++c.launches;
    }
    // forward solves
    GJ_CUDA(err, cudaMemsetAsync(B, 0, vn * sizeof(double), st));
    k_dc_rhs_src<<<(nsys + 127) / 128, 128, 0, st>>>(N, P.ab.as<long>(), P.cur.as<double>(), nky, sys0, nsys, B);
    ++c.launches;
    int iters = 0; double rel = 0;
    GJ_TRY(pcg<TF>(err, c, P, sys0, nsys, B, X, tol, maxit, iters, rel, st, ic0));
    it_max = std::max(it_max, iters); rel_max = std::max(rel_max, rel);
    GJ_CUDA(err, cudaMemcpyAsync(U, X, vn * sizeof(double), cudaMemcpyDeviceToDevice, st));
    // per-wavenumber potentials u_k of the batch's sources: [source][ky][node], the
    // column-major N x n_ky u_k of dc_fwd2_5d.m:61 per source
    if (uk_out)
      GJ_CUDA(err, cudaMemcpyAsync(uk_out + size_t(sys0) * N, U, vn * sizeof(double), cudaMemcpyDeviceToHost, st));
    k_dc_data<<<dim3(4, nsb), 256, 0, st>>>(N, nky, s0, nsb, P.mnoff.as<long>(), P.mnbuf.as<long>(), P.wts.as<double>(),
                                             U, P.dbuf.as<double>());
    ++c.launches;
    if (u_out) {
      k_dc_stack<<<dim3(64, nsb), 256, 0, st>>>(N, nky, s0, nsb, P.wts.as<double>(), U,
                                                 P.ubuf.as<double>() + size_t(s0) * N);
      ++c.launches;
    }
    if (grad) {
      // e = d - d_obs for the batch (host: small), adjoint right-hand sides
      const long o0 = P.off[s0], o1 = P.off[s0 + nsb];
      std::vector<double> hd(o1 - o0), he(o1 - o0);
      GJ_CUDA(err, cudaMemcpyAsync(hd.data(), P.dbuf.as<double>() + o0, (o1 - o0) * sizeof(double),
                                   cudaMemcpyDeviceToHost, st));
      GJ_CUDA(err, cudaStreamSynchronize(st));
      for (int s = s0; s < s0 + nsb; ++s)
        for (long j = P.off[s]; j < P.off[s + 1]; ++j)
          he[j - o0] = hd[j - o0] - srcs[s].d_obs[j - P.off[s]];  // dc_fwd2_5d.m:56
      GJ_CUDA(err, cudaMemcpyAsync(P.ebuf.as<double>() + o0, he.data(), he.size() * sizeof(double),
                                   cudaMemcpyHostToDevice, st));
      GJ_CUDA(err, cudaMemsetAsync(B, 0, vn * sizeof(double), st));
      k_dc_rhs_adj<<<dim3(1, nsb), 256, 0, st>>>(N, nky, s0, nsb, P.mnoff.as<long>(), P.mnbuf.as<long>(),
                                                 P.ebuf.as<double>(), B);
      ++c.launches;
      GJ_TRY(pcg<TF>(err, c, P, sys0, nsys, B, X, tol, maxit, iters, rel, st, ic0));
      it_max = std::max(it_max, iters); rel_max = std::max(rel_max, rel);
      k_dc_sens<<<dim3(64, nsys), 256, 0, st>>>(G, P.sig.as<double>(), P.alpha.as<double>(), P.ky2.as<double>(),
                                                P.wts.as<double>(), sys0, nky, U, X, P.gbuf.as<double>(), nsys);
      ++c.launches;
      GJ_CUDA(err, cudaStreamSynchronize(st));
    }
  }
  GJ_CUDA(err, cudaGetLastError());
  GJ_CUDA(err, cudaDeviceSynchronize());
  c.timer.collect(marks);
  std::vector<int> hst(nsys_all);
  GJ_CUDA(err, cudaMemcpy(hst.data(), P.status.p, nsys_all * sizeof(int), cudaMemcpyDeviceToHost));
  for (int s = 0; s < nsys_all; ++s)
    if (hst[s]) return err.set(GJ_ENUMERIC, "zero or non-finite pivot in the %s of system %d",
                               ic0 ? "IC(0) factor" : "band factor", s);
  if (stats) { stats->max_iterations = it_max; stats->max_rel_residual = rel_max; }
  if (rel_max > tol * 10)
    return err.set(GJ_ENUMERIC, "CG reached relative residual %.3e > %.1e after %d iterations", rel_max, tol, it_max);
  std::vector<double> hd(ndat);
  if (ndat) GJ_CUDA(err, cudaMemcpy(hd.data(), P.dbuf.p, ndat * sizeof(double), cudaMemcpyDeviceToHost));
  if (d_out) std::copy(hd.begin(), hd.end(), d_out);
  if (u_out) GJ_CUDA(err, cudaMemcpy(u_out, P.ubuf.p, size_t(nsrc) * N * sizeof(double), cudaMemcpyDeviceToHost));
  if (grad) {
    std::vector<double> he(ndat);
    if (ndat) GJ_CUDA(err, cudaMemcpy(he.data(), P.ebuf.p, ndat * sizeof(double), cudaMemcpyDeviceToHost));
    if (e_out) std::copy(he.begin(), he.end(), e_out);
    if (misfit_out)  // 0.5 e'e per source (dc_E with identity weights)
      for (int s = 0; s < nsrc; ++s) {
        double a = 0;
        for (long j = P.off[s]; j < P.off[s + 1]; ++j) a += he[j] * he[j];
        misfit_out[s] = 0.5 * a;
      }
    std::vector<double> hg(size_t(nsrc) * N);
    GJ_CUDA(err, cudaMemcpy(hg.data(), P.gbuf.p, hg.size() * sizeof(double), cudaMemcpyDeviceToHost));
    // trim the Robin padding: g(1+robin:nx-robin, 1:nz-robin) (dc_gradient2_5d.m:161-162)
    const int n0 = gg.n - 2 * gg.robin, m0 = gg.m - gg.robin;
    const size_t per = size_t(n0) * m0;
    for (size_t i = 0; i < (o.per_source ? size_t(nsrc) : 1) * per; ++i) g_out[i] = 0;
    for (int s = 0; s < nsrc; ++s) {
      double* dst = g_out + (o.per_source ? size_t(s) * per : 0);
      for (int h = 0; h < m0; ++h)
        for (int l = 0; l < n0; ++l) dst[l + size_t(h) * n0] += hg[size_t(s) * N + (l + gg.robin) + size_t(h) * gg.n];
    }
  }
  return GJ_OK;
}

gj_status dc_run(Ctx& c, const gj_dc_grid& gg, const double* sigma, const gj_dc_src* srcs, int nsrc, bool grad,
                 const gj_dc_opts& o, double* d_out, double* e_out, double* u_out, double* g_out,
                 double* misfit_out, gj_dc_stats* stats, double* uk_out) {
  if (o.factor_fp32)
    return dc_run_t<float>(c, gg, sigma, srcs, nsrc, grad, o, d_out, e_out, u_out, g_out, misfit_out, stats, uk_out);
  return dc_run_t<double>(c, gg, sigma, srcs, nsrc, grad, o, d_out, e_out, u_out, g_out, misfit_out, stats, uk_out);
}

}  // namespace gj

// Radar (GPR) solver: device plan, forward, checkpointed gradient, w_grad.
//
// Host orchestration of the kernels in w_kernels.cuh.  One plan holds the
// padded grid, the coefficient arrays (built on the device from the model),
// the per-shot source/receiver tables, the A/B state buffers of the forward
// and adjoint fields, the checkpoints and the u-history ring.
#include <algorithm>
#include <array>
#include <cmath>
#include <cstring>
#include <map>

#include "gj_internal.h"
#include "w_kernels.cuh"
#include "w_kernels_vec.cuh"
#include "w_kernels_ring.cuh"
#include "w_tblock.cuh"
#include "w_tblock_plan.h"
#include "w_misfit.cuh"
#include "w_condition.cuh"
#include "w_band.cuh"

namespace gj {

static inline int round_up(int a, int b) { return (a + b - 1) / b * b; }

// Graded PML profiles (w_cpml.m:47-55, 70-78, 110-118, 151-159), 0-based rows/cols.
static void pml_profiles(const gj_w_grid& g, int NX, int NY, std::vector<double>& sex,
                         std::vector<double>& smx, std::vector<double>& sey,
                         std::vector<double>& smy) {
  const double P = g.pml, c = 1.0 / std::sqrt(g.mu0 * g.eps0);
  const double sx = -(g.order + 1) * g.eps0 * c * std::log(g.R0) / (2.0 * g.dx * g.pml);
  const double sy = -(g.order + 1) * g.eps0 * c * std::log(g.R0) / (2.0 * g.dy * g.pml);
  const double rm = g.mu0 / g.eps0;
  sex.assign(NX + 2, 0.0); smx.assign(NX + 2, 0.0); sey.assign(NY + 2, 0.0); smy.assign(NY + 2, 0.0);
  for (int I = 1; I <= g.pml_top; ++I) sex[I] = sx * std::pow((P - I + 0.25) / P, g.order);
  for (int I = 0; I <= g.pml_top - 1; ++I) smx[I] = rm * sx * std::pow((P - I - 0.25) / P, g.order);
  for (int I = NX - g.pml; I <= NX - 1; ++I) {
    const double k = I - (NX - g.pml) + 1;
    sex[I] = sx * std::pow((k - 0.75) / P, g.order);
    smx[I] = rm * sx * std::pow((k - 0.25) / P, g.order);
  }
  for (int J = 1; J <= g.pml; ++J) sey[J] = sy * std::pow((P - J + 0.25) / P, g.order);
  for (int J = 0; J <= g.pml - 1; ++J) smy[J] = rm * sy * std::pow((P - J - 0.25) / P, g.order);
  for (int J = NY - g.pml; J <= NY - 1; ++J) {
    const double k = J - (NY - g.pml) + 1;
    sey[J] = sy * std::pow((k - 0.75) / P, g.order);
    smy[J] = rm * sy * std::pow((k - 0.25) / P, g.order);
  }
}

template <class TM>
__global__ void k_cezj(const CoefBuild c, const TM* eps, const TM* sig, const int* si, const int* sj,
                       int nshots, void* out, int is_double) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nshots) return;
  double e = 1, sg = 0;
  pad_model(c, eps, sig, si[s], sj[s], e, sg);
  const double v = -(2 * c.dt) / (2 * e * c.eps0 + c.dt * sg);  // w_coeff.m:44-45
  if (is_double) static_cast<double*>(out)[s] = v;
  else static_cast<float*>(out)[s] = float(v);
}

// Residual e = d - d_obs and the two sums of the normalised L2 misfit
// (w_bozdag.m:14, w_E.m:15-16, w_update_e.m:75-76).
template <class T>
__global__ void k_residual(const T* d, const T* dobs, T* e, size_t per_shot, double* sums) {
  const int s = blockIdx.y;
  double num = 0, den = 0;
  const size_t base = size_t(s) * per_shot;
  for (size_t i = threadIdx.x + size_t(blockIdx.x) * blockDim.x; i < per_shot; i += size_t(blockDim.x) * gridDim.x) {
    const T r = d[base + i] - dobs[base + i];
    e[base + i] = r;
    num += double(r) * double(r);
    den += double(dobs[base + i]) * double(dobs[base + i]);
  }
  for (int o = 16; o > 0; o >>= 1) {
    num += __shfl_down_sync(0xffffffffu, num, o);
    den += __shfl_down_sync(0xffffffffu, den, o);
  }
  if ((threadIdx.x & 31) == 0) {
    atomicAdd(sums + 2 * s, num);
    atomicAdd(sums + 2 * s + 1, den);
  }
}

template <class TI, class TO>
__global__ void k_convert(const TI* in, TO* out, size_t n) {
  for (size_t i = threadIdx.x + size_t(blockIdx.x) * blockDim.x; i < n; i += size_t(blockDim.x) * gridDim.x)
    out[i] = TO(in[i]);
}

template <class T>
class WSolver : public WSolverBase {
 public:
  gj_w_grid g{};
  int NX = 0, NY = 0, ld = 0, nshots = 0, nr = 0;  // nr = max receivers per shot
  int hr0 = 0, hld = 0;  // rows of the domain-node layout (history, accumulators, rings)
  size_t fstride = 0, sstride = 0, mn = 0, dn = 0;  // dn: domain-node elements per shot (ld*n)
  WDev<T> w{};   // forward coefficients
  WDev<T> wr{};  // reference-adjoint coefficients (sigma -> -sigma in the interior)
  DevBuf coef, model_d, prof, shotbuf, recbuf, selbuf, nrsbuf, nselbuf, sibuf, sjbuf;
  DevBuf rsbuf;  // per shot nrr x {column, row, receiver}, sorted by column (ring kernels)
  DevBuf nosrc;  // per shot -1: steps without a source (the reference adjoint)
  DevBuf fwdA, fwdB, adjA, adjB, hist, ckpt, acc, dbuf, ebuf, dobsbuf, sums, scratch, stage, stage2, gout;
  std::vector<ShotHost> sh;
  std::vector<int> sh_src_i, sh_src_j;  // source nodes as given (Ez row, column)
  std::vector<int> nrs, nsel;
  // layout of shotbuf: src (long) | cezj (T) | wav (T, nshots*nt)
  long* d_src = nullptr; T* d_cezj = nullptr; T* d_wav = nullptr;
  double* eps_m = nullptr; double* sig_m = nullptr;
  size_t hist_slots = 0, n_ckpt = 0;
  int K = 0;
  // launch shape
  int bx = 128, tj = 16;
  // warp-task ring kernels (w_kernels_ring.cuh): threads per CTA (0 = not
  // available for T), ring stages, resident CTAs per SM, SMs; ring_on per call
  int ring_nth = 0, nsm = 148;
  bool ring_on = false;
  int Kd = 32;   // adjoint steps per imaging pass (slots of the l ring)
  DevBuf lring;
  // exact adjoint: PML band history, adjoint band ring and band accumulators (w_band.cuh)
  bool band_on = false;
  DevBuf bhist, blam, bacc;
  DevBuf nanbuf;  // non-finite counters of the results (GJ_ENUMERIC)

  // Queues a count of the non-finite values of x[0, n) into counter q.
  gj_status count_nonfinite_async(Err& err, const void* x, size_t n, bool dbl, int q, cudaStream_t st) {
    GJ_TRY(nanbuf.alloc(err, 4 * sizeof(unsigned)));
    unsigned* c = nanbuf.as<unsigned>() + q;
    GJ_CUDA(err, cudaMemsetAsync(c, 0, sizeof(unsigned), st));
    const int nb = int(std::min<size_t>((n + 255) / 256, 1024));
    if (n == 0) return GJ_OK;
    if (dbl) k_count_nonfinite<double><<<nb, 256, 0, st>>>(static_cast<const double*>(x), n, c);
    else k_count_nonfinite<float><<<nb, 256, 0, st>>>(static_cast<const float*>(x), n, c);
    GJ_CUDA(err, cudaGetLastError());
    return GJ_OK;
  }


  static std::string key(const gj_w_grid& g, const gj_w_shot* shots, int nshots) {
    std::string k((const char*)&g, sizeof g);
    k.append((const char*)&nshots, sizeof nshots);
    for (int s = 0; s < nshots; ++s) {
      k.append((const char*)&shots[s].src_i, 2 * sizeof(int));
      k.append((const char*)&shots[s].nr, sizeof(int));
      k.append((const char*)shots[s].rec, sizeof(long) * size_t(shots[s].nr));
      k.append((const char*)shots[s].wavelet, sizeof(double) * size_t(g.nt));
    }
    return k;
  }

  gj_status setup(Err& err, const gj_w_grid& gg, const gj_w_shot* shots, int ns) {
    g = gg;
    if (g.m < 3 || g.n < 3 || g.pml < 1 || g.nt < 3)
      return err.set(GJ_EINVAL, "grid too small: need m, n >= 3, pml >= 1, nt >= 3");
    if (!(g.pml_top == 0 || g.pml_top == g.pml))
      return err.set(GJ_EINVAL, "pml_top must be 0 (free top) or equal to pml");
    if (g.air < 0 || (g.pml_top == 0 && g.air < 1))
      return err.set(GJ_EINVAL, "air must be >= 0, and >= 1 with a free top");
    if (!(g.dx > 0 && g.dy > 0 && g.dt > 0 && g.eps0 > 0 && g.mu0 > 0 && g.R0 > 0 && g.R0 < 1))
      return err.set(GJ_EINVAL, "dx, dy, dt, eps0, mu0 must be positive and 0 < R0 < 1");
    if (ns < 1 || !shots) return err.set(GJ_EINVAL, "need at least one shot");
    NX = g.pml_top + g.air + g.m + g.pml;
    NY = g.n + 2 * g.pml;
    ld = round_up(NX + 2, 32);
    fstride = size_t(ld) * size_t(NY + 3);
    sstride = size_t(NFIELDS) * fstride;
    mn = size_t(g.m) * size_t(g.n);
    hr0 = (g.pml_top + g.air) / 4 * 4;
    hld = (g.pml_top + g.air + g.m + 3) / 4 * 4 - hr0;
    dn = size_t(hld) * size_t(g.n);
    nshots = ns;
    nr = 0;
    max_rec_row = -1;
    sh.assign(ns, ShotHost{});
    sh_src_i.assign(ns, 0);
    sh_src_j.assign(ns, 0);
    nrs.assign(ns, 0);
    nsel.assign(ns, 0);
    for (int s = 0; s < ns; ++s) {
      const gj_w_shot& q = shots[s];
      if (!q.wavelet) return err.set(GJ_EINVAL, "shot %d: null wavelet", s);
      if (q.nr < 0 || (q.nr > 0 && !q.rec)) return err.set(GJ_EINVAL, "shot %d: bad receivers", s);
      if (q.src_i < 1 || q.src_i > NX - 1 || q.src_j < 1 || q.src_j > NY - 1)
        return err.set(GJ_EINVAL, "shot %d: source (%d,%d) must be an updated Ez node, 1..NX-1 x 1..NY-1", s,
                       q.src_i, q.src_j);
      const bool interior = q.src_i >= g.pml_top + 1 && q.src_i <= NX - g.pml - 1 &&
                            q.src_j >= g.pml + 1 && q.src_j <= NY - g.pml - 1;
      // A source in the PML band is overwritten by new_Ez_pml (w_solve.m:92-94): no effect.
      sh[s].src = interior ? long(q.src_i) + long(q.src_j) * ld : -1;
      sh[s].wav.assign(q.wavelet, q.wavelet + g.nt);
      sh[s].rec.resize(q.nr);
      std::map<long, int> last;
      for (int r = 0; r < q.nr; ++r) {
        const long L = q.rec[r];
        if (L < 0 || L >= long(NX + 1) * long(NY + 1))
          return err.set(GJ_EINVAL, "shot %d receiver %d: node %ld outside the (NX+1)x(NY+1) grid", s, r, L);
        const long i = L % (NX + 1), j = L / (NX + 1);
        sh[s].rec[r] = i + j * ld;
        last[sh[s].rec[r]] = r;
        max_rec_row = std::max(max_rec_row, int(i));
      }
      for (int r = 0; r < q.nr; ++r)
        if (last[sh[s].rec[r]] == r) sh[s].sel.push_back(r);
      nrs[s] = q.nr;
      nsel[s] = int(sh[s].sel.size());
      nr = std::max(nr, q.nr);
    }
    // device geometry
    w.NX = NX; w.NY = NY; w.ld = ld; w.P = g.pml; w.Pt = g.pml_top; w.m = g.m; w.n = g.n;
    w.di0 = g.pml_top + g.air; w.dj0 = g.pml;
    w.hr0 = hr0; w.hld = hld;
    w.ei0 = g.pml_top + 1; w.ei1 = NX - g.pml - 1; w.ej0 = g.pml + 1; w.ej1 = NY - g.pml - 1;
    w.hyi0 = g.pml_top; w.hyi1 = NX - g.pml - 1; w.hxj0 = g.pml; w.hxj1 = NY - g.pml - 1;
    w.chxez = T(-(2 * g.dt / g.dy) / (2 * g.mu0));
    w.chyez = T((2 * g.dt / g.dx) / (2 * g.mu0));
    w.rxy = T(-g.dx / g.dy);
    band_geometry(w);
    // coefficient arrays: 12 node arrays
    GJ_TRY(coef.alloc(err, 12 * fstride * sizeof(T)));
    GJ_CUDA(err, cudaMemset(coef.p, 0, 12 * fstride * sizeof(T)));
    T* cb = coef.as<T>() + ld;  // base one column in
    T* arr[12];
    for (int q = 0; q < 12; ++q) arr[q] = cb + q * fstride;
    w.ce = arr[0]; w.chy = arr[1]; w.ax = arr[2]; w.bx = arr[3]; w.ay = arr[4]; w.by = arr[5];
    w.hxa = arr[6]; w.hxb = arr[7]; w.hya = arr[8]; w.hyb = arr[9];
    wr = w;
    wr.ce = arr[10]; wr.chy = arr[11];
    GJ_TRY(model_d.alloc(err, 2 * mn * sizeof(double)));
    eps_m = model_d.as<double>(); sig_m = eps_m + mn;
    // PML profiles
    std::vector<double> sex, smx, sey, smy;
    pml_profiles(g, NX, NY, sex, smx, sey, smy);
    GJ_TRY(prof.alloc(err, (2 * (NX + 2) + 2 * (NY + 2)) * sizeof(double)));
    double* pp = prof.as<double>();
    GJ_CUDA(err, cudaMemcpy(pp, sex.data(), (NX + 2) * sizeof(double), cudaMemcpyHostToDevice));
    GJ_CUDA(err, cudaMemcpy(pp + NX + 2, smx.data(), (NX + 2) * sizeof(double), cudaMemcpyHostToDevice));
    GJ_CUDA(err, cudaMemcpy(pp + 2 * (NX + 2), sey.data(), (NY + 2) * sizeof(double), cudaMemcpyHostToDevice));
    GJ_CUDA(err, cudaMemcpy(pp + 2 * (NX + 2) + NY + 2, smy.data(), (NY + 2) * sizeof(double), cudaMemcpyHostToDevice));
    // shot tables
    const size_t sb = ns * sizeof(long) + ns * sizeof(T) + size_t(ns) * g.nt * sizeof(T) + 64;
    GJ_TRY(shotbuf.alloc(err, sb));
    d_src = shotbuf.as<long>();
    d_cezj = reinterpret_cast<T*>(d_src + ns);
    d_wav = d_cezj + ns;
    std::vector<long> hsrc(ns);
    std::vector<T> hwav(size_t(ns) * g.nt);
    std::vector<int> hsi(ns), hsj(ns);
    for (int s = 0; s < ns; ++s) {
      hsrc[s] = sh[s].src;
      hsi[s] = shots[s].src_i; hsj[s] = shots[s].src_j;
      sh_src_i[s] = shots[s].src_i; sh_src_j[s] = shots[s].src_j;
      for (int t = 0; t < g.nt; ++t) hwav[size_t(s) * g.nt + t] = T(sh[s].wav[t]);
    }
    GJ_CUDA(err, cudaMemcpy(d_src, hsrc.data(), ns * sizeof(long), cudaMemcpyHostToDevice));
    GJ_CUDA(err, cudaMemcpy(d_wav, hwav.data(), hwav.size() * sizeof(T), cudaMemcpyHostToDevice));
    GJ_TRY(sibuf.alloc(err, ns * sizeof(int)));
    GJ_TRY(sjbuf.alloc(err, ns * sizeof(int)));
    GJ_CUDA(err, cudaMemcpy(sibuf.p, hsi.data(), ns * sizeof(int), cudaMemcpyHostToDevice));
    GJ_CUDA(err, cudaMemcpy(sjbuf.p, hsj.data(), ns * sizeof(int), cudaMemcpyHostToDevice));
    const int nrr = std::max(nr, 1);
    std::vector<long> hrec(size_t(ns) * nrr, 0);
    std::vector<int> hsel(size_t(ns) * nrr, 0);
    for (int s = 0; s < ns; ++s) {
      for (int r = 0; r < nrs[s]; ++r) hrec[size_t(s) * nrr + r] = sh[s].rec[r];
      for (int q = 0; q < nsel[s]; ++q) hsel[size_t(s) * nrr + q] = sh[s].sel[q];
    }
    GJ_TRY(recbuf.alloc(err, hrec.size() * sizeof(long)));
    GJ_TRY(selbuf.alloc(err, hsel.size() * sizeof(int)));
    GJ_TRY(nrsbuf.alloc(err, ns * sizeof(int)));
    GJ_TRY(nselbuf.alloc(err, ns * sizeof(int)));
    GJ_CUDA(err, cudaMemcpy(recbuf.p, hrec.data(), hrec.size() * sizeof(long), cudaMemcpyHostToDevice));
    GJ_CUDA(err, cudaMemcpy(selbuf.p, hsel.data(), hsel.size() * sizeof(int), cudaMemcpyHostToDevice));
    GJ_CUDA(err, cudaMemcpy(nrsbuf.p, nrs.data(), ns * sizeof(int), cudaMemcpyHostToDevice));
    GJ_CUDA(err, cudaMemcpy(nselbuf.p, nsel.data(), ns * sizeof(int), cudaMemcpyHostToDevice));
    {
      std::vector<int> hrs(size_t(ns) * nrr * 3, 0);
      for (int s = 0; s < ns; ++s) {
        std::vector<std::array<int, 3>> v(nrs[s]);
        for (int r = 0; r < nrs[s]; ++r) {
          const long kk = sh[s].rec[r];
          v[r] = {int(kk / ld), int(kk % ld), r};
        }
        std::sort(v.begin(), v.end());
        for (int r = 0; r < nrs[s]; ++r)
          for (int q = 0; q < 3; ++q) hrs[(size_t(s) * nrr + r) * 3 + q] = v[r][q];
      }
      GJ_TRY(rsbuf.alloc(err, hrs.size() * sizeof(int)));
      GJ_CUDA(err, cudaMemcpy(rsbuf.p, hrs.data(), hrs.size() * sizeof(int), cudaMemcpyHostToDevice));
      std::vector<long> hns(ns, -1);
      GJ_TRY(nosrc.alloc(err, ns * sizeof(long)));
      GJ_CUDA(err, cudaMemcpy(nosrc.p, hns.data(), ns * sizeof(long), cudaMemcpyHostToDevice));
    }
    // traces
    GJ_TRY(dbuf.alloc(err, size_t(ns) * nrr * g.nt * sizeof(T)));
    GJ_TRY(ebuf.alloc(err, size_t(ns) * nrr * g.nt * sizeof(T)));
    GJ_TRY(dobsbuf.alloc(err, size_t(ns) * nrr * g.nt * sizeof(T)));
    GJ_TRY(sums.alloc(err, 2 * ns * sizeof(double)));
    GJ_TRY(fwdA.alloc(err, size_t(ns) * sstride * sizeof(T)));
    GJ_TRY(fwdB.alloc(err, size_t(ns) * sstride * sizeof(T)));
    // launch shape: 128 rows per block; columns per block sized for >= ~4 waves
    bx = 128;
    const long blocks_per_col = (ld + bx - 1) / bx;
    tj = 64;
    while (tj > 4 && blocks_per_col * ((NY + tj) / tj) * ns < 148L * 16) tj /= 2;
    GJ_TRY(ring_setup(err));
    ring_on = ring_nth > 0;
    return GJ_OK;
  }

  // Launch shape of the warp-task ring kernels (w_kernels_ring.cuh).  Each
  // step launches the fast-only kernel (interior blocks x interior columns) on
  // the calling stream and the general kernel (the rest) on a forked side
  // stream.  RingCfg holds the knobs: ring stages of the general (S) and fast
  // (SF) kernels, warps per CTA of the general kernel (RWG; the fast one has
  // RW), and the column chunk of a fast (tjF) and a general (tjS) warp task.
  // The autotuner (autotune) times candidate configurations on the plan's own
  // grid at the launch size and keeps the fastest per launch size; the
  // GJ_RING_* environment variables fix a configuration instead.
  static constexpr int RW = 4;
  struct RingCfg {
    int S = 2, SF = 3, RWG = 2, tjF = 32, tjS = 8;
    bool operator==(const RingCfg& o) const {
      return S == o.S && SF == o.SF && RWG == o.RWG && tjF == o.tjF && tjS == o.tjS;
    }
  };
  RingCfg rc;                    // configuration of the forward launches being enqueued
  RingCfg rca;                   // and of the exact-adjoint launches
  bool light_tune = false;       // batch plans: a smaller candidate set
  const bool no_split = getenv("GJ_NO_SPLIT") != nullptr;  // one shot per general task everywhere
  int max_rec_row = -1;          // largest receiver row over all shots (split tasks hold none)
  RingCfg rc_env;                // default, with the environment's overrides
  bool env_fixed = false;        // a GJ_RING_* variable is set: no tuning
  std::map<int, std::pair<RingCfg, RingCfg>> tuned;  // (forward, adjoint) per launch size
  int maxsm_dyn = 0;
  const bool ring_serial = getenv("GJ_RING_SERIAL") != nullptr;
  int last_kernels = 0;  // kernels launched by the last launch_fwd / launch_adjr
  cudaStream_t side = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  template <int S, bool F>
  gj_status ring_attr(Err& err) {
    const size_t sm = ring_smem(RW, S, F);  // the largest CTA of either kernel
    if (sm > size_t(maxsm_dyn)) return GJ_OK;
    GJ_CUDA(err, cudaFuncSetAttribute(k_fwdw<T, S, F>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(sm)));
    GJ_CUDA(err, cudaFuncSetAttribute(k_adjw<T, S, F>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(sm)));
    return GJ_OK;
  }
  gj_status ring_setup(Err& err) {
    ring_nth = 0;
    tasks.clear();
    tuned.clear();
    tb_tiles.clear();
    tb_tuned.clear();
    if constexpr (VT<T>::V * sizeof(T) == 16) {
      int dev = 0;
      GJ_CUDA(err, cudaGetDevice(&dev));
      GJ_CUDA(err, cudaDeviceGetAttribute(&maxsm_dyn, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
      GJ_CUDA(err, cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
      RingCfg d;
      auto env = [&](const char* k, int& v, int lo, int hi) {
        if (const char* e = getenv(k)) { v = std::min(std::max(atoi(e), lo), hi); env_fixed = true; }
      };
      env("GJ_RING_CTA_WARPS", d.RWG, 1, 4);
      env("GJ_RING_STAGES", d.S, 2, 4);
      env("GJ_RING_STAGES_FAST", d.SF, 2, 4);
      env("GJ_RING_TJF", d.tjF, 2, 1 << 20);
      env("GJ_RING_TJS", d.tjS, 2, 1 << 20);
      if (const char* e = getenv("GJ_AUTOTUNE")) env_fixed = env_fixed || atoi(e) == 0;
      if (ring_smem(RW, 2, false) > size_t(maxsm_dyn)) return GJ_OK;
      while (d.S > 2 && ring_smem(RW, d.S, false) > size_t(maxsm_dyn)) --d.S;
      GJ_TRY((ring_attr<2, false>(err))); GJ_TRY((ring_attr<3, false>(err))); GJ_TRY((ring_attr<4, false>(err)));
      GJ_TRY((ring_attr<2, true>(err))); GJ_TRY((ring_attr<3, true>(err))); GJ_TRY((ring_attr<4, true>(err)));
      rc_env = d;
      rc = d;
      rca = d;
      // the general kernel (PML band) sets the step time: its stream gets the
      // highest priority so its CTAs are dispatched before the fast kernel's
      // (graphs honour the captured priority, cudaGraphInstantiateFlagUseNodePriority)
      if (!side) {
        int lo = 0, hi = 0;
        GJ_CUDA(err, cudaDeviceGetStreamPriorityRange(&lo, &hi));
        const char* e = getenv("GJ_SIDE_PRIORITY");
        const bool prio = !(e && atoi(e) == 0);
        GJ_CUDA(err, cudaStreamCreateWithPriority(&side, cudaStreamNonBlocking, prio ? hi : lo));
      }
      if (!ev_fork) GJ_CUDA(err, cudaEventCreateWithFlags(&ev_fork, cudaEventDisableTiming));
      if (!ev_join) GJ_CUDA(err, cudaEventCreateWithFlags(&ev_join, cudaEventDisableTiming));
      ring_nth = 32 * RW;
      if (const char* e = getenv("GJ_IMAGE_WINDOW")) Kd = std::min(std::max(atoi(e), 1), 256);
    }
    return GJ_OK;
  }
  // The configuration for launches of gn shots: the tuned one when there is.
  void select_cfg(int gn) {
    auto it = tuned.find(gn);
    rc = it != tuned.end() ? it->second.first : rc_env;
    rca = it != tuned.end() ? it->second.second : rc_env;
  }
  // Fast rows of the ring kernels: interior Ez rows (plus the free-top Ez = 0
  // row, whose Ceze/Cezhy are 1/0) that are also Hy interior rows.
  bool fast_row(int I) const {
    const bool e = (I >= w.ei0 && I <= w.ei1) || (I == 0 && g.pml_top == 0);
    return e && I >= w.hyi0 && I <= w.hyi1;
  }
  bool interior_row(int I) const { return I >= w.ei0 && I <= w.ei1 && I >= w.hyi0 && I <= w.hyi1; }
  // Task tables for launches of gn shots (built outside graph capture):
  // [0] forward fast, [1] forward general, [2] adjoint fast, [3] adjoint general.
  struct TaskTable { DevBuf buf[4]; int n[4] = {0, 0, 0, 0}; };
  std::map<long, std::unique_ptr<TaskTable>> tasks;
  static long task_key(int gn, const RingCfg& q) { return (long(gn) << 40) | (long(q.tjF) << 20) | long(q.tjS); }
  const TaskTable& task_table(int gn, const RingCfg& q) const { return *tasks.at(task_key(gn, q)); }
  // Task tables of launches of gn shots for the column chunks of rc and rca.
  gj_status prepare_tasks(Err& err, int gn) {
    GJ_TRY(prepare_tasks_for(err, gn, rc));
    return prepare_tasks_for(err, gn, rca);
  }
  gj_status prepare_tasks_for(Err& err, int gn, const RingCfg& q) {
    if (ring_nth == 0 || tasks.count(task_key(gn, q))) return GJ_OK;
    constexpr int V = VT<T>::V;
    const int rows = 32 * V, nrb = (NX + 1 + rows - 1) / rows;
    std::vector<int> fast(nrb, 0);
    int nF = 0;
    for (int rb = 0; rb < nrb; ++rb) {
      const int r0 = rb * rows;
      bool f = (r0 == 0 || interior_row(r0 - 1)) && interior_row(r0 + rows);
      for (int I = r0; f && I < r0 + rows; ++I) f = fast_row(I);
      fast[rb] = f ? 1 : 0;
      nF += fast[rb];
    }
    const int tjS = q.tjS;
    auto tt = std::make_unique<TaskTable>();
    for (int dir = 0; dir < 2; ++dir) {
      const int c0 = w.ej0, c1 = dir == 0 ? w.ej1 : w.ej1 - 1;  // fast columns
      const int ncol = std::max(c1 - c0 + 1, 0);
      const int tjF = std::min(q.tjF, std::max(ncol, 1));
      std::vector<int4> hf, hg;
      // task word: (shot << 2) | (split << 1) | fast
      auto chunks = [&](std::vector<int4>& h, int z, int r0, int a0, int a1, int tj, int split) {
        for (int j0 = a0; j0 <= a1; j0 += tj)
          h.push_back(make_int4(r0, j0, std::min(j0 + tj - 1, a1), (z << 2) | (split << 1)));
      };
      // Split general tasks: a block whose live rows fit 16 lanes (r0 + 16 V > NX)
      // runs two shots per warp, when no receiver of any shot lies in its rows
      // (split tasks skip the fused receiver record and injection).
      auto splittable = [&](int rb) {
        const int r0 = rb * rows;
        return !no_split && !fast[rb] && r0 + 16 * V > NX && max_rec_row < r0;
      };
      for (int z = 0; z < gn; ++z)
        for (int rb = 0; rb < nrb; ++rb) {
          const int r0 = rb * rows;
          if (fast[rb] && ncol > 0) {
            chunks(hf, z, r0, c0, c1, tjF, 0);
            if (c0 > 0) chunks(hg, z, r0, 0, c0 - 1, tjS, 0);
            if (c1 < NY) chunks(hg, z, r0, c1 + 1, NY, tjS, 0);
          } else if (!splittable(rb)) {
            chunks(hg, z, r0, 0, NY, tjS, 0);
          } else if (z % 2 == 0) {
            chunks(hg, z, r0, 0, NY, tjS, z + 1 < gn ? 1 : 0);
          }
        }
      for (auto& q : hf) q.w |= 1;
      std::vector<int4>* hh[2] = {&hf, &hg};
      for (int k = 0; k < 2; ++k) {
        const int slot = 2 * dir + k;
        tt->n[slot] = int(hh[k]->size());
        if (tt->n[slot] == 0) continue;
        GJ_TRY(tt->buf[slot].alloc(err, hh[k]->size() * sizeof(int4)));
        GJ_CUDA(err, cudaMemcpy(tt->buf[slot].p, hh[k]->data(), hh[k]->size() * sizeof(int4),
                                cudaMemcpyHostToDevice));
      }
    }
    tasks.emplace(task_key(gn, q), std::move(tt));
    return GJ_OK;
  }

  // Launches the fast-only kernel on st and the general kernel on the side
  // stream, joined back into st.
  template <class Args, class LF, class LG>
  gj_status fork_join(Err& err, const TaskTable& tt, int dir, cudaStream_t st, LF launch_fast, LG launch_gen) {
    const int nf = tt.n[2 * dir], ng = tt.n[2 * dir + 1];
    const int4* tf = static_cast<const int4*>(tt.buf[2 * dir].p);
    const int4* tg = static_cast<const int4*>(tt.buf[2 * dir + 1].p);
    last_kernels = (nf > 0) + (ng > 0);
    if (ring_serial) {  // both kernels on st, one after the other (for timing each)
      if (ng > 0) launch_gen(tg, ng, st);
      if (nf > 0) launch_fast(tf, nf, st);
      return GJ_OK;
    }
    if (ng > 0) {
      GJ_CUDA(err, cudaEventRecord(ev_fork, st));
      GJ_CUDA(err, cudaStreamWaitEvent(side, ev_fork, 0));
      launch_gen(tg, ng, side);
      GJ_CUDA(err, cudaEventRecord(ev_join, side));
    }
    if (nf > 0) launch_fast(tf, nf, st);
    if (ng > 0) GJ_CUDA(err, cudaStreamWaitEvent(st, ev_join, 0));
    return GJ_OK;
  }

  // One forward step of gn shots (A -> B).
  RecArgs<T> rec_args(int g0) const {
    RecArgs<T> r{};
    const int nrr = std::max(nr, 1);
    r.rs = rsbuf.as<int>() + size_t(g0) * nrr * 3;
    r.nrs = nrsbuf.as<int>() + g0;
    r.nrr = nrr;
    r.nt = g.nt;
    r.d = nullptr; r.it = 0; r.e = nullptr; r.kinj = -1;
    return r;
  }
  gj_status launch_fwd(Err& err, StepArgs<T> a, int gn, cudaStream_t st, RecArgs<T> ra = RecArgs<T>{},
                       const WDev<T>* wsel = nullptr) {
    if constexpr (VT<T>::V * sizeof(T) == 16) {
      if (ring_on) {
        const TaskTable& tt = task_table(gn, rc);
        const WDev<T> wd = wsel ? *wsel : w;
        const int S = rc.S, SF = rc.SF;
        auto lf = [&](const int4* tk, int n, cudaStream_t s_) {
          const dim3 grd((n + RW - 1) / RW);
          const size_t sm = ring_smem(RW, SF, true);
          if (SF == 2) k_fwdw<T, 2, true><<<grd, 32 * RW, sm, s_>>>(wd, a, tk, n, ra);
          else if (SF == 3) k_fwdw<T, 3, true><<<grd, 32 * RW, sm, s_>>>(wd, a, tk, n, ra);
          else k_fwdw<T, 4, true><<<grd, 32 * RW, sm, s_>>>(wd, a, tk, n, ra);
        };
        const int rw = rc.RWG;
        auto lg = [&](const int4* tk, int n, cudaStream_t s_) {
          const dim3 grd((n + rw - 1) / rw);
          const size_t sm = ring_smem(rw, S, false);
          if (S == 2) k_fwdw<T, 2, false><<<grd, 32 * rw, sm, s_>>>(wd, a, tk, n, ra);
          else if (S == 3) k_fwdw<T, 3, false><<<grd, 32 * rw, sm, s_>>>(wd, a, tk, n, ra);
          else k_fwdw<T, 4, false><<<grd, 32 * rw, sm, s_>>>(wd, a, tk, n, ra);
        };
        return fork_join<StepArgs<T>>(err, tt, 0, st, lf, lg);
      }
    }
    constexpr int V = VT<T>::V;
    a.tj = tj_for(gn);
    const dim3 grd((NX + 1 + 128 * V - 1) / (128 * V), (NY + 1 + a.tj - 1) / a.tj, gn);
    k_stepv<T, 0><<<grd, 128, 0, st>>>(w, a);
    last_kernels = 1;
    return GJ_OK;
  }
  // One exact adjoint step of gn shots with the l ring (ring kernels only).
  gj_status launch_adjr(Err& err, AdjRingArgs<T> a, int gn, cudaStream_t st, RecArgs<T> ra) {
    if constexpr (VT<T>::V * sizeof(T) == 16) {
      const TaskTable& tt = task_table(gn, rca);
      const WDev<T> wd = w;
      const int S = rca.S, SF = rca.SF;
      auto lf = [&](const int4* tk, int n, cudaStream_t s_) {
        const dim3 grd((n + RW - 1) / RW);
        const size_t sm = ring_smem(RW, SF, true);
        if (SF == 2) k_adjw<T, 2, true><<<grd, 32 * RW, sm, s_>>>(wd, a, tk, n, ra);
        else if (SF == 3) k_adjw<T, 3, true><<<grd, 32 * RW, sm, s_>>>(wd, a, tk, n, ra);
        else k_adjw<T, 4, true><<<grd, 32 * RW, sm, s_>>>(wd, a, tk, n, ra);
      };
      const int rw = rca.RWG;
      auto lg = [&](const int4* tk, int n, cudaStream_t s_) {
        const dim3 grd((n + rw - 1) / rw);
        const size_t sm = ring_smem(rw, S, false);
        if (S == 2) k_adjw<T, 2, false><<<grd, 32 * rw, sm, s_>>>(wd, a, tk, n, ra);
        else if (S == 3) k_adjw<T, 3, false><<<grd, 32 * rw, sm, s_>>>(wd, a, tk, n, ra);
        else k_adjw<T, 4, false><<<grd, 32 * rw, sm, s_>>>(wd, a, tk, n, ra);
      };
      return fork_join<AdjRingArgs<T>>(err, tt, 1, st, lf, lg);
    }
    return GJ_OK;
  }

  // Autotuner: times candidate ring configurations for launches of gn shots
  // on this grid (forward + exact-adjoint steps of zeroed states with the
  // work of a real step: history and band-history writes, receiver record,
  // adjoint-source injection, adjoint-field and band rings) and keeps the
  // fastest for gn.  Coordinate search: the fast kernel's
  // stages x column chunk first, then the general kernel's stages x column
  // chunk x CTA width.  Needs the states and the adjoint-field ring of the
  // memory plan allocated for at least gn shots.
  gj_status autotune(Err& err, int gn, cudaStream_t st) {
    if (ring_nth == 0 || gn < 1) return GJ_OK;
    if (env_fixed || tuned.count(gn)) { select_cfg(gn); return prepare_tasks(err, gn); }
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    GJ_CUDA(err, cudaEventCreate(&e0));
    GJ_CUDA(err, cudaEventCreate(&e1));
    struct EvGuard { cudaEvent_t a, b; ~EvGuard() { cudaEventDestroy(a); cudaEventDestroy(b); } } guard{e0, e1};
    const int reps = 10, trials = 3;
    const bool adj_ok = lring.p != nullptr;
    // history and band slots rotate over the buffers (strided), so their
    // writes reach DRAM as in a real step instead of one L2-resident slot
    const size_t nslot = hist_slots > 1 ? hist_slots : 1;
    auto slot_of = [&](int i) { return nslot > 1 ? 1 + (size_t(i) * 97) % (nslot - 1) : size_t(0); };
    auto clear = [&]() -> gj_status {
      GJ_CUDA(err, cudaMemsetAsync(fwdA.p, 0, size_t(gn) * sstride * sizeof(T), st));
      GJ_CUDA(err, cudaMemsetAsync(fwdB.p, 0, size_t(gn) * sstride * sizeof(T), st));
      if (adj_ok) {
        GJ_CUDA(err, cudaMemsetAsync(adjA.p, 0, size_t(gn) * sstride * sizeof(T), st));
        GJ_CUDA(err, cudaMemsetAsync(adjB.p, 0, size_t(gn) * sstride * sizeof(T), st));
      }
      return GJ_OK;
    };
    // dir 0: forward steps with cfg as rc; dir 1: adjoint steps with cfg as rca
    auto time_cfg = [&](int dir, const RingCfg& cfg, float& ms) -> gj_status {
      if (dir == 0) rc = cfg; else rca = cfg;
      GJ_TRY(prepare_tasks_for(err, gn, cfg));
      GJ_TRY(clear());
      T* A = (dir == 0 ? fwdA : adjA).template as<T>() + ld;
      T* B = (dir == 0 ? fwdB : adjB).template as<T>() + ld;
      auto run = [&](int n, cudaStream_t rs) -> gj_status {
        for (int i = 0; i < n; ++i) {
          if (dir == 0) {
            StepArgs<T> a = step_args(A, B, i % g.nt);
            if (hist.p && nslot > 1) { a.hist = hist.as<T>() + slot_of(i) * gn * dn; a.hstride = dn; }
            if (band_on && bhist.p && nslot > 1) a.band = bhist.as<T>() + slot_of(i) * gn * size_t(w.bsz);
            RecArgs<T> ra = rec_args(0);
            if (nr > 0) { ra.d = dbuf.as<T>(); ra.it = i % g.nt; }
            GJ_TRY(launch_fwd(err, a, gn, rs, ra));
          } else {
            AdjRingArgs<T> b{};
            b.A = A; b.B = B; b.fstride = fstride; b.sstride = sstride; b.shot0 = 0;
            b.lout = lring.as<T>() + size_t(i % Kd) * gn * dn; b.hstride = dn;
            if (band_on && blam.p) b.band = blam.as<T>() + size_t(i % Kd) * gn * size_t(w.bsz);
            RecArgs<T> rb = rec_args(0);
            if (nr > 0) { rb.e = ebuf.as<T>(); rb.kinj = i % g.nt; }
            GJ_TRY(launch_adjr(err, b, gn, rs, rb));
          }
          std::swap(A, B);
        }
        return GJ_OK;
      };
      // The steps run as the solver runs them: captured into a CUDA graph
      // (node priorities kept) and replayed.  Launched one by one from a
      // stream instead, configurations with larger general-kernel CTAs timed
      // about as fast as the best and then ran twice as long inside graphs.
      cudaStream_t cs = nullptr;
      GJ_CUDA(err, cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
      GJ_CUDA(err, cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
      gj_status rs = run(reps, cs);
      cudaGraph_t gr = nullptr;
      cudaError_t ce = cudaStreamEndCapture(cs, &gr);
      cudaStreamDestroy(cs);
      if (rs != GJ_OK) { if (gr) cudaGraphDestroy(gr); return rs; }
      if (ce != cudaSuccess) return err.set(GJ_ECUDA, "tuning graph capture failed: %s", cudaGetErrorString(ce));
      cudaGraphExec_t ex = nullptr;
      ce = cudaGraphInstantiate(&ex, gr, cudaGraphInstantiateFlagUseNodePriority);
      cudaGraphDestroy(gr);
      if (ce != cudaSuccess) return err.set(GJ_ECUDA, "tuning graph instantiate failed: %s", cudaGetErrorString(ce));
      struct ExecGuard { cudaGraphExec_t e; ~ExecGuard() { cudaGraphExecDestroy(e); } } eg{ex};
      GJ_CUDA(err, cudaGraphLaunch(ex, st));  // warm-up replay
      // the least of a few timed replays (others' launches and clock changes
      // only ever add time)
      ms = 0.f;
      for (int trial = 0; trial < trials; ++trial) {
        GJ_CUDA(err, cudaEventRecord(e0, st));
        GJ_CUDA(err, cudaGraphLaunch(ex, st));
        GJ_CUDA(err, cudaEventRecord(e1, st));
        GJ_CUDA(err, cudaEventSynchronize(e1));
        float t = 0.f;
        GJ_CUDA(err, cudaEventElapsedTime(&t, e0, e1));
        ms = trial ? std::min(ms, t) : t;
      }
      GJ_CUDA(err, cudaGetLastError());
      return GJ_OK;
    };
    const std::vector<int> SFs = light_tune ? std::vector<int>{2, 3} : std::vector<int>{2, 3, 4};
    // small launches (few shots) need short column chunks to spread over the SMs
    const bool small = long(gn) * ((NX + 1 + 127) / 128) * ((NY + 31) / 32) < 8L * nsm;
    std::vector<int> tjFs = light_tune ? std::vector<int>{16, 32} : std::vector<int>{16, 24, 32, 48};
    const std::vector<int> Ss = light_tune ? std::vector<int>{2} : std::vector<int>{2, 3};
    // the general kernel runs in about one wave, its time about proportional
    // to the column chunk of a task: short chunks first
    const std::vector<int> tjSs = light_tune ? std::vector<int>{4, 8, 16} : std::vector<int>{4, 6, 8, 12, 16, 32};
    if (small) tjFs.insert(tjFs.begin(), 8);
    const std::vector<int> rws = {2, 4};
    RingCfg best[2] = {rc_env, rc_env};
    float tb[2] = {0.f, 0.f};
    const char* vb = getenv("GJ_AUTOTUNE_VERBOSE");
    const bool every = vb && atoi(vb) >= 2;  // print every candidate's time
    auto show = [&](int dir, const RingCfg& q, float t) {
      if (every)
        fprintf(stderr, "gerjoii_b200 autotune candidate %s S=%d SF=%d RWG=%d tjF=%d tjS=%d %.2f us/step\n",
                dir ? "adjoint" : "forward", q.S, q.SF, q.RWG, q.tjF, q.tjS, 1e3f * t / reps);
    };
    for (int dir = 0; dir < (adj_ok ? 2 : 1); ++dir) {
      if (dir == 0) GJ_TRY(time_cfg(dir, best[dir], tb[dir]));  // clocks up before the first timing
      GJ_TRY(time_cfg(dir, best[dir], tb[dir]));
      show(dir, best[dir], tb[dir]);
      auto consider = [&](const RingCfg& q) -> gj_status {
        if (q == best[dir]) return GJ_OK;
        if (ring_smem(q.RWG, q.S, false) > size_t(maxsm_dyn) || ring_smem(RW, q.SF, true) > size_t(maxsm_dyn))
          return GJ_OK;
        float t = 0.f;
        GJ_TRY(time_cfg(dir, q, t));
        show(dir, q, t);
        if (t < 0.98f * tb[dir]) { tb[dir] = t; best[dir] = q; }  // a clear gain, not timing noise
        return GJ_OK;
      };
      // The two kernels of a step run concurrently and the step takes about
      // the longer of them, so the general kernel's knobs go first (with the
      // fast kernel's default), then the fast kernel's, then the general
      // kernel's again when the fast ones changed.
      auto general = [&]() -> gj_status {
        const RingCfg from = best[dir];
        for (int S : Ss)
          for (int tjS : tjSs)
            for (int rw : rws) {
              RingCfg q = from;
              q.S = S; q.tjS = tjS; q.RWG = rw;
              GJ_TRY(consider(q));
            }
        return GJ_OK;
      };
      GJ_TRY(general());
      const RingCfg before = best[dir];
      for (int SF : SFs)
        for (int tjF : tjFs) {
          RingCfg q = before;
          q.SF = SF; q.tjF = tjF;
          GJ_TRY(consider(q));
        }
      if (!(best[dir] == before)) GJ_TRY(general());
    }
    GJ_TRY(clear());
    tuned[gn] = {best[0], best[1]};
    select_cfg(gn);
    GJ_TRY(prepare_tasks(err, gn));
    if (vb)
      fprintf(stderr,
              "gerjoii_b200 autotune %dx%d, %d shots/launch: forward S=%d SF=%d RWG=%d tjF=%d tjS=%d %.2f us/step; "
              "adjoint S=%d SF=%d RWG=%d tjF=%d tjS=%d %.2f us/step\n",
              NX, NY, gn, best[0].S, best[0].SF, best[0].RWG, best[0].tjF, best[0].tjS, 1e3f * tb[0] / reps,
              best[1].S, best[1].SF, best[1].RWG, best[1].tjF, best[1].tjS, 1e3f * tb[1] / reps);
    return GJ_OK;
  }

  // ------------------------------------------------ temporal blocking
  // Forward passes that keep no history (gj_w_forward without u, the misfit
  // and trial-misfit calls) can advance D = 1..4 Yee steps per launch
  // (w_tblock.cuh).  TbCfg: depth D (0 = the one-step ring kernels), tile
  // shape (tb_shape_G / tb_shape_RC), shots per tile CTA, and the streaming
  // mode: the interior rows and columns run as streaming warp tasks
  // (k_fwd_tbs, column chunks of lc) and only the rest of the grid as tiles.
  // The tuner (tb_tune) times the ring kernels and the blocked candidates on
  // this grid at the launch size and keeps the fastest; GJ_TB_DEPTH,
  // GJ_TB_SHAPE, GJ_TB_SPB, GJ_TB_STREAM and GJ_TB_CHUNK fix a configuration
  // instead (GJ_TB_DEPTH=0: ring kernels).
  struct TbCfg {
    int D = 0, shape = 1, spb = 1, stream = 0, lc = 32, ss = 6;  // ss: ring stages of the streaming tasks
    bool operator==(const TbCfg& o) const {
      return D == o.D && shape == o.shape && spb == o.spb && stream == o.stream && lc == o.lc && ss == o.ss;
    }
  };
  std::map<int, TbCfg> tb_tuned;
  // the gradient's forward with the whole history kept: blocked passes per
  // launch size when GJ_TB_GRAD=1 and the tuner chose them (else one step per launch)
  std::map<int, TbCfg> tb_grad;
  // Partition of one pass: tiles (interior tiles first, then PML tiles) and,
  // in streaming mode, the streaming tasks of gn shots.
  struct TbTiles {
    DevBuf buf; int nI = 0, nP = 0;
    DevBuf sbuf; int nS = 0;
  };
  std::map<long, std::unique_ptr<TbTiles>> tb_tiles;
  float tb_us = 0.f;  // tuned time per step (tb_tune), us
  // A batch of models in one blocked run (misfit_trials): tb_spt shots per
  // model, the coefficient sets tb_cstride elements apart from tb_w's, cezj per
  // (model, shot), the states and traces in the batch's own buffers; tb_spt = 0
  // for the plan's one model.
  int tb_spt = 0;
  size_t tb_cstride = 0;
  const WDev<T>* tb_w = nullptr;
  const T* tb_cezj = nullptr;
  DevBuf* tb_sA = nullptr;
  DevBuf* tb_sB = nullptr;
  DevBuf* tb_d = nullptr;
  static long tb_key(const TbCfg& q, int gn) {
    return (((((long(q.D) * 8 + q.shape) * 2 + (q.stream ? 1 : 0)) * 1024 + (q.stream ? q.lc : 0)) * 8 +
             (q.stream ? q.ss : 0)) << 24) | long(q.stream ? gn : 0);
  }

  // The partition of a pass of depth D for gn shots.  Streaming rows: tasks
  // of 32 V loaded rows at R = R0 + k stride whose rows R-1 .. R+32V are all
  // interior (fast) rows, columns [ej0 + D - 1, ej1 - D + 1] in chunks of lc;
  // every other node belongs to a clipped tile of TR x TC owned nodes,
  // classified interior when every node that a step updates in its staged
  // region (owned + D halo) uses the interior formulas.
  gj_status tb_prepare(Err& err, const TbCfg& q, int gn) {
    const long key = tb_key(q, gn);
    if (tb_tiles.count(key)) return GJ_OK;
    const int D = q.D, shape = q.shape;
    const int G = tb_shape_G(shape), RC = tb_shape_RC(shape);
    for (int pml = 0; pml < 2; ++pml) {
      const size_t sm = tb_smem(shape, pml, sizeof(T));
      if (sm > size_t(maxsm_dyn)) return err.set(GJ_EINVAL, "tile shape %d needs %zu B of shared memory", shape, sm);
      GJ_CUDA(err, cudaFuncSetAttribute(tb_kernel<T>(D, shape, pml), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        int(sm)));
    }
    auto tt = std::make_unique<TbTiles>();
    TbGeom gm{};
    gm.NX = NX; gm.NY = NY; gm.ei0 = w.ei0; gm.ei1 = w.ei1; gm.ej0 = w.ej0; gm.ej1 = w.ej1;
    gm.hyi0 = w.hyi0; gm.hyi1 = w.hyi1; gm.hxj0 = w.hxj0; gm.hxj1 = w.hxj1; gm.pml_top = g.pml_top; gm.bR0 = w.bR0;
    const TbPlan pl = tb_plan(gm, D, G, RC, q.stream != 0, VT<T>::V);
    if (!pl.rows.empty()) {
      const int cs_lo = pl.cs_lo, cs_hi = pl.cs_hi;
      // per (row task, chunk): a receiver of any shot among its owned nodes (so
      // the table serves every shot group of the same size)
      const int nch = (cs_hi - cs_lo + q.lc) / q.lc;
      std::vector<char> recf(pl.rows.size() * size_t(nch), 0);
      for (int zs = 0; zs < nshots; ++zs)
        for (int r = 0; r < nrs[zs]; ++r) {
          const long kk = sh[zs].rec[r];
          const int I = int(kk % ld), J = int(kk / ld);
          if (J < cs_lo || J > cs_hi) continue;
          for (size_t k = 0; k < pl.rows.size(); ++k)
            if (I >= pl.rows[k].own_lo && I < pl.rows[k].own_hi) recf[k * nch + (J - cs_lo) / q.lc] = 1;
        }
      std::vector<int4> ts;
      for (int z = 0; z < gn; ++z)
        for (size_t k = 0; k < pl.rows.size(); ++k)
          for (int c0 = cs_lo, ch = 0; c0 <= cs_hi; c0 += q.lc, ++ch) {
            const int c1 = std::min(c0 + q.lc - 1, cs_hi);
            ts.push_back(make_int4(pl.rows[k].R, c0 | (c1 << 16), pl.rows[k].own_lo | (pl.rows[k].own_hi << 16),
                                   z | (recf[k * nch + ch] ? TBS_HAS_REC : 0)));
          }
      tt->nS = int(ts.size());
      GJ_TRY(tt->sbuf.alloc(err, ts.size() * sizeof(int4)));
      GJ_CUDA(err, cudaMemcpy(tt->sbuf.p, ts.data(), ts.size() * sizeof(int4), cudaMemcpyHostToDevice));
      if (tbs_smem(q.ss) > size_t(maxsm_dyn)) return err.set(GJ_EINVAL, "streaming stages %d too many", q.ss);
      GJ_CUDA(err, cudaFuncSetAttribute(tbs_kernel<T>(D, q.ss), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        int(tbs_smem(q.ss))));
    }
    // tiles: interior ones first, then PML ones
    std::vector<int4> ti;
    for (const TbTile& t : pl.tiles) {
      ti.push_back(make_int4(t.r0, t.c0, t.tr, t.tc));
      (t.interior ? tt->nI : tt->nP) += 1;
    }
    if (!ti.empty()) {
      GJ_TRY(tt->buf.alloc(err, ti.size() * sizeof(int4)));
      GJ_CUDA(err, cudaMemcpy(tt->buf.p, ti.data(), ti.size() * sizeof(int4), cudaMemcpyHostToDevice));
    }
    tb_tiles.emplace(key, std::move(tt));
    return GJ_OK;
  }
  // q.D forward steps it .. it+q.D-1 of gn shots (A -> B); traces of the
  // steps into d ([shot][nrr][nt]) and Jz into jz when given.  PML tiles on
  // the side stream; streaming tasks and interior tiles on st.
  gj_status launch_fwd_tb(Err& err, const T* A, T* B, int it, int gn, const TbCfg& q, T* d, T* jz,
                          cudaStream_t st, int shot0 = 0, T* hist = nullptr, size_t hslot = 0, T* band = nullptr,
                          size_t bslot = 0) {
    if (q.D < 1 || q.D > 4 || it + q.D > g.nt) return err.set(GJ_EINVAL, "blocked pass of %d steps at %d", q.D, it);
    GJ_TRY(tb_prepare(err, q, gn));
    auto itt = tb_tiles.find(tb_key(q, gn));
    if (itt == tb_tiles.end()) return err.set(GJ_ECUDA, "blocked pass tables missing");
    const TbTiles& tt = *itt->second;
    TbArgs<T> a{};
    a.A = A; a.B = B; a.fstride = fstride; a.sstride = sstride; a.gn = gn; a.spb = std::max(q.spb, 1);
    a.it = it; a.nd = q.D; a.src = d_src; a.cezj = d_cezj; a.wav = d_wav; a.nt = g.nt; a.shot0 = shot0;
    a.nrr = std::max(nr, 1);
    a.rs = rsbuf.as<int>() + size_t(shot0) * a.nrr * 3; a.nrs = nrsbuf.as<int>() + shot0;
    a.hist = hist; a.hstride = dn; a.hslot = hslot;
    a.band = band; a.bslot = bslot;
    a.d = nr > 0 ? d : nullptr; a.jz = jz;
    a.spt = tb_spt > 0 ? tb_spt : gn;
    a.cstride = tb_cstride;
    if (tb_cezj) a.cezj = tb_cezj;
    if (tb_spt > 0 && a.spt % a.spb != 0) a.spb = 1;  // a tile CTA's shots stay in one model
    const WDev<T>& wd = tb_w ? *tb_w : w;
    const int gy = (gn + a.spb - 1) / a.spb;
    const int4* tl = tt.buf.template as<int4>();
    const int nth = 32 * TB_WARPS;
    last_kernels = (tt.nI > 0) + (tt.nP > 0) + (tt.nS > 0);
    const bool fork = side && tt.nP > 0 && (tt.nI > 0 || tt.nS > 0);
    if (fork) {
      GJ_CUDA(err, cudaEventRecord(ev_fork, st));
      GJ_CUDA(err, cudaStreamWaitEvent(side, ev_fork, 0));
    }
    if (tt.nP > 0)
      tb_kernel<T>(q.D, q.shape, true)<<<dim3(tt.nP, gy), nth, tb_smem(q.shape, true, sizeof(T)), fork ? side : st>>>(
          wd, a, tl + tt.nI);
    if (tt.nS > 0)
      tbs_kernel<T>(q.D, q.ss)<<<(tt.nS + TBS_WARPS - 1) / TBS_WARPS, 32 * TBS_WARPS, tbs_smem(q.ss), st>>>(
          wd, a, tt.sbuf.template as<int4>(), tt.nS);
    if (tt.nI > 0)
      tb_kernel<T>(q.D, q.shape, false)<<<dim3(tt.nI, gy), nth, tb_smem(q.shape, false, sizeof(T)), st>>>(wd, a, tl);
    if (fork) {
      GJ_CUDA(err, cudaEventRecord(ev_join, side));
      GJ_CUDA(err, cudaStreamWaitEvent(st, ev_join, 0));
    }
    return GJ_OK;
  }
  // A pass of up to q.D steps from step it: the last pass of a run shorter
  // than q.D uses the same configuration at the remaining depth.
  gj_status launch_fwd_tb_at(Err& err, const T* A, T* B, int it, int gn, const TbCfg& q, T* d, T* jz,
                             cudaStream_t st, int& nd) {
    TbCfg qq = q;
    qq.D = std::min(q.D, g.nt - it);
    nd = qq.D;
    return launch_fwd_tb(err, A, B, it, gn, qq, d, jz, st);
  }
  // The configuration for forward-only passes of gn shots: the environment's,
  // else the tuned one (timed on first use), else the ring kernels.
  gj_status tb_select(Err& err, int gn, cudaStream_t st, TbCfg& out) {
    TbCfg e;
    bool fixed = false;
    auto env = [&](const char* k, int& v, int lo, int hi) {
      if (const char* x = getenv(k)) { v = std::min(std::max(atoi(x), lo), hi); fixed = true; }
    };
    env("GJ_TB_DEPTH", e.D, 0, 4);
    env("GJ_TB_SHAPE", e.shape, 0, TB_NSHAPE - 1);
    env("GJ_TB_SPB", e.spb, 1, 8);
    env("GJ_TB_STREAM", e.stream, 0, 1);
    env("GJ_TB_CHUNK", e.lc, 4, 1 << 20);
    env("GJ_TB_STAGES", e.ss, 3, 6);
    e.ss = e.ss >= 6 ? 6 : 3;
    if constexpr (VT<T>::V * sizeof(T) != 16) e.stream = 0;
    if (fixed) {
      if (e.D > 0 && tb_smem(e.shape, true, sizeof(T)) > size_t(maxsm_dyn)) e.shape = 0;
      out = e;
      return GJ_OK;
    }
    if (const char* x = getenv("GJ_AUTOTUNE"))
      if (atoi(x) == 0) { out = TbCfg{}; return GJ_OK; }
    auto itc = tb_tuned.find(gn);
    if (itc == tb_tuned.end()) {
      GJ_TRY(tb_tune(err, gn, st));
      itc = tb_tuned.find(gn);
    }
    out = itc->second;
    return GJ_OK;
  }
  // Times forward passes of gn zeroed shots (24 steps, receivers recorded,
  // the least of three runs after a warm-up run) for the ring kernels and for
  // every depth 1..4 x tile shape x shots per CTA (1, 2), and keeps the fastest.
  gj_status tb_tune(Err& err, int gn, cudaStream_t st) {
    // the ring candidate runs the ring configuration (and task tables) of gn shots
    if (ring_nth > 0 && tb_spt == 0) {
      select_cfg(gn);
      GJ_TRY(prepare_tasks(err, gn));
    }
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    GJ_CUDA(err, cudaEventCreate(&e0));
    GJ_CUDA(err, cudaEventCreate(&e1));
    struct EvGuard { cudaEvent_t a, b; ~EvGuard() { cudaEventDestroy(a); cudaEventDestroy(b); } } guard{e0, e1};
    const int nsteps = 24, trials = 3;
    const char* vb = getenv("GJ_AUTOTUNE_VERBOSE");
    const bool every = vb && atoi(vb) >= 2;
    DevBuf& sA = tb_sA ? *tb_sA : fwdA;
    DevBuf& sB = tb_sB ? *tb_sB : fwdB;
    DevBuf& dB = tb_d ? *tb_d : dbuf;
    auto run = [&](const TbCfg& q) -> gj_status {
      T* A = sA.as<T>() + ld;
      T* B = sB.as<T>() + ld;
      for (int it = 0; it < nsteps;) {
        if (q.D == 0) {
          StepArgs<T> a = step_args(A, B, it % g.nt);
          GJ_TRY(launch_fwd(err, a, gn, st));
          k_record<T><<<dim3(1, gn), 128, 0, st>>>(B, sstride, recbuf.as<long>(), std::max(nr, 1),
                                                   nrsbuf.as<int>(), it % g.nt, g.nt, dbuf.as<T>(), d_src,
                                                   static_cast<T*>(nullptr), gn);
          ++it;
        } else {
          int nd = 0;
          GJ_TRY(launch_fwd_tb_at(err, A, B, it % g.nt, gn, q, dB.as<T>(), nullptr, st, nd));
          it += nd;
        }
        std::swap(A, B);
      }
      return GJ_OK;
    };
    auto time_cfg = [&](const TbCfg& q, float& ms) -> gj_status {
      GJ_CUDA(err, cudaMemsetAsync(sA.p, 0, size_t(gn) * sstride * sizeof(T), st));
      GJ_CUDA(err, cudaMemsetAsync(sB.p, 0, size_t(gn) * sstride * sizeof(T), st));
      GJ_TRY(run(q));  // warm-up
      for (int trial = 0; trial < trials; ++trial) {
        GJ_CUDA(err, cudaEventRecord(e0, st));
        GJ_TRY(run(q));
        GJ_CUDA(err, cudaEventRecord(e1, st));
        GJ_CUDA(err, cudaEventSynchronize(e1));
        float t = 0.f;
        GJ_CUDA(err, cudaEventElapsedTime(&t, e0, e1));
        ms = trial ? std::min(ms, t) : t;
      }
      GJ_CUDA(err, cudaGetLastError());
      if (every)
        fprintf(stderr, "gerjoii_b200 tb candidate D=%d shape=%d spb=%d stream=%d lc=%d ss=%d %.2f us/step\n", q.D,
                q.shape, q.spb, q.stream, q.lc, q.ss, 1e3f * ms / nsteps);
      return GJ_OK;
    };
    std::vector<TbCfg> cands;
    if (ring_nth > 0 && tb_spt == 0) cands.push_back(TbCfg{});  // the ring kernels run the plan's model only
    for (int D = 1; D <= 4; ++D)
      for (int sh = 0; sh < TB_NSHAPE; ++sh)
        for (int spb : {1, 2}) {
          if (tb_smem(sh, true, sizeof(T)) > size_t(maxsm_dyn)) continue;
          if (spb > gn) continue;
          TbCfg q; q.D = D; q.shape = sh; q.spb = spb;
          cands.push_back(q);
        }
    if constexpr (VT<T>::V * sizeof(T) == 16)
      for (int D = 1; D <= 4; ++D)
        for (int lc : {16, 32, 64})
          for (int ss : {3, 6})
            for (int spb : {1, 2}) {
              if (spb > gn) continue;
              TbCfg q; q.D = D; q.shape = 0; q.stream = 1; q.lc = lc; q.ss = ss; q.spb = spb;
              cands.push_back(q);
            }
    TbCfg best = cands.front();
    float tbest = 0.f;
    GJ_TRY(time_cfg(best, tbest));  // clocks up before the first timing
    GJ_TRY(time_cfg(best, tbest));
    for (size_t k = 1; k < cands.size(); ++k) {
      float t = 0.f;
      GJ_TRY(time_cfg(cands[k], t));
      if (t < 0.98f * tbest) { tbest = t; best = cands[k]; }
    }
    tb_tuned[gn] = best;
    tb_us = 1e3f * tbest / nsteps;
    if (vb)
      fprintf(stderr, "gerjoii_b200 tb autotune %dx%d, %d shots/launch: D=%d shape=%d spb=%d stream=%d lc=%d ss=%d "
              "%.2f us/step\n", NX, NY, gn, best.D, best.shape, best.spb, best.stream, best.lc, best.ss, tb_us);
    return GJ_OK;
  }

  // Coefficients from the model (host doubles or device T / double).
  template <class TM>
  gj_status build(Err& err, Ctx& c, const TM* eps_dev, const TM* sig_dev, cudaStream_t st) {
    CoefBuild cb;
    cb.NX = NX; cb.NY = NY; cb.ld = ld; cb.P = g.pml; cb.Pt = g.pml_top; cb.air = g.air; cb.m = g.m; cb.n = g.n;
    cb.dx = g.dx; cb.dy = g.dy; cb.dt = g.dt; cb.eps0 = g.eps0; cb.mu0 = g.mu0;
    const double* pp = prof.as<double>();
    cb.sex = pp; cb.smx = pp + NX + 2; cb.sey = pp + 2 * (NX + 2); cb.smy = pp + 2 * (NX + 2) + NY + 2;
    dim3 blk(32, 8), grd((NX + 1 + 31) / 32, (NY + 1 + 7) / 8);
    k_build_coefs<T, TM><<<grd, blk, 0, st>>>(cb, eps_dev, sig_dev, const_cast<T*>(w.ce), const_cast<T*>(w.chy),
                                            const_cast<T*>(w.ax), const_cast<T*>(w.bx), const_cast<T*>(w.ay),
                                            const_cast<T*>(w.by), const_cast<T*>(w.hxa), const_cast<T*>(w.hxb),
                                            const_cast<T*>(w.hya), const_cast<T*>(w.hyb), const_cast<T*>(wr.ce),
                                            const_cast<T*>(wr.chy), eps_m, sig_m);
    k_cezj<TM><<<(nshots + 127) / 128, 128, 0, st>>>(cb, eps_dev, sig_dev, sibuf.as<int>(), sjbuf.as<int>(), nshots,
                                                   d_cezj, sizeof(T) == 8);
    c.launches += 2;
    GJ_CUDA(err, cudaGetLastError());
    return GJ_OK;
  }

  StepArgs<T> step_args(const T* A, T* B, int it) const {
    StepArgs<T> a{};
    a.A = A; a.B = B; a.fstride = fstride; a.sstride = sstride; a.shot0 = 0; a.tj = tj; a.it = it;
    a.src = d_src; a.cezj = d_cezj; a.wav = d_wav; a.nt = g.nt; a.hist = nullptr; a.hstride = 0;
    a.kahan = 1;
    return a;
  }

  gj_status alloc_states(Err& err) {
    GJ_TRY(fwdA.alloc(err, size_t(nshots) * sstride * sizeof(T)));
    GJ_TRY(fwdB.alloc(err, size_t(nshots) * sstride * sizeof(T)));
    return GJ_OK;
  }

  // ------------------------------------------------------------ forward
  gj_status forward(Err& err, Ctx& c, const double* eps, const double* sig, double* d_out,
                    double* jz_out, double* u_out) {
    cudaStream_t st = 0;
    DevBuf mh;
    GJ_TRY(mh.alloc(err, 2 * mn * sizeof(double)));
    GJ_CUDA(err, cudaMemcpy(mh.as<double>(), eps, mn * sizeof(double), cudaMemcpyHostToDevice));
    GJ_CUDA(err, cudaMemcpy(mh.as<double>() + mn, sig, mn * sizeof(double), cudaMemcpyHostToDevice));
    GJ_TRY(build<double>(err, c, mh.as<double>(), mh.as<double>() + mn, st));
    ring_on = ring_nth > 0;
    select_cfg(nshots);
    GJ_TRY(prepare_tasks(err, nshots));
    TbCfg tq;  // several steps per launch when no history is kept
    if (!u_out) GJ_TRY(tb_select(err, nshots, st, tq));
    GJ_CUDA(err, cudaMemsetAsync(fwdA.p, 0, nshots * sstride * sizeof(T), st));
    GJ_CUDA(err, cudaMemsetAsync(fwdB.p, 0, nshots * sstride * sizeof(T), st));
    T* A = fwdA.as<T>() + ld;
    T* B = fwdB.as<T>() + ld;
    const int nrr = std::max(nr, 1);
    DevBuf jzb, ub;
    if (jz_out) GJ_TRY(jzb.alloc(err, size_t(nshots) * g.nt * sizeof(T)));
    if (u_out) GJ_TRY(ub.alloc(err, size_t(nshots) * dn * (g.nt + 1) * sizeof(T)));
    Marks tbm;  // per-launch device time when kernel timing is on
    struct CurGuard { KernelTimer& t; ~CurGuard() { t.cur = nullptr; t.open = -1; } } cg{c.timer};
    c.timer.cur = &tbm;
    for (int it = 0, nd = 0; tq.D > 0 && it < g.nt; it += nd) {
      const bool tm = c.timer.begin(KK_TB_PASS, st, nshots);
      GJ_TRY(launch_fwd_tb_at(err, A, B, it, nshots, tq, dbuf.as<T>(), jz_out ? jzb.as<T>() : nullptr, st, nd));
      c.timer.end(tm, st);
      c.launches += last_kernels;
      std::swap(A, B);
    }
    c.timer.close(st);
    for (int it = 0; tq.D == 0 && it < g.nt; ++it) {
      StepArgs<T> a = step_args(A, B, it);
      if (u_out) { a.hist = ub.as<T>() + size_t(it) * nshots * dn; a.hstride = dn; }
      // receivers recorded inside the ring step unless Jz is wanted too
      const bool fused = ring_on && nr > 0 && !jz_out;
      RecArgs<T> ra = rec_args(0);
      if (fused) { ra.d = dbuf.as<T>(); ra.it = it; }
      const bool tm = c.timer.begin(KK_FWD_STEP, st, nshots);
      GJ_TRY(launch_fwd(err, a, nshots, st, ra));
      if (!fused)
        k_record<T><<<dim3(1, nshots), 128, 0, st>>>(B, sstride, recbuf.as<long>(), nrr, nrsbuf.as<int>(), it,
                                                     g.nt, dbuf.as<T>(), d_src, jz_out ? jzb.as<T>() : nullptr,
                                                     nshots);
      c.timer.end(tm, st);
      c.launches += (fused ? 0 : 1) + last_kernels;
      std::swap(A, B);
    }
    c.timer.close(st);
    GJ_CUDA(err, cudaGetLastError());
    GJ_CUDA(err, cudaDeviceSynchronize());
    c.timer.collect(tbm);
    // copy out (per shot nt x nr, time fastest)
    std::vector<T> hd(size_t(nshots) * nrr * g.nt);
    GJ_CUDA(err, cudaMemcpy(hd.data(), dbuf.p, hd.size() * sizeof(T), cudaMemcpyDeviceToHost));
    size_t o = 0, nbad = 0;
    for (int s = 0; s < nshots; ++s)
      for (int r = 0; r < nrs[s]; ++r)
        for (int t = 0; t < g.nt; ++t) {
          d_out[o] = double(hd[(size_t(s) * nrr + r) * g.nt + t]);
          nbad += std::isfinite(d_out[o++]) ? 0 : 1;
        }
    if (jz_out) {
      std::vector<T> hj(size_t(nshots) * g.nt);
      GJ_CUDA(err, cudaMemcpy(hj.data(), jzb.p, hj.size() * sizeof(T), cudaMemcpyDeviceToHost));
      for (size_t i = 0; i < hj.size(); ++i) jz_out[i] = double(hj[i]);
    }
    if (u_out) {
      std::vector<T> hu(size_t(nshots) * dn * g.nt);
      GJ_CUDA(err, cudaMemcpy(hu.data(), ub.p, hu.size() * sizeof(T), cudaMemcpyDeviceToHost));
      // device [t][shot][domain-node] -> host [shot][t][m x n]
      const int di0 = w.di0;
      for (int s = 0; s < nshots; ++s)
        for (int t = 0; t < g.nt; ++t)
          for (int b = 0; b < g.n; ++b)
            for (int a_ = 0; a_ < g.m; ++a_)
              u_out[(size_t(s) * g.nt + t) * mn + size_t(b) * g.m + a_] =
                  double(hu[(size_t(t) * nshots + s) * dn + size_t(b) * hld + di0 - hr0 + a_]);
    }
    if (nbad) return err.set(GJ_ENUMERIC, "%zu non-finite trace samples (outputs written)", nbad);
    return GJ_OK;
  }

  // Conditioning of nshots per-shot gradients g (double, m x n each) in place:
  // source taper, k-space low-pass with widths (ka, kb), normali, NaN guard.
  DevBuf cbuf, condX, condF, condP;
  cufftHandle condplan = 0;
  int cond_batch = 0;
  gj_status condition(Err& err, Ctx& c, const gj_w_opts& o, double* gdev, double ka, double kb, cudaStream_t st) {
    const int m = g.m, n = g.n;
    int m_ = 1, n_ = 1;
    while (m_ < m) m_ <<= 1;  // 2^nextpow2
    while (n_ < n) n_ <<= 1;
    if (!(o.cond_fo > 0)) return err.set(GJ_EINVAL, "condition needs cond_fo > 0");
    if (!(ka > 0 && kb > 0)) return err.set(GJ_EINVAL, "condition needs cond_ax, cond_az > 0");
    // taper parameters per shot: source cell (clamped to the model), L = 4 lo
    std::vector<double> em(mn);
    GJ_CUDA(err, cudaMemcpyAsync(em.data(), eps_m, mn * sizeof(double), cudaMemcpyDeviceToHost, st));
    GJ_CUDA(err, cudaStreamSynchronize(st));
    const double cl = 1.0 / std::sqrt(g.mu0 * g.eps0);
    std::vector<double> par(4 * size_t(nshots));
    for (int s = 0; s < nshots; ++s) {
      const int as = std::min(std::max(sh_src_i[s] - w.di0, 0), m - 1);
      const int bs = std::min(std::max(sh_src_j[s] - w.dj0, 0), n - 1);
      const double lo = cl / std::sqrt(em[size_t(as) + size_t(bs) * m]) / o.cond_fo;
      const double L = 2.0 * (2.0 * lo);
      double mx = 0.0;  // normali of the taper: its largest value is at a corner
      for (int a : {0, m - 1})
        for (int b : {0, n - 1}) {
          const double xa = (b - bs) * g.dx / L, za = (a - as) * g.dy / L;
          mx = std::max(mx, std::fabs(1.0 - std::exp(-(xa * xa + za * za))));
        }
      par[4 * s] = as; par[4 * s + 1] = bs; par[4 * s + 2] = L; par[4 * s + 3] = 1.0 / (mx == 0.0 ? 1.0 : mx);
    }
    // low-pass filter in k (image_gaussian.m:37-52), fftshift-ed, with 1/(m_ n_)
    std::vector<double> F(size_t(m_) * n_);
    const double A = n_ * (ka / 2) * std::sqrt(2.0), B = m_ * (kb / 2) * std::sqrt(2.0);
    for (int j = 0; j < n_; ++j)
      for (int i = 0; i < m_; ++i) {
        const int X = (j + n_ / 2) % n_, Y = (i + m_ / 2) % m_;
        const double kx = (X - n_ / 2) / A, ky = (Y - m_ / 2) / B;
        F[size_t(i) + size_t(j) * m_] = std::exp(-(kx * kx + ky * ky)) / (double(m_) * n_);
      }
    GJ_TRY(condP.alloc(err, par.size() * sizeof(double)));
    GJ_TRY(condF.alloc(err, F.size() * sizeof(double)));
    GJ_TRY(condX.alloc(err, size_t(nshots) * m_ * n_ * sizeof(cuDoubleComplex)));
    GJ_CUDA(err, cudaMemcpyAsync(condP.p, par.data(), par.size() * sizeof(double), cudaMemcpyHostToDevice, st));
    GJ_CUDA(err, cudaMemcpyAsync(condF.p, F.data(), F.size() * sizeof(double), cudaMemcpyHostToDevice, st));
    if (condplan && cond_batch != nshots) { cufftDestroy(condplan); condplan = 0; }
    if (!condplan) {
      int dims[2] = {n_, m_};  // column-major m_ x n_: the slow dimension is n_
      if (cufftPlanMany(&condplan, 2, dims, nullptr, 1, m_ * n_, nullptr, 1, m_ * n_, CUFFT_Z2Z, nshots) !=
          CUFFT_SUCCESS)
        return err.set(GJ_ENOMEM, "cufftPlanMany(%d x %d, batch=%d) failed", m_, n_, nshots);
      cond_batch = nshots;
    }
    cuDoubleComplex* X = condX.as<cuDoubleComplex>();
    k_cond_taper<<<512, 256, 0, st>>>(gdev, nshots, m, n, g.dx, g.dy, condP.as<double>());
    k_cond_pad<<<512, 256, 0, st>>>(gdev, X, nshots, m, n, m_, n_);
    cufftSetStream(condplan, st);
    if (cufftExecZ2Z(condplan, X, X, CUFFT_FORWARD) != CUFFT_SUCCESS) return err.set(GJ_ECUDA, "cufft 2-D failed");
    k_cond_mul<<<512, 256, 0, st>>>(X, condF.as<double>(), size_t(m_) * n_, nshots);
    if (cufftExecZ2Z(condplan, X, X, CUFFT_INVERSE) != CUFFT_SUCCESS) return err.set(GJ_ECUDA, "cufft 2-D failed");
    k_cond_trim<<<512, 256, 0, st>>>(X, gdev, nshots, m, n, m_, n_);
    k_cond_norm<<<nshots, 1024, 0, st>>>(gdev, mn);
    c.launches += 7;
    GJ_CUDA(err, cudaStreamSynchronize(st));  // F and par go out of scope
    return GJ_OK;
  }

  // ------------------------------------------------------------ misfit only
  // Forward runs and misfits of all shots, no history and no adjoint: the
  // objective evaluations of a step-length search (w_objs_e.m:24-65, called
  // by w_stepparabola_e.m:20-41 for each trial model).
  // With opts->filt_high > filt_low both trace sets are band-filtered first
  // (w_objs_e.m:33-36 / w_objs_s.m), so the misfit and its normaliser are
  // those of the filtered traces.
  gj_status misfit(Err& err, Ctx& c, const double* eps, const double* sig, const double* dobs, gj_misfit_kind mk,
                   double* misfit_out, cudaStream_t st, const gj_w_opts* opts = nullptr) {
    GJ_TRY(stage_inputs(err, c, eps, sig, false, dobs, false, st));
    ring_on = ring_nth > 0;
    select_cfg(nshots);
    GJ_TRY(prepare_tasks(err, nshots));
    TbCfg tq;  // several steps per launch
    GJ_TRY(tb_select(err, nshots, st, tq));
    GJ_CUDA(err, cudaMemsetAsync(fwdA.p, 0, nshots * sstride * sizeof(T), st));
    GJ_CUDA(err, cudaMemsetAsync(fwdB.p, 0, nshots * sstride * sizeof(T), st));
    GJ_CUDA(err, cudaMemsetAsync(sums.p, 0, 2 * nshots * sizeof(double), st));
    T* A = fwdA.as<T>() + ld;
    T* B = fwdB.as<T>() + ld;
    const int nrr = std::max(nr, 1);
    const size_t tr = size_t(nrr) * g.nt;
    Marks tbm;  // per-launch device time when kernel timing is on
    struct CurGuard { KernelTimer& t; ~CurGuard() { t.cur = nullptr; t.open = -1; } } cg{c.timer};
    c.timer.cur = &tbm;
    for (int it = 0, nd = 0; tq.D > 0 && it < g.nt; it += nd) {
      const bool tm = c.timer.begin(KK_TB_PASS, st, nshots);
      GJ_TRY(launch_fwd_tb_at(err, A, B, it, nshots, tq, dbuf.as<T>(), nullptr, st, nd));
      c.timer.end(tm, st);
      c.launches += last_kernels;
      std::swap(A, B);
    }
    c.timer.close(st);
    for (int it = 0; tq.D == 0 && it < g.nt; ++it) {
      StepArgs<T> a = step_args(A, B, it);
      const bool fused = ring_on && nr > 0;  // receivers recorded inside the ring step
      RecArgs<T> ra = rec_args(0);
      if (fused) { ra.d = dbuf.as<T>(); ra.it = it; }
      const bool tm = c.timer.begin(KK_FWD_STEP, st, nshots);
      GJ_TRY(launch_fwd(err, a, nshots, st, ra));
      if (!fused)
        k_record<T><<<dim3(1, nshots), 128, 0, st>>>(B, sstride, recbuf.as<long>(), nrr, nrsbuf.as<int>(), it,
                                                     g.nt, dbuf.as<T>(), d_src, static_cast<T*>(nullptr), nshots);
      c.timer.end(tm, st);
      c.launches += (fused ? 0 : 1) + last_kernels;
      std::swap(A, B);
    }
    c.timer.close(st);
    if (opts && opts->filt_high > opts->filt_low) {
      GJ_TRY(filt_traces(err, c, *opts, dbuf.as<T>(), nshots, st));
      GJ_TRY(filt_traces(err, c, *opts, dobsbuf.as<T>(), nshots, st));
    }
    if (mk != GJ_MISFIT_L2) {
      GJ_TRY(env_residual(err, c, 0, nshots, mk, st));
    } else {
      k_residual<T><<<dim3(64, nshots), 256, 0, st>>>(dbuf.as<T>(), dobsbuf.as<T>(), ebuf.as<T>(), tr,
                                                      sums.as<double>());
      ++c.launches;
    }
    GJ_CUDA(err, cudaGetLastError());
    std::vector<double> hs(2 * nshots);
    GJ_CUDA(err, cudaMemcpyAsync(hs.data(), sums.p, hs.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
    GJ_CUDA(err, cudaStreamSynchronize(st));
    c.timer.collect(tbm);
    int nbad = 0;
    for (int q = 0; q < nshots; ++q) {
      misfit_out[q] = hs[2 * q + 1] > 0 ? 0.5 * hs[2 * q] / hs[2 * q + 1] : 0.5 * hs[2 * q];
      nbad += std::isfinite(misfit_out[q]) ? 0 : 1;
    }
    if (nbad) return err.set(GJ_ENUMERIC, "%d non-finite misfits (outputs written)", nbad);
    return GJ_OK;
  }

  // All trial models of one step-length search (w_stepparabola_e.m:20-27) as
  // one blocked forward run: every pass is one launch over the ntrial x nshots
  // (model, shot) pairs, each model with its own coefficient set; then the
  // misfits of each model as misfit() computes them.  done = false (nothing
  // run) when the configuration for the batch is one step per launch: the
  // ring kernels run the plan's model only, and the caller then runs the
  // models one by one.
  gj_status misfit_trials(Err& err, Ctx& c, int ntrial, const double* eps, const double* sig, const double* dobs,
                          gj_misfit_kind mk, double* out, cudaStream_t st, const gj_w_opts* opts, bool& done) {
    done = false;
    if constexpr (VT<T>::V * sizeof(T) != 16) return GJ_OK;
    if (ntrial < 2 || ring_nth == 0) return GJ_OK;
    const int gn = ntrial * nshots;
    const size_t cset = 12 * fstride;  // elements of one coefficient set
    const int nrr = std::max(nr, 1);
    const size_t tr = size_t(nrr) * g.nt;
    {  // the batch's states, traces and coefficient sets must fit; else one model at a time
      size_t fr = 0, tot = 0;
      GJ_CUDA(err, cudaMemGetInfo(&fr, &tot));
      const size_t need = (size_t(gn) * (2 * sstride + tr) + size_t(ntrial) * cset) * sizeof(T);
      if (need > fr / 10 * 8) return GJ_OK;
    }
    GJ_TRY(stage_inputs(err, c, eps, sig, false, dobs, false, st));  // observed traces (and model 0)
    ring_on = true;
    select_cfg(nshots);
    GJ_TRY(prepare_tasks(err, nshots));
    DevBuf tcoef, tcz, tA, tB, td, mh;
    GJ_TRY(tcoef.alloc(err, size_t(ntrial) * cset * sizeof(T)));
    GJ_TRY(tcz.alloc(err, size_t(gn) * sizeof(T)));
    GJ_TRY(mh.alloc(err, 2 * mn * sizeof(double)));
    GJ_CUDA(err, cudaMemsetAsync(tcoef.p, 0, size_t(ntrial) * cset * sizeof(T), st));
    T* base = tcoef.as<T>() + ld;  // one column in, like the plan's arrays
    {
      struct Restore {
        WSolver& s; WDev<T> w0, wr0;
        ~Restore() { s.w = w0; s.wr = wr0; }
      } rs{*this, w, wr};
      for (int t = 0; t < ntrial; ++t) {
        GJ_CUDA(err, cudaMemcpyAsync(mh.as<double>(), eps + size_t(t) * mn, mn * sizeof(double),
                                     cudaMemcpyHostToDevice, st));
        GJ_CUDA(err, cudaMemcpyAsync(mh.as<double>() + mn, sig + size_t(t) * mn, mn * sizeof(double),
                                     cudaMemcpyHostToDevice, st));
        T* cb = base + size_t(t) * cset;
        w.ce = cb; w.chy = cb + fstride; w.ax = cb + 2 * fstride; w.bx = cb + 3 * fstride;
        w.ay = cb + 4 * fstride; w.by = cb + 5 * fstride; w.hxa = cb + 6 * fstride; w.hxb = cb + 7 * fstride;
        w.hya = cb + 8 * fstride; w.hyb = cb + 9 * fstride;
        wr.ce = cb + 10 * fstride; wr.chy = cb + 11 * fstride;
        GJ_TRY(build<double>(err, c, mh.as<double>(), mh.as<double>() + mn, st));
        GJ_CUDA(err, cudaMemcpyAsync(tcz.as<T>() + size_t(t) * nshots, d_cezj, nshots * sizeof(T),
                                     cudaMemcpyDeviceToDevice, st));
        // mh is rewritten by the next model: its build must have read it
        GJ_CUDA(err, cudaStreamSynchronize(st));
      }
    }
    WDev<T> wt = w;  // model 0's arrays; model t's lie t * cset further
    wt.ce = base; wt.chy = base + fstride; wt.ax = base + 2 * fstride; wt.bx = base + 3 * fstride;
    wt.ay = base + 4 * fstride; wt.by = base + 5 * fstride; wt.hxa = base + 6 * fstride; wt.hxb = base + 7 * fstride;
    wt.hya = base + 8 * fstride; wt.hyb = base + 9 * fstride;
    GJ_TRY(tA.alloc(err, size_t(gn) * sstride * sizeof(T)));
    GJ_TRY(tB.alloc(err, size_t(gn) * sstride * sizeof(T)));
    GJ_TRY(td.alloc(err, size_t(gn) * tr * sizeof(T)));
    struct Batch {
      WSolver& s;
      ~Batch() {
        s.tb_spt = 0; s.tb_cstride = 0; s.tb_w = nullptr; s.tb_cezj = nullptr;
        s.tb_sA = s.tb_sB = s.tb_d = nullptr;
      }
    } bg{*this};
    tb_spt = nshots; tb_cstride = cset; tb_w = &wt; tb_cezj = tcz.as<T>();
    tb_sA = &tA; tb_sB = &tB; tb_d = &td;
    TbCfg tq;
    GJ_TRY(tb_select(err, gn, st, tq));
    if (tq.D == 0) return GJ_OK;  // one step per launch: the caller runs the models one by one
    GJ_CUDA(err, cudaMemsetAsync(tA.p, 0, size_t(gn) * sstride * sizeof(T), st));
    GJ_CUDA(err, cudaMemsetAsync(tB.p, 0, size_t(gn) * sstride * sizeof(T), st));
    T* A = tA.as<T>() + ld;
    T* B = tB.as<T>() + ld;
    Marks tbm;
    struct CurGuard { KernelTimer& t; ~CurGuard() { t.cur = nullptr; t.open = -1; } } cg{c.timer};
    c.timer.cur = &tbm;
    for (int it = 0, nd = 0; it < g.nt; it += nd) {
      const bool tm = c.timer.begin(KK_TB_PASS, st, gn);
      GJ_TRY(launch_fwd_tb_at(err, A, B, it, gn, tq, td.as<T>(), nullptr, st, nd));
      c.timer.end(tm, st);
      c.launches += last_kernels;
      std::swap(A, B);
    }
    c.timer.close(st);
    const bool filt = opts && opts->filt_high > opts->filt_low;
    if (filt) GJ_TRY(filt_traces(err, c, *opts, dobsbuf.as<T>(), nshots, st));
    int nbad = 0;
    std::vector<double> hs(2 * nshots);
    for (int t = 0; t < ntrial; ++t) {
      GJ_CUDA(err, cudaMemcpyAsync(dbuf.p, td.as<T>() + size_t(t) * nshots * tr, size_t(nshots) * tr * sizeof(T),
                                   cudaMemcpyDeviceToDevice, st));
      GJ_CUDA(err, cudaMemsetAsync(sums.p, 0, 2 * nshots * sizeof(double), st));
      if (filt) GJ_TRY(filt_traces(err, c, *opts, dbuf.as<T>(), nshots, st));
      if (mk != GJ_MISFIT_L2) {
        GJ_TRY(env_residual(err, c, 0, nshots, mk, st));
      } else {
        k_residual<T><<<dim3(64, nshots), 256, 0, st>>>(dbuf.as<T>(), dobsbuf.as<T>(), ebuf.as<T>(), tr,
                                                        sums.as<double>());
        ++c.launches;
      }
      GJ_CUDA(err, cudaGetLastError());
      GJ_CUDA(err, cudaMemcpyAsync(hs.data(), sums.p, hs.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
      GJ_CUDA(err, cudaStreamSynchronize(st));
      for (int q = 0; q < nshots; ++q) {
        double& m = out[size_t(t) * nshots + q];
        m = hs[2 * q + 1] > 0 ? 0.5 * hs[2 * q] / hs[2 * q + 1] : 0.5 * hs[2 * q];
        nbad += std::isfinite(m) ? 0 : 1;
      }
    }
    c.timer.collect(tbm);
    done = true;
    if (nbad) return err.set(GJ_ENUMERIC, "%d non-finite misfits (outputs written)", nbad);
    return GJ_OK;
  }

  // ------------------------------------------------------------ gradient
  // Chooses K: the whole history when it fits, else checkpoints every K steps.
  void choose_k(const gj_w_opts& o, size_t free_bytes) {
    const size_t budget = o.mem_budget_bytes ? o.mem_budget_bytes : size_t(0.8 * double(free_bytes));
    const size_t bnd = band_on ? size_t(w.bsz) : 0;  // band history per shot and slot
    const size_t per_slot = size_t(nshots) * (dn + bnd) * sizeof(T);
    const size_t per_ck = size_t(nshots) * sstride * sizeof(T);
    if (o.ckpt_every > 0) { K = std::min(std::max(o.ckpt_every, 2), g.nt); return; }
    const size_t extra = ring_on ? size_t(Kd) * per_slot : 0;  // the l ring (and the band ring)
    if (size_t(g.nt + 1) * per_slot + extra <= budget) { K = g.nt; return; }
    double k = std::sqrt(double(g.nt) * double(per_ck) / double(per_slot));
    K = std::min(std::max(int(k), 2), g.nt);
    while (K > 2 && (size_t(g.nt / K + 2) * per_ck + size_t(K + 3) * per_slot + extra) > budget) K = K * 3 / 4;
  }

  // Inputs of a gradient call on the device: coefficients built from the model,
  // observed traces converted to T in dobsbuf ([shot][r][t]).
  gj_status stage_inputs(Err& err, Ctx& c, const void* eps, const void* sig, bool dev_in, const void* dobs,
                         bool dev_dobs, cudaStream_t st) {
    const int nrr = std::max(nr, 1);
    const size_t tr = size_t(nrr) * g.nt;
    if (!dev_in) {
      GJ_TRY(stage.alloc(err, 2 * mn * sizeof(double)));
      GJ_CUDA(err, cudaMemcpyAsync(stage.as<double>(), eps, mn * sizeof(double), cudaMemcpyHostToDevice, st));
      GJ_CUDA(err, cudaMemcpyAsync(stage.as<double>() + mn, sig, mn * sizeof(double), cudaMemcpyHostToDevice, st));
      GJ_TRY(build<double>(err, c, stage.as<double>(), stage.as<double>() + mn, st));
    } else {
      GJ_TRY(build<T>(err, c, static_cast<const T*>(eps), static_cast<const T*>(sig), st));
    }
    if (dev_dobs) {
      GJ_CUDA(err, cudaMemcpyAsync(dobsbuf.p, dobs, size_t(nshots) * tr * sizeof(T), cudaMemcpyDeviceToDevice, st));
      return GJ_OK;
    }
    bool uniform = true;
    for (int s = 0; s < nshots; ++s) uniform = uniform && nrs[s] == nrr;
    if (uniform) {
      // host doubles straight to the device, converted there
      GJ_TRY(stage2.alloc(err, size_t(nshots) * tr * sizeof(double)));
      GJ_CUDA(err, cudaMemcpyAsync(stage2.p, dobs, size_t(nshots) * tr * sizeof(double), cudaMemcpyHostToDevice, st));
      k_convert<double, T><<<1024, 256, 0, st>>>(stage2.as<double>(), dobsbuf.as<T>(), size_t(nshots) * tr);
      ++c.launches;
      GJ_CUDA(err, cudaGetLastError());
      return GJ_OK;
    }
    std::vector<T> hd(size_t(nshots) * tr, T(0));
    size_t q = 0;
    for (int s = 0; s < nshots; ++s)
      for (int r = 0; r < nrs[s]; ++r)
        for (int t = 0; t < g.nt; ++t) hd[(size_t(s) * nrr + r) * g.nt + t] = T(static_cast<const double*>(dobs)[q++]);
    GJ_CUDA(err, cudaMemcpyAsync(dobsbuf.p, hd.data(), hd.size() * sizeof(T), cudaMemcpyHostToDevice, st));
    GJ_CUDA(err, cudaStreamSynchronize(st));
    return GJ_OK;
  }

  // Segments [s0, s1) of the time axis; a remainder of one step joins the previous one.
  std::vector<std::pair<int, int>> segments() const {
    std::vector<std::pair<int, int>> segs;
    for (int s0 = 0; s0 < g.nt; s0 += K) segs.push_back({s0, std::min(g.nt, s0 + K)});
    if (segs.size() > 1 && segs.back().second - segs.back().first < 2) {
      segs[segs.size() - 2].second = segs.back().second;
      segs.pop_back();
    }
    return segs;
  }

  // d/dt u stencil of differentiate_cube.m:33-51 for 1-based history slot k.
  void ddt_stencil(int k, int& k0, int& k1, int& k2, double& c0, double& c1, double& c2) const {
    const int nt = g.nt;
    const double dt = g.dt;
    if (k == 1) { k0 = 1; k1 = 2; k2 = 3; c0 = -1.5 / dt; c1 = 2.0 / dt; c2 = -0.5 / dt; }
    else if (k == nt) { k0 = nt - 2; k1 = nt - 1; k2 = nt; c0 = 0.5 / dt; c1 = -2.0 / dt; c2 = 1.5 / dt; }
    else { k0 = k - 1; k1 = k; k2 = k + 1; c0 = -0.5 / dt; c1 = 0.0; c2 = 0.5 / dt; }
  }

  // Band terms of the exact eps gradient added to gdev (double, per shot or summed).
  void band_finish(Ctx& c, double* gdev, int per_shot, cudaStream_t st) {
    BandFinish f;
    f.dt = g.dt; f.eps0 = g.eps0; f.mu0 = g.mu0; f.Pt = g.pml_top; f.air = g.air; f.eps_m = eps_m;
    const double* pp = prof.as<double>();
    f.sex = pp; f.smx = pp + NX + 2; f.sey = pp + 2 * (NX + 2); f.smy = pp + 2 * (NX + 2) + NY + 2;
    k_band_finish<T><<<2 * nsm, 256, 0, st>>>(w, bacc.as<T>(), 2 * size_t(w.bsz), nshots, per_shot, f, gdev);
    ++c.launches;
  }

  // Final scaling, shot reduction and outputs.
  gj_status finish(Err& err, Ctx& c, gj_adj_mode mode, const gj_w_opts& o, void* geps, void* gsig, bool dev_out,
                   double* misfit_out, double* d_out, double* e_out, const std::vector<double>& hsums,
                   cudaStream_t st) {
    const int nrr = std::max(nr, 1);
    const size_t tr = size_t(nrr) * g.nt;
    const size_t gsz = (o.per_shot ? size_t(nshots) : 1) * mn;
    double* ge_d; double* gs_d;
    if (dev_out && sizeof(T) == 8) { ge_d = static_cast<double*>(geps); gs_d = static_cast<double*>(gsig); }
    else {
      GJ_TRY(gout.alloc(err, 2 * gsz * sizeof(double)));
      ge_d = gout.as<double>(); gs_d = ge_d + gsz;
    }
    if (o.condition) {
      // per-shot gradients, conditioned, then averaged (or returned per shot)
      GJ_TRY(cbuf.alloc(err, 2 * size_t(nshots) * mn * sizeof(double)));
      double* ce_ = cbuf.as<double>();
      double* cs_ = ce_ + size_t(nshots) * mn;
      k_finish<T><<<256, 256, 0, st>>>(w, acc.as<T>(), 4 * dn, nshots, 1, mode == GJ_ADJ_EXACT ? 1 : 0, g.dt,
                                       g.eps0, eps_m, sig_m, ce_, cs_);
      ++c.launches;
      if (mode == GJ_ADJ_EXACT && band_on) band_finish(c, ce_, 1, st);
      GJ_TRY(condition(err, c, o, ce_, o.cond_ax, o.cond_az, st));
      GJ_TRY(condition(err, c, o, cs_, 2 * o.cond_ax, 2 * o.cond_az, st));
      if (o.per_shot) {
        GJ_CUDA(err, cudaMemcpyAsync(ge_d, ce_, gsz * sizeof(double), cudaMemcpyDeviceToDevice, st));
        GJ_CUDA(err, cudaMemcpyAsync(gs_d, cs_, gsz * sizeof(double), cudaMemcpyDeviceToDevice, st));
      } else {
        k_shot_mean<<<256, 256, 0, st>>>(ce_, nshots, mn, ge_d);
        k_shot_mean<<<256, 256, 0, st>>>(cs_, nshots, mn, gs_d);
        c.launches += 2;
      }
    } else {
      k_finish<T><<<256, 256, 0, st>>>(w, acc.as<T>(), 4 * dn, nshots, o.per_shot, mode == GJ_ADJ_EXACT ? 1 : 0,
                                       g.dt, g.eps0, eps_m, sig_m, ge_d, gs_d);
      ++c.launches;
      if (mode == GJ_ADJ_EXACT && band_on) band_finish(c, ge_d, o.per_shot, st);
    }
    GJ_TRY(count_nonfinite_async(err, ge_d, gsz, true, 0, st));
    GJ_TRY(count_nonfinite_async(err, gs_d, gsz, true, 1, st));
    unsigned hnan[2] = {0, 0};
    GJ_CUDA(err, cudaMemcpyAsync(hnan, nanbuf.p, 2 * sizeof(unsigned), cudaMemcpyDeviceToHost, st));
    c.launches += 2;
    if (dev_out && sizeof(T) == 4) {
      k_convert<double, float><<<256, 256, 0, st>>>(ge_d, static_cast<float*>(geps), gsz);
      k_convert<double, float><<<256, 256, 0, st>>>(gs_d, static_cast<float*>(gsig), gsz);
      c.launches += 2;
    }
    GJ_CUDA(err, cudaGetLastError());
    if (!dev_out) {
      GJ_CUDA(err, cudaMemcpyAsync(geps, ge_d, gsz * sizeof(double), cudaMemcpyDeviceToHost, st));
      GJ_CUDA(err, cudaMemcpyAsync(gsig, gs_d, gsz * sizeof(double), cudaMemcpyDeviceToHost, st));
    }
    std::vector<T> hd, he;
    if (d_out) { hd.resize(size_t(nshots) * tr); GJ_CUDA(err, cudaMemcpyAsync(hd.data(), dbuf.p, hd.size() * sizeof(T), cudaMemcpyDeviceToHost, st)); }
    if (e_out) { he.resize(size_t(nshots) * tr); GJ_CUDA(err, cudaMemcpyAsync(he.data(), ebuf.p, he.size() * sizeof(T), cudaMemcpyDeviceToHost, st)); }
    GJ_CUDA(err, cudaStreamSynchronize(st));
    if (misfit_out)
      for (int s = 0; s < nshots; ++s)
        misfit_out[s] = hsums[2 * s + 1] > 0 ? 0.5 * hsums[2 * s] / hsums[2 * s + 1] : 0.5 * hsums[2 * s];
    auto unpack = [&](const std::vector<T>& v, double* out) {
      size_t q = 0;
      for (int s = 0; s < nshots; ++s)
        for (int r = 0; r < nrs[s]; ++r)
          for (int t = 0; t < g.nt; ++t) out[q++] = double(v[(size_t(s) * nrr + r) * g.nt + t]);
    };
    if (d_out) unpack(hd, d_out);
    if (e_out) unpack(he, e_out);
    bool bad_mis = false;
    for (int s = 0; s < nshots; ++s) bad_mis = bad_mis || !std::isfinite(hsums[2 * s]) || !std::isfinite(hsums[2 * s + 1]);
    if (hnan[0] || hnan[1] || bad_mis)
      return err.set(GJ_ENUMERIC, "non-finite results: %u of g_eps, %u of g_sig%s (outputs written; the reference "
                     "zeroes such gradients, w_update_e.m:131-137, which opts.condition does)",
                     hnan[0], hnan[1], bad_mis ? ", misfit" : "");
    return GJ_OK;
  }

  // ------------------------------------------------------------ envelope
  DevBuf envA, envAo, envG, envF;
  cufftHandle fftplan = 0;
  int fft_batch = 0;
  ~WSolver() override {
    if (fftplan) cufftDestroy(fftplan);
    if (filtplan) cufftDestroy(filtplan);
    if (condplan) cufftDestroy(condplan);
    if (side) cudaStreamDestroy(side);
    if (ev_fork) cudaEventDestroy(ev_fork);
    if (ev_join) cudaEventDestroy(ev_join);
  }

  gj_status analytic(Err& err, typename CplxT<T>::type* X, cudaStream_t st) {
    using C = typename CplxT<T>::type;
    cufftResult r;
    cufftSetStream(fftplan, st);
    if (sizeof(T) == 8) r = cufftExecZ2Z(fftplan, (cufftDoubleComplex*)X, (cufftDoubleComplex*)X, CUFFT_FORWARD);
    else r = cufftExecC2C(fftplan, (cufftComplex*)X, (cufftComplex*)X, CUFFT_FORWARD);
    if (r != CUFFT_SUCCESS) return err.set(GJ_ECUDA, "cufft forward failed (%d)", int(r));
    k_env_mask<T, C><<<512, 256, 0, st>>>(X, g.nt, size_t(fft_batch));
    if (sizeof(T) == 8) r = cufftExecZ2Z(fftplan, (cufftDoubleComplex*)X, (cufftDoubleComplex*)X, CUFFT_INVERSE);
    else r = cufftExecC2C(fftplan, (cufftComplex*)X, (cufftComplex*)X, CUFFT_INVERSE);
    if (r != CUFFT_SUCCESS) return err.set(GJ_ECUDA, "cufft inverse failed (%d)", int(r));
    return GJ_OK;
  }

  // Envelope / phase residual and misfit sums for shots [g0, g0+gn) (w_bozdag.m:16-54).
  gj_status env_residual(Err& err, Ctx& c, int g0, int gn, gj_misfit_kind mk, cudaStream_t st) {
    using C = typename CplxT<T>::type;
    const int nrr = std::max(nr, 1), nt = g.nt;
    const size_t tr = size_t(nrr) * nt, n = size_t(gn) * tr;
    const int batch = gn * nrr;
    if (fftplan && fft_batch != batch) { cufftDestroy(fftplan); fftplan = 0; }
    if (!fftplan) {
      int dims[1] = {nt};
      if (cufftPlanMany(&fftplan, 1, dims, nullptr, 1, nt, nullptr, 1, nt, sizeof(T) == 8 ? CUFFT_Z2Z : CUFFT_C2C,
                        batch) != CUFFT_SUCCESS)
        return err.set(GJ_ENOMEM, "cufftPlanMany(nt=%d, batch=%d) failed", nt, batch);
      fft_batch = batch;
    }
    GJ_TRY(envA.alloc(err, n * sizeof(C)));
    GJ_TRY(envAo.alloc(err, n * sizeof(C)));
    GJ_TRY(envG.alloc(err, n * sizeof(C)));
    GJ_TRY(envF.alloc(err, n * sizeof(T)));
    const T* d = dbuf.as<T>() + size_t(g0) * tr;
    const T* dob = dobsbuf.as<T>() + size_t(g0) * tr;
    k_env_to_complex<T, C><<<512, 256, 0, st>>>(d, envA.as<C>(), n);
    k_env_to_complex<T, C><<<512, 256, 0, st>>>(dob, envAo.as<C>(), n);
    GJ_TRY(analytic(err, envA.as<C>(), st));
    GJ_TRY(analytic(err, envAo.as<C>(), st));
    k_env_mid<T, C><<<dim3(64, gn), 256, 0, st>>>(d, envA.as<C>(), envAo.as<C>(), envF.as<T>(), envG.as<C>(), nt,
                                                 nrr, gn, int(mk), sums.as<double>() + 2 * g0);
    GJ_TRY(analytic(err, envG.as<C>(), st));
    k_env_final<T, C><<<512, 256, 0, st>>>(d, envF.as<T>(), envG.as<C>(), ebuf.as<T>() + size_t(g0) * tr, n,
                                           int(mk));
    c.launches += 10;
    GJ_CUDA(err, cudaGetLastError());
    return GJ_OK;
  }

  // Gaussian band filter of the residual traces of shots [g0, g0+gn)
  // (filt_gauss.m:16-47 on e_2d, w_update_e.m:69-70), in place in ebuf.
  DevBuf filtX, filtW, filtG;
  cufftHandle filtplan = 0;
  int filt_batch = 0, filt_ntp = 0;
  double filt_key[4] = {0, 0, 0, 0};
  gj_status filt_residual(Err& err, Ctx& c, const gj_w_opts& o, int g0, int gn, cudaStream_t st) {
    return filt_traces(err, c, o, ebuf.as<T>() + size_t(g0) * std::max(nr, 1) * g.nt, gn, st);
  }
  // The same filter in place on gn shots of traces x ([shot][r][t]).
  gj_status filt_traces(Err& err, Ctx& c, const gj_w_opts& o, T* x, int gn, cudaStream_t st) {
    using C = typename CplxT<T>::type;
    const int nrr = std::max(nr, 1), nt = g.nt;
    int ntp = 1;
    while (ntp < nt) ntp <<= 1;  // 2^nextpow2(nt)
    const int batch = gn * nrr;
    if (filtplan && (filt_batch != batch || filt_ntp != ntp)) { cufftDestroy(filtplan); filtplan = 0; }
    if (!filtplan) {
      int dims[1] = {ntp};
      if (cufftPlanMany(&filtplan, 1, dims, nullptr, 1, ntp, nullptr, 1, ntp, sizeof(T) == 8 ? CUFFT_Z2Z : CUFFT_C2C,
                        batch) != CUFFT_SUCCESS)
        return err.set(GJ_ENOMEM, "cufftPlanMany(n=%d, batch=%d) failed", ntp, batch);
      filt_batch = batch;
      filt_ntp = ntp;
    }
    const int steep = o.filt_steep > 0 ? o.filt_steep : 8;
    const double key[4] = {g.dt, o.filt_low, o.filt_high, double(steep)};
    if (!filtW.p || !filtG.p || std::memcmp(key, filt_key, sizeof key) != 0 || filtG.bytes < ntp * sizeof(T)) {
      // MATLAB tukeywin(nt, 0.1) and the fftshift-ed Gaussian of filt_gauss.m:26-33
      std::vector<T> win(nt), gk(ntp);
      const double r = 0.1, per = r / 2;
      const int tl = int(std::floor(per * (nt - 1))) + 1, th = nt - tl + 1;
      for (int t = 0; t < nt; ++t) {
        const double x = nt > 1 ? double(t) / (nt - 1) : 0.0;
        double v = 1.0;
        if (t < tl) v = 0.5 * (1 + std::cos(M_PI / per * (x - per)));
        else if (t >= th - 1) v = 0.5 * (1 + std::cos(M_PI / per * (x - 1 + per)));
        win[t] = T(v);
      }
      const double df = 1.0 / g.dt / ntp, width = o.filt_high - o.filt_low, middle = o.filt_low + 0.5 * width;
      for (int q = 0; q < ntp; ++q) {
        const double f = double(q - ntp / 2) * df;  // f = (-ntp/2 : ntp/2-1) df
        const double gq = std::exp(-std::pow(f - middle, steep) / ((df * 0.5) * std::pow(width, steep - 1)));
        gk[(q + ntp / 2) % ntp] = T(gq / ntp);      // fftshift, with the inverse FFT's 1/ntp
      }
      GJ_TRY(filtW.alloc(err, nt * sizeof(T)));
      GJ_TRY(filtG.alloc(err, ntp * sizeof(T)));
      GJ_CUDA(err, cudaMemcpyAsync(filtW.p, win.data(), nt * sizeof(T), cudaMemcpyHostToDevice, st));
      GJ_CUDA(err, cudaMemcpyAsync(filtG.p, gk.data(), ntp * sizeof(T), cudaMemcpyHostToDevice, st));
      GJ_CUDA(err, cudaStreamSynchronize(st));  // host vectors go out of scope
      std::memcpy(filt_key, key, sizeof key);
    }
    GJ_TRY(filtX.alloc(err, size_t(batch) * ntp * sizeof(C)));
    T* e = x;
    C* X = filtX.as<C>();
    k_filt_pre<T, C><<<512, 256, 0, st>>>(e, filtW.as<T>(), X, nt, ntp, size_t(batch));
    cufftSetStream(filtplan, st);
    cufftResult rr;
    if (sizeof(T) == 8) rr = cufftExecZ2Z(filtplan, (cufftDoubleComplex*)X, (cufftDoubleComplex*)X, CUFFT_FORWARD);
    else rr = cufftExecC2C(filtplan, (cufftComplex*)X, (cufftComplex*)X, CUFFT_FORWARD);
    if (rr != CUFFT_SUCCESS) return err.set(GJ_ECUDA, "cufft forward failed (%d)", int(rr));
    k_filt_mul<T, C><<<512, 256, 0, st>>>(X, filtG.as<T>(), ntp, size_t(batch));
    if (sizeof(T) == 8) rr = cufftExecZ2Z(filtplan, (cufftDoubleComplex*)X, (cufftDoubleComplex*)X, CUFFT_INVERSE);
    else rr = cufftExecC2C(filtplan, (cufftComplex*)X, (cufftComplex*)X, CUFFT_INVERSE);
    if (rr != CUFFT_SUCCESS) return err.set(GJ_ECUDA, "cufft inverse failed (%d)", int(rr));
    k_filt_post<T, C><<<512, 256, 0, st>>>(X, e, nt, ntp, size_t(batch));
    c.launches += 5;
    GJ_CUDA(err, cudaGetLastError());
    return GJ_OK;
  }

  // ---------------------------------------------------------------- groups
  // Shots are processed in groups of G: every group runs the whole gradient
  // (forward, residual, recompute, adjoint) before the next starts, so the
  // fields of one group can stay resident in L2.  State, checkpoint and
  // history buffers are sized for one group; traces and accumulators hold all
  // shots.
  int G = 0;
  struct GraphRec {
    cudaGraphExec_t exec = nullptr;
    std::unique_ptr<Marks> marks;
    long launches = 0;
    ~GraphRec() { if (exec) cudaGraphExecDestroy(exec); }
  };
  std::map<std::string, std::unique_ptr<GraphRec>> graphs;

  void drop_graphs() { graphs.clear(); }

  // Shot-group size.  Keeping the whole u history in HBM saves the recompute
  // pass (about a third of the work), so the default is the largest group
  // whose history fits the memory budget, as long as a group still fills the
  // GPU (at least 8 shots, or all of them); otherwise all shots at once with
  // checkpoints.
  int choose_group(const gj_w_opts& o, size_t free_bytes) const {
    if (o.shots_per_launch > 0) return std::min(o.shots_per_launch, nshots);
    if (const char* e = getenv("GJ_SHOTS_PER_GROUP")) {
      const int v = atoi(e);
      if (v > 0) return std::min(v, nshots);
    }
    if (o.ckpt_every > 0) return nshots;
    const size_t budget = o.mem_budget_bytes ? o.mem_budget_bytes : size_t(0.8 * double(free_bytes));
    const size_t bnd = band_on ? size_t(w.bsz) : 0;
    const size_t per_shot = (size_t(g.nt + 1 + (ring_on ? Kd : 0)) * (dn + bnd) + 4 * sstride) * sizeof(T);
    const int fit = int(std::min<size_t>(budget / std::max<size_t>(per_shot, 1), size_t(nshots)));
    if (fit >= nshots) return nshots;
    if (fit >= std::min(8, nshots)) {
      const int ngroups = (nshots + fit - 1) / fit;  // balance the groups
      return (nshots + ngroups - 1) / ngroups;
    }
    return nshots;
  }

  // Columns per block for a launch of `ns` shots: enough blocks for ~48 warps per SM.
  int tj_for(int ns) const {
    constexpr int V = VT<T>::V;
    const long bxs = (NX + 1 + 128 * V - 1) / (128 * V);
    int t = 64;
    while (t > 2 && bxs * ((NY + t) / t) * ns < 148L * 12) t /= 2;
    return t;
  }

  // Band kernels of the exact adjoint (w_band.cuh): band fields of a state
  // into a band slot, the adjoint band values of a state, band imaging.
  int band_blocks() const { return int(std::min<long>((w.bsz + 255) / 256, 4L * nsm)); }
  void band_rec(const T* state, T* slot, int gn, cudaStream_t st, long& nl) {
    k_band_rec<T><<<dim3(band_blocks(), gn), 256, 0, st>>>(w, state, sstride, fstride, slot);
    ++nl;
  }
  void band_adj(const T* state, T* slot, int gn, cudaStream_t st, long& nl) {
    k_band_adj<T><<<dim3(band_blocks(), gn), 256, 0, st>>>(w, state, sstride, fstride, slot);
    ++nl;
  }
  void band_image(const T* lam, const T* Fk0, int cnt, int gn, int shot0, int kahan, cudaStream_t st, long& nl) {
    const size_t sl = size_t(gn) * size_t(w.bsz);
    k_image_band<T><<<dim3(band_blocks(), gn), 256, 0, st>>>(w, lam, sl, Fk0, sl, cnt, bacc.as<T>(),
                                                             2 * size_t(w.bsz), shot0, kahan);
    ++nl;
  }

  // Enqueues the whole gradient of shots [g0, g0+gn) on stream st.
  // phase: 1 = forward (+ the L2 residual when l2), 2 = adjoint, 3 = both.
  gj_status enqueue_group(Err& err, Ctx& c, int g0, int gn, gj_adj_mode mode, int kahan,
                          const std::vector<std::pair<int, int>>& segs, bool full, long& nl, cudaStream_t st,
                          int phase = 3, bool l2 = true) {
    const int nrr = std::max(nr, 1), nt = g.nt;
    const size_t tr = size_t(nrr) * nt;
    constexpr int V = VT<T>::V;
    const int tjg = tj_for(gn);
    const dim3 grd((NX + 1 + 128 * V - 1) / (128 * V), (NY + 1 + tjg - 1) / tjg, gn);
    T* H = hist.as<T>();
    const size_t hs = dn;
    auto slot_ptr = [&](long k, long base) { return H + size_t(k - base) * gn * hs; };
    T* BH = bhist.as<T>();
    auto bslot = [&](long k, long base) { return BH + size_t(k - base) * gn * size_t(w.bsz); };
    const long* rec = recbuf.as<long>() + size_t(g0) * nrr;
    const int* nrs_d = nrsbuf.as<int>() + g0;
    const int* sel = selbuf.as<int>() + size_t(g0) * nrr;
    const int* nsel_d = nselbuf.as<int>() + g0;
    T* dgrp = dbuf.as<T>() + size_t(g0) * tr;
    T* egrp = ebuf.as<T>() + size_t(g0) * tr;
    T* A = fwdA.as<T>() + ld;
    T* B = fwdB.as<T>() + ld;
    if (phase & 1) {
    GJ_CUDA(err, cudaMemsetAsync(fwdA.p, 0, gn * sstride * sizeof(T), st));
    GJ_CUDA(err, cudaMemsetAsync(fwdB.p, 0, gn * sstride * sizeof(T), st));
    if (full) GJ_CUDA(err, cudaMemsetAsync(H, 0, gn * hs * sizeof(T), st));  // slot 0 = zero state
    if (full && band_on) GJ_CUDA(err, cudaMemsetAsync(BH, 0, gn * size_t(w.bsz) * sizeof(T), st));
    size_t segi = 0;
    // whole history kept and blocked passes chosen: D steps per launch, the
    // history and band history of every step written by the pass
    const TbCfg* tgc = nullptr;
    if (full && ring_on) {
      auto itg = tb_grad.find(gn);
      if (itg != tb_grad.end() && itg->second.D > 0) tgc = &itg->second;
    }
    for (int it = 0, nd = 0; tgc && it < nt; it += nd) {
      TbCfg qq = *tgc;
      qq.D = std::min(tgc->D, nt - it);
      nd = qq.D;
      if (!tb_tiles.count(tb_key(qq, gn))) return err.set(GJ_ECUDA, "blocked pass tables were not prepared");
      const bool tm = c.timer.begin(KK_TB_PASS, st, gn);
      GJ_TRY(launch_fwd_tb(err, A, B, it, gn, qq, nr > 0 ? dgrp : nullptr, nullptr, st, g0, slot_ptr(it + 1, 0),
                           size_t(gn) * hs, band_on ? bslot(it + 1, 0) : nullptr, size_t(gn) * size_t(w.bsz)));
      c.timer.end(tm, st);
      nl += last_kernels;
      std::swap(A, B);
    }
    for (int it = 0; !tgc && it < nt; ++it) {
      if (!full && segi < segs.size() && it == segs[segi].first) {
        GJ_CUDA(err, cudaMemcpyAsync(ckpt.as<T>() + segi * gn * sstride, A - ld, gn * sstride * sizeof(T),
                                     cudaMemcpyDeviceToDevice, st));
        ++segi;
      }
      StepArgs<T> a = step_args(A, B, it);
      a.shot0 = g0;
      if (full) { a.hist = slot_ptr(it + 1, 0); a.hstride = hs; }
      const bool tm = c.timer.begin(KK_FWD_STEP, st, gn);
      RecArgs<T> ra = rec_args(g0);
      if (ring_on && nr > 0) { ra.d = dgrp; ra.it = it; }  // receivers recorded inside the step
      if (ring_on && full && band_on) a.band = bslot(it + 1, 0);  // band history written inside the step
      GJ_TRY(launch_fwd(err, a, gn, st, ra));
      c.timer.end(tm, st);
      nl += last_kernels;
      if (!ring_on && full && band_on) band_rec(B, bslot(it + 1, 0), gn, st, nl);
      if (!ring_on) {
        k_record<T><<<dim3(1, gn), 128, 0, st>>>(B, sstride, rec, nrr, nrs_d, it, nt, dgrp, d_src + g0,
                                                 static_cast<T*>(nullptr), gn);
        ++nl;
      }
      std::swap(A, B);
    }
    if (l2) {
      k_residual<T><<<dim3(64, gn), 256, 0, st>>>(dgrp, dobsbuf.as<T>() + size_t(g0) * tr, egrp, tr,
                                                  sums.as<double>() + 2 * g0);
      ++nl;
    }
    }  // phase 1
    if (!(phase & 2)) { GJ_CUDA(err, cudaGetLastError()); return GJ_OK; }
    A = fwdA.as<T>() + ld;
    B = fwdB.as<T>() + ld;
    T* LA = adjA.as<T>() + ld;
    T* LB = adjB.as<T>() + ld;
    GJ_CUDA(err, cudaMemsetAsync(adjA.p, 0, gn * sstride * sizeof(T), st));
    GJ_CUDA(err, cudaMemsetAsync(adjB.p, 0, gn * sstride * sizeof(T), st));
    for (int sidx = int(segs.size()) - 1; sidx >= 0; --sidx) {
      const int s0 = segs[sidx].first, s1 = segs[sidx].second;
      long base = 0;
      if (!full) {
        base = s0;
        GJ_CUDA(err, cudaMemcpyAsync(A - ld, ckpt.as<T>() + size_t(sidx) * gn * sstride, gn * sstride * sizeof(T),
                                     cudaMemcpyDeviceToDevice, st));
        k_domain_copy<T><<<dim3(64, gn), 256, 0, st>>>(w, A, sstride, slot_ptr(s0, base), hs, gn);
        ++nl;
        if (band_on) band_rec(A, bslot(s0, base), gn, st, nl);
        const int iend = std::min(s1 + 1, nt);
        for (int it = s0; it < iend; ++it) {
          StepArgs<T> a = step_args(A, B, it);
          a.shot0 = g0;
          a.hist = slot_ptr(it + 1, base); a.hstride = hs;
          if (ring_on && band_on) a.band = bslot(it + 1, base);
          const bool tm = c.timer.begin(KK_FWD_STEP, st, gn);
          GJ_TRY(launch_fwd(err, a, gn, st));
          c.timer.end(tm, st);
          nl += last_kernels;
          if (!ring_on && band_on) band_rec(B, bslot(it + 1, base), gn, st, nl);
          std::swap(A, B);
        }
      }
      int win = 0;  // adjoint steps in the l ring not yet imaged
      for (int k = s1; k >= s0 + 1; --k) {  // k = history slot of forward step k-1
        const int itf = k - 1;
        if (mode == GJ_ADJ_REFERENCE && ring_on) {
          // w_grad.m:70-87: receivers hard-set, a sigma-flipped source-free step
          // (the forward ring kernel with the flipped coefficients), its Ez at the
          // model nodes into the ring; imaging every Kd steps (k_image_ref)
          if (nr > 0) {
            k_inject_set<T><<<dim3(1, gn), 128, 0, st>>>(LA, sstride, rec, sel, nrr, nsel_d, egrp, itf, nt, gn);
            ++nl;
          }
          StepArgs<T> a = step_args(LA, LB, itf);
          a.shot0 = g0;
          a.src = nosrc.as<long>();
          a.hist = lring.as<T>() + size_t(win) * gn * hs; a.hstride = hs;
          const bool tm = c.timer.begin(KK_REF_STEP, st, gn);
          GJ_TRY(launch_fwd(err, a, gn, st, RecArgs<T>{}, &wr));
          c.timer.end(tm, st);
          nl += last_kernels;
          ++win;
          if (win == Kd || k == s0 + 1) {
            const bool ti = c.timer.begin(KK_IMAGE, st, gn);
            const int ng = (w.di0 + g.m - 1) / V - w.di0 / V + 1;
            const int nblk = int(std::min<long>((long(ng) * g.n + 255) / 256, 4L * nsm));
            k_image_ref<T><<<dim3(nblk, gn), 256, 0, st>>>(w, lring.as<T>(), size_t(gn) * hs, H, base,
                                                           size_t(gn) * hs,
                                                           k + win - 1, win, nt, T(1.0 / g.dt), hs, acc.as<T>(),
                                                           4 * dn, g0, kahan);
            c.timer.end(ti, st);
            win = 0;
            ++nl;
          }
        } else if (mode == GJ_ADJ_REFERENCE) {
          if (nr > 0)
            k_inject_set<T><<<dim3(1, gn), 128, 0, st>>>(LA, sstride, rec, sel, nrr, nsel_d, egrp, itf, nt, gn);
          StepArgs<T> a = step_args(LA, LB, itf);
          a.shot0 = g0; a.tj = tjg; a.hist = nullptr;
          int k0, k1, k2; double c0, c1, c2;
          ddt_stencil(k, k0, k1, k2, c0, c1, c2);
          a.u0 = slot_ptr(k0, base); a.u1 = slot_ptr(k1, base); a.u2 = slot_ptr(k2, base);
          a.c0 = T(c0); a.c1 = T(c1); a.c2 = T(c2);
          a.uk = slot_ptr(k, base);
          a.hstride = hs;
          a.acc = acc.as<T>(); a.astride = 4 * dn; a.kahan = kahan;
          const bool tm = c.timer.begin(KK_REF_STEP, st, gn);
          k_stepv<T, 1><<<grd, 128, 0, st>>>(wr, a);
          c.timer.end(tm, st);
          nl += 2;
        } else if (ring_on) {
          // the adjoint source of step k is added by step k+1's kernel; only the
          // first adjoint step (k = nt) needs its own injection
          if (nr > 0 && k == nt) {
            k_inject_add<T><<<dim3(1, gn), 128, 0, st>>>(LA, sstride, rec, nrr, nrs_d, egrp, itf, nt, gn);
            ++nl;
          }
          RecArgs<T> ra = rec_args(g0);
          if (nr > 0 && itf - 1 >= 0) { ra.e = egrp; ra.kinj = itf - 1; }
          AdjRingArgs<T> a{};
          a.A = LA; a.B = LB; a.fstride = fstride; a.sstride = sstride; a.shot0 = g0;
          a.lout = lring.as<T>() + size_t(win) * gn * hs; a.hstride = hs;
          if (band_on) a.band = blam.as<T>() + size_t(win) * gn * size_t(w.bsz);  // written inside the step
          const bool tm = c.timer.begin(KK_ADJ_STEP, st, gn);
          GJ_TRY(launch_adjr(err, a, gn, st, ra));
          c.timer.end(tm, st);
          nl += last_kernels;
          ++win;
          if (win == Kd || k == s0 + 1) {
            // imaging over the steps k + win - 1 .. k
            const bool ti = c.timer.begin(KK_IMAGE, st, gn);
            const int ng = (w.di0 + g.m - 1) / V - w.di0 / V + 1;
            const int nblk = int(std::min<long>((long(ng) * g.n + 255) / 256, 4L * nsm));
            k_image<T><<<dim3(nblk, gn), 256, 0, st>>>(w, lring.as<T>(), size_t(gn) * hs,
                                                       slot_ptr(k + win - 1, base), size_t(gn) * hs, win, hs,
                                                       acc.as<T>(), 4 * dn, g0, kahan);
            if (band_on) band_image(blam.as<T>(), bslot(k + win - 1, base), win, gn, g0, kahan, st, nl);
            c.timer.end(ti, st);
            win = 0;
            ++nl;
          }
        } else {
          if (nr > 0)
            k_inject_add<T><<<dim3(1, gn), 128, 0, st>>>(LA, sstride, rec, nrr, nrs_d, egrp, itf, nt, gn);
          AdjArgs<T> a{};
          a.A = LA; a.B = LB; a.fstride = fstride; a.sstride = sstride; a.shot0 = g0; a.tj = tjg;
          a.ek = slot_ptr(k, base); a.ekm1 = slot_ptr(k - 1, base); a.hstride = hs;
          a.acc = acc.as<T>(); a.astride = 4 * dn; a.kahan = kahan;
          if (band_on) {
            band_adj(LA, blam.as<T>(), gn, st, nl);
            band_image(blam.as<T>(), bslot(k, base), 1, gn, g0, kahan, st, nl);
          }
          const bool tm = c.timer.begin(KK_ADJ_STEP, st, gn);
          k_adj_stepv<T><<<grd, 128, 0, st>>>(w, a);
          c.timer.end(tm, st);
          nl += 2;
        }
        std::swap(LA, LB);
      }
    }
    GJ_CUDA(err, cudaGetLastError());
    return GJ_OK;
  }

  // Memory plan of a gradient call: shot groups G, checkpoint interval K,
  // and the history, checkpoint, adjoint-state and ring buffers (carved from
  // the pool when pool_p is set, as gj_w_gradient_batch does); then the
  // autotuner for the launch sizes.  avail = 0 measures the free memory.
  std::vector<std::pair<int, int>> segs_;
  bool full_ = false;
  unsigned char* pool_p = nullptr;  // batch: next free byte of the shared pool
  gj_status take(Err& err, DevBuf& b, size_t bytes) {
    if (!pool_p) return b.alloc(err, bytes);
    b.borrow(pool_p, bytes);
    pool_p += (bytes + 255) / 256 * 256;
    return GJ_OK;
  }
  gj_status plan_buffers(Err& err, const gj_w_opts& o, size_t avail, gj_adj_mode mode, cudaStream_t st) {
    ring_on = ring_nth > 0 && !o.no_ring;
    band_on = mode == GJ_ADJ_EXACT;
    // memory plan for one group
    size_t free_b = avail, total_b = 0;
    (void)total_b;
    if (!avail) GJ_CUDA(err, cudaMemGetInfo(&free_b, &total_b));
    const size_t owned = hist.bytes + ckpt.bytes + bhist.bytes + blam.bytes +
                         (G > 0 ? 4 * size_t(G) * sstride * sizeof(T) : 0);
    const int Gnew = choose_group(o, free_b + owned);
    const int ns_save = nshots;
    nshots = Gnew;  // choose_k sizes buffers per group
    const int Kold = K;
    choose_k(o, free_b + owned);
    nshots = ns_save;
    if (Gnew != G || K != Kold) drop_graphs();
    G = Gnew;
    const bool full = (K >= g.nt);
    std::vector<std::pair<int, int>> segs = segments();
    int maxlen = 0;
    for (auto& q : segs) maxlen = std::max(maxlen, q.second - q.first);
    hist_slots = full ? size_t(g.nt + 1) : size_t(maxlen + 3);
    const size_t hbytes = hist_slots * G * dn * sizeof(T);
    const size_t cbytes = full ? 0 : segs.size() * G * sstride * sizeof(T);
    void* old[8] = {hist.p, ckpt.p, fwdA.p, adjA.p, acc.p, bhist.p, blam.p, bacc.p};
    if (!band_on) { bhist.release(); blam.release(); }
    GJ_TRY(take(err, hist, hbytes));
    if (!full) GJ_TRY(take(err, ckpt, cbytes));
    GJ_TRY(fwdA.alloc(err, size_t(G) * sstride * sizeof(T)));
    GJ_TRY(fwdB.alloc(err, size_t(G) * sstride * sizeof(T)));
    GJ_TRY(take(err, adjA, size_t(G) * sstride * sizeof(T)));
    GJ_TRY(take(err, adjB, size_t(G) * sstride * sizeof(T)));
    GJ_TRY(acc.alloc(err, size_t(nshots) * 4 * dn * sizeof(T)));
    if (band_on) {
      GJ_TRY(take(err, bhist, hist_slots * G * size_t(w.bsz) * sizeof(T)));
      GJ_TRY(take(err, blam, size_t(ring_on ? Kd : 1) * G * size_t(w.bsz) * sizeof(T)));
      GJ_TRY(bacc.alloc(err, size_t(nshots) * 2 * size_t(w.bsz) * sizeof(T)));
    }
    if (ring_on) {
      const void* lold = lring.p;
      GJ_TRY(take(err, lring, size_t(Kd) * G * dn * sizeof(T)));
      if (lring.p != lold) {
        drop_graphs();
        // rows that no lane writes stay zero
        GJ_CUDA(err, cudaMemsetAsync(lring.p, 0, size_t(Kd) * G * dn * sizeof(T), st));
      }
    }
    void* nw[8] = {hist.p, ckpt.p, fwdA.p, adjA.p, acc.p, bhist.p, blam.p, bacc.p};
    for (int q = 0; q < 8; ++q)
      if (old[q] != nw[q]) { drop_graphs(); break; }
    if (ring_on) {
      GJ_TRY(autotune(err, G, st));
      if (nshots % G) GJ_TRY(autotune(err, nshots % G, st));
    }
    const std::map<int, TbCfg> tb_prev = tb_grad;
    tb_grad.clear();
    // off unless GJ_TB_GRAD=1: on the benchmark grid the passes' history and
    // band-history stores made a blocked step slower than a ring step
    const char* tg = getenv("GJ_TB_GRAD");
    if (ring_on && full && tg && atoi(tg) != 0) {
      // tuned (and the pass tables built) here, outside any graph capture
      for (int gn : {G, nshots % G}) {
        if (gn < 1 || tb_grad.count(gn)) continue;
        TbCfg q;
        GJ_TRY(tb_select(err, gn, st, q));
        if (q.D > 0) {
          GJ_TRY(tb_prepare(err, q, gn));
          if (g.nt % q.D) { TbCfg r = q; r.D = g.nt % q.D; GJ_TRY(tb_prepare(err, r, gn)); }
        }
        tb_grad[gn] = q;
      }
    }
    if (!(tb_grad == tb_prev)) drop_graphs();  // captured forwards of another pass configuration
    segs_ = segs;
    full_ = full;
    return GJ_OK;
  }

  // ------------------------------------------------------------ batch
  // The whole gradient of all shots after plan_buffers (L2, no residual
  // filter): accumulators cleared, then every shot group; capturable.
  gj_status enqueue_all(Err& err, Ctx& c, gj_adj_mode mode, int kahan, cudaStream_t st, long& nl) {
    // a ring in a shared pool holds what the pool's previous user left there
    if (ring_on && !lring.owned) GJ_CUDA(err, cudaMemsetAsync(lring.p, 0, size_t(Kd) * G * dn * sizeof(T), st));
    GJ_CUDA(err, cudaMemsetAsync(sums.p, 0, 2 * nshots * sizeof(double), st));
    GJ_CUDA(err, cudaMemsetAsync(acc.p, 0, nshots * 4 * dn * sizeof(T), st));
    if (band_on) GJ_CUDA(err, cudaMemsetAsync(bacc.p, 0, size_t(nshots) * 2 * size_t(w.bsz) * sizeof(T), st));
    for (int g0 = 0; g0 < nshots; g0 += G) {
      const int gn = std::min(G, nshots - g0);
      if (ring_on) select_cfg(gn);
      GJ_TRY(enqueue_group(err, c, g0, gn, mode, kahan, segs_, full_, nl, st));
    }
    return GJ_OK;
  }
  // Pool bytes plan_buffers carves with groups of `shots` shots (0: all in
  // one group) and checkpoint interval Kc (Kc >= nt: the whole history kept).
  size_t pool_need(int Kc, bool exact, int shots = 0) const {
    auto al = [](size_t b) { return (b + 255) / 256 * 256; };
    const size_t Gs = size_t(shots > 0 ? shots : nshots), sz = sizeof(T), bs = exact ? size_t(w.bsz) : 0;
    const bool full = Kc >= g.nt;
    const size_t nseg = full ? 0 : size_t((g.nt + Kc - 1) / Kc);
    const size_t slots = full ? size_t(g.nt + 1) : size_t(Kc + 4);
    size_t b = al(slots * Gs * dn * sz) + al(nseg * Gs * sstride * sz) + 2 * al(Gs * sstride * sz) +
               al(size_t(Kd) * Gs * dn * sz);
    if (exact) b += al(slots * Gs * bs * sz) + al(size_t(Kd) * Gs * bs * sz);
    return b + 4096;
  }
  // Checkpoint interval of least pool memory.
  int best_k(bool exact) const {
    int kb = g.nt;
    size_t nb = pool_need(g.nt, exact);
    for (int k = 8; k < g.nt; k += std::max(1, k / 8)) {
      const size_t b = pool_need(k, exact);
      if (b < nb) { nb = b; kb = k; }
    }
    return kb;
  }

  // e_given: `dobs` holds the adjoint sources themselves (per shot nt x nr),
  // the backward half of gj_w_backward: no residual, no misfit.
  gj_status gradient(Err& err, Ctx& c, const void* eps, const void* sig, bool dev_in, const void* dobs,
                     bool dev_dobs, gj_adj_mode mode, gj_misfit_kind mk, const gj_w_opts& o, void* geps,
                     void* gsig, bool dev_out, double* misfit_out, double* d_out, double* e_out, cudaStream_t st,
                     bool e_given = false) {
    GJ_TRY(stage_inputs(err, c, eps, sig, dev_in, dobs, dev_dobs, st));
    if (e_given) mk = GJ_MISFIT_L2;
    if (o.plain) {
      if (mk != GJ_MISFIT_L2) return err.set(GJ_EUNSUPPORTED, "the plain form supports the L2 misfit only");
      if (o.filt_high > o.filt_low) return err.set(GJ_EUNSUPPORTED, "the plain form has no residual filter");
      return gradient_plain(err, c, mode, o, geps, gsig, dev_out, misfit_out, d_out, e_out, st, e_given);
    }
    const bool env = (mk != GJ_MISFIT_L2);
    const bool filt = o.filt_high > o.filt_low;
    GJ_TRY(plan_buffers(err, o, 0, mode, st));
    const std::vector<std::pair<int, int>> segs = segs_;
    const bool full = full_;
    const int kahan = o.no_kahan ? 0 : 1;
    GJ_CUDA(err, cudaMemsetAsync(sums.p, 0, 2 * nshots * sizeof(double), st));
    GJ_CUDA(err, cudaMemsetAsync(acc.p, 0, nshots * 4 * dn * sizeof(T), st));
    if (band_on) GJ_CUDA(err, cudaMemsetAsync(bacc.p, 0, size_t(nshots) * 2 * size_t(w.bsz) * sizeof(T), st));
    long nl = 0;
    for (int g0 = 0; g0 < nshots; g0 += G) {
      const int gn = std::min(G, nshots - g0);
      if (ring_on) select_cfg(gn);
      if (env || filt || e_given) {
        // forward, residual (envelope: cuFFT) or the given adjoint sources,
        // band filter (cuFFT), adjoint: launched directly
        Marks m;
        c.timer.cur = &m;
        gj_status rs = enqueue_group(err, c, g0, gn, mode, kahan, segs, full, nl, st, 1, !env && !e_given);
        if (rs == GJ_OK && e_given) {
          const size_t tr = size_t(std::max(nr, 1)) * g.nt;
          if (cudaMemcpyAsync(ebuf.as<T>() + size_t(g0) * tr, dobsbuf.as<T>() + size_t(g0) * tr,
                              size_t(gn) * tr * sizeof(T), cudaMemcpyDeviceToDevice, st) != cudaSuccess)
            rs = err.set(GJ_ECUDA, "copy of the adjoint sources failed");
        }
        if (rs == GJ_OK && env) rs = env_residual(err, c, g0, gn, mk, st);
        if (rs == GJ_OK && filt) rs = filt_residual(err, c, o, g0, gn, st);
        if (rs == GJ_OK) rs = enqueue_group(err, c, g0, gn, mode, kahan, segs, full, nl, st, 2, false);
        c.timer.close(st);
        c.timer.cur = nullptr;
        GJ_TRY(rs);
        GJ_CUDA(err, cudaStreamSynchronize(st));
        c.timer.collect(m);
        continue;
      }
      if (o.no_graph) {
        Marks m;
        c.timer.cur = &m;
        gj_status rs = enqueue_group(err, c, g0, gn, mode, kahan, segs, full, nl, st);
        c.timer.close(st);
        c.timer.cur = nullptr;
        GJ_TRY(rs);
        GJ_CUDA(err, cudaStreamSynchronize(st));
        c.timer.collect(m);
        continue;
      }
      char kb[160];
      snprintf(kb, sizeof kb, "%d/%d/%d/%d/%d/%d/%d/%d/%d/%d.%d.%d.%d.%d", g0, gn, int(mode), kahan, K, G,
               c.timer.on ? 1 : 0, ring_on ? 1 : 0, Kd, rc.S, rc.SF, rc.RWG, rc.tjF, rc.tjS);
      snprintf(kb + strlen(kb), sizeof kb - strlen(kb), "/%d.%d.%d.%d.%d", rca.S, rca.SF, rca.RWG, rca.tjF, rca.tjS);
      auto itg = graphs.find(kb);
      if (itg == graphs.end()) {
        auto rec = std::make_unique<GraphRec>();
        rec->marks = std::make_unique<Marks>();
        cudaStream_t cs;
        GJ_CUDA(err, cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
        GJ_CUDA(err, cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
        c.timer.cur = rec->marks.get();
        long cnt = 0;
        gj_status rs = enqueue_group(err, c, g0, gn, mode, kahan, segs, full, cnt, cs);
        c.timer.close(cs);
        c.timer.cur = nullptr;
        cudaGraph_t graph = nullptr;
        cudaError_t ce = cudaStreamEndCapture(cs, &graph);
        cudaStreamDestroy(cs);
        GJ_TRY(rs);
        if (ce != cudaSuccess) return err.set(GJ_ECUDA, "graph capture failed: %s", cudaGetErrorString(ce));
        ce = cudaGraphInstantiate(&rec->exec, graph, cudaGraphInstantiateFlagUseNodePriority);
        cudaGraphDestroy(graph);
        if (ce != cudaSuccess) return err.set(GJ_ECUDA, "graph instantiate failed: %s", cudaGetErrorString(ce));
        rec->launches = cnt;
        itg = graphs.emplace(kb, std::move(rec)).first;
      }
      GJ_CUDA(err, cudaGraphLaunch(itg->second->exec, st));
      nl += itg->second->launches;
      if (c.timer.on) {
        GJ_CUDA(err, cudaStreamSynchronize(st));
        c.timer.collect(*itg->second->marks);
      }
    }
    c.launches += nl;
    std::vector<double> hsums(2 * nshots);
    GJ_CUDA(err, cudaMemcpyAsync(hsums.data(), sums.p, 2 * nshots * sizeof(double), cudaMemcpyDeviceToHost, st));
    return finish(err, c, mode, o, geps, gsig, dev_out, misfit_out, d_out, e_out, hsums, st);
  }

  // The plain form: one half-step per launch, one thread per node, one shot at a
  // time, full u history in HBM when it fits (else the same checkpointing).
  gj_status gradient_plain(Err& err, Ctx& c, gj_adj_mode mode, const gj_w_opts& o, void* geps, void* gsig,
                           bool dev_out, double* misfit_out, double* d_out, double* e_out, cudaStream_t st,
                           bool e_given = false) {
    const int nrr = std::max(nr, 1), nt = g.nt;
    const size_t tr = size_t(nrr) * nt;
    size_t free_b = 0, total_b = 0;
    GJ_CUDA(err, cudaMemGetInfo(&free_b, &total_b));
    // per-shot sizing: pretend a single shot
    band_on = mode == GJ_ADJ_EXACT;
    const int ns_save = nshots;
    nshots = 1;
    choose_k(o, free_b + hist.bytes + ckpt.bytes + bhist.bytes + blam.bytes);
    nshots = ns_save;
    const bool full = (K >= nt);
    std::vector<std::pair<int, int>> segs = segments();
    int maxlen = 0;
    for (auto& q : segs) maxlen = std::max(maxlen, q.second - q.first);
    hist_slots = full ? size_t(nt + 1) : size_t(maxlen + 3);
    GJ_TRY(hist.alloc(err, hist_slots * dn * sizeof(T)));
    if (!full) GJ_TRY(ckpt.alloc(err, segs.size() * sstride * sizeof(T)));
    GJ_TRY(adjA.alloc(err, sstride * sizeof(T)));
    GJ_TRY(acc.alloc(err, size_t(nshots) * 4 * dn * sizeof(T)));
    GJ_TRY(scratch.alloc(err, 5 * fstride * sizeof(T)));
    if (band_on) {
      GJ_TRY(bhist.alloc(err, hist_slots * size_t(w.bsz) * sizeof(T)));
      GJ_TRY(blam.alloc(err, size_t(w.bsz) * sizeof(T)));
      GJ_TRY(bacc.alloc(err, size_t(nshots) * 2 * size_t(w.bsz) * sizeof(T)));
      GJ_CUDA(err, cudaMemsetAsync(bacc.p, 0, size_t(nshots) * 2 * size_t(w.bsz) * sizeof(T), st));
    }
    GJ_CUDA(err, cudaMemsetAsync(acc.p, 0, nshots * 4 * dn * sizeof(T), st));
    GJ_CUDA(err, cudaMemsetAsync(scratch.p, 0, 5 * fstride * sizeof(T), st));
    T* px = scratch.as<T>() + ld; T* py = px + fstride; T* lm = py + fstride; T* qx = lm + fstride; T* qy = qx + fstride;
    std::vector<T> hcezj(nshots), hwav(size_t(nshots) * nt);
    GJ_CUDA(err, cudaMemcpyAsync(hcezj.data(), d_cezj, nshots * sizeof(T), cudaMemcpyDeviceToHost, st));
    GJ_CUDA(err, cudaMemcpyAsync(hwav.data(), d_wav, hwav.size() * sizeof(T), cudaMemcpyDeviceToHost, st));
    GJ_CUDA(err, cudaStreamSynchronize(st));
    GJ_CUDA(err, cudaMemsetAsync(sums.p, 0, 2 * nshots * sizeof(double), st));
    const dim3 blk(32, 8), grd((NX + 1 + 31) / 32, (NY + 1 + 7) / 8);
    T* H = hist.as<T>();
    auto slot = [&](long k, long base) { return H + size_t(k - base) * dn; };
    auto bslot = [&](long k, long base) { return band_on ? bhist.as<T>() + size_t(k - base) * size_t(w.bsz) : nullptr; };
    long nlb = 0;  // band kernel launches
    T* S = fwdA.as<T>() + ld;  // shot state (in place)
    T* L = adjA.as<T>() + ld;
    Marks marks;
    c.timer.cur = &marks;
    for (int s = 0; s < nshots; ++s) {
      const long src = sh[s].src;
      auto fwd_step = [&](int it, T* hslot, T* bsl) {
        const bool tm = c.timer.begin(KK_PLAIN, st);
        k_plain_h<T><<<grd, blk, 0, st>>>(w, S, fstride);
        k_plain_e<T><<<grd, blk, 0, st>>>(w, S, fstride, src, hcezj[s] * hwav[size_t(s) * nt + it], hslot);
        if (bsl) band_rec(S, bsl, 1, st, nlb);
        c.timer.end(tm, st);
        c.launches += 2;
      };
      GJ_CUDA(err, cudaMemsetAsync(S - ld, 0, sstride * sizeof(T), st));
      if (full) GJ_CUDA(err, cudaMemsetAsync(H, 0, dn * sizeof(T), st));
      if (full && band_on) GJ_CUDA(err, cudaMemsetAsync(bhist.p, 0, size_t(w.bsz) * sizeof(T), st));
      size_t segi = 0;
      for (int it = 0; it < nt; ++it) {
        if (!full && segi < segs.size() && it == segs[segi].first) {
          GJ_CUDA(err, cudaMemcpyAsync(ckpt.as<T>() + segi * sstride, S - ld, sstride * sizeof(T),
                                       cudaMemcpyDeviceToDevice, st));
          ++segi;
        }
        fwd_step(it, full ? slot(it + 1, 0) : nullptr, full ? bslot(it + 1, 0) : nullptr);
        k_record<T><<<dim3(1, 1), 128, 0, st>>>(S, sstride, recbuf.as<long>() + size_t(s) * nrr, nrr,
                                                nrsbuf.as<int>() + s, it, nt, dbuf.as<T>() + size_t(s) * tr, d_src + s,
                                                static_cast<T*>(nullptr), 1);
        ++c.launches;
      }
      if (e_given) {
        GJ_CUDA(err, cudaMemcpyAsync(ebuf.as<T>() + size_t(s) * tr, dobsbuf.as<T>() + size_t(s) * tr,
                                     tr * sizeof(T), cudaMemcpyDeviceToDevice, st));
      } else {
        k_residual<T><<<dim3(64, 1), 256, 0, st>>>(dbuf.as<T>() + size_t(s) * tr, dobsbuf.as<T>() + size_t(s) * tr,
                                                    ebuf.as<T>() + size_t(s) * tr, tr, sums.as<double>() + 2 * s);
        ++c.launches;
      }
      GJ_CUDA(err, cudaMemsetAsync(L - ld, 0, sstride * sizeof(T), st));
      T* A_ = acc.as<T>() + size_t(s) * 4 * dn;
      for (int sidx = int(segs.size()) - 1; sidx >= 0; --sidx) {
        const int s0 = segs[sidx].first, s1 = segs[sidx].second;
        long base = 0;
        if (!full) {
          base = s0;
          GJ_CUDA(err, cudaMemcpyAsync(S - ld, ckpt.as<T>() + size_t(sidx) * sstride, sstride * sizeof(T),
                                       cudaMemcpyDeviceToDevice, st));
          k_domain_copy<T><<<dim3(64, 1), 256, 0, st>>>(w, S, sstride, slot(s0, base), dn, 1);
          ++c.launches;
          if (band_on) band_rec(S, bslot(s0, base), 1, st, nlb);
          for (int it = s0; it < std::min(s1 + 1, nt); ++it) fwd_step(it, slot(it + 1, base), bslot(it + 1, base));
        }
        for (int k = s1; k >= s0 + 1; --k) {
          const int itf = k - 1;
          const bool tm = c.timer.begin(KK_PLAIN, st);
          if (mode == GJ_ADJ_REFERENCE) {
            k_inject_set<T><<<dim3(1, 1), 128, 0, st>>>(L, sstride, recbuf.as<long>() + size_t(s) * nrr,
                                                        selbuf.as<int>() + size_t(s) * nrr, nrr, nselbuf.as<int>() + s,
                                                        ebuf.as<T>() + size_t(s) * tr, itf, nt, 1);
            k_plain_h<T><<<grd, blk, 0, st>>>(wr, L, fstride);
            k_plain_e<T><<<grd, blk, 0, st>>>(wr, L, fstride, -1, T(0), static_cast<T*>(nullptr));
            int k0, k1, k2; double c0, c1, c2;
            ddt_stencil(k, k0, k1, k2, c0, c1, c2);
            k_plain_img_ref<T><<<256, 256, 0, st>>>(wr, L, slot(k0, base), slot(k1, base), slot(k2, base), T(c0),
                                                    T(c1), T(c2), slot(k, base), A_);
            c.launches += 4;
          } else {
            k_inject_add<T><<<dim3(1, 1), 128, 0, st>>>(L, sstride, recbuf.as<long>() + size_t(s) * nrr, nrr,
                                                        nrsbuf.as<int>() + s, ebuf.as<T>() + size_t(s) * tr, itf, nt, 1);
            if (band_on) {
              band_adj(L, blam.as<T>(), 1, st, nlb);
              band_image(blam.as<T>(), bslot(k, base), 1, 1, s, 0, st, nlb);
            }
            k_plain_adj_e<T><<<grd, blk, 0, st>>>(w, L, fstride, px, py, lm, slot(k, base), slot(k - 1, base), A_);
            k_plain_adj_h<T><<<grd, blk, 0, st>>>(w, L, fstride, px, py, qx, qy);
            k_plain_adj_assemble<T><<<grd, blk, 0, st>>>(w, L, lm, qx, qy);
            c.launches += 4;
          }
          c.timer.end(tm, st);
        }
      }
    }
    c.timer.close(st);
    c.timer.cur = nullptr;
    c.launches += nlb;
    GJ_CUDA(err, cudaGetLastError());
    std::vector<double> hsums(2 * nshots);
    GJ_CUDA(err, cudaMemcpyAsync(hsums.data(), sums.p, 2 * nshots * sizeof(double), cudaMemcpyDeviceToHost, st));
    gj_status r = finish(err, c, mode, o, geps, gsig, dev_out, misfit_out, d_out, e_out, hsums, st);
    c.timer.collect(marks);
    return r;
  }

  // ------------------------------------------------------------ w_grad only
  gj_status grad_only(Err& err, Ctx& c, const double* eps, const double* sig, const double* e,
                      const double* u, double* gout, double* amax) {
    cudaStream_t st = 0;
    DevBuf mh;
    GJ_TRY(mh.alloc(err, 2 * mn * sizeof(double)));
    GJ_CUDA(err, cudaMemcpy(mh.as<double>(), eps, mn * sizeof(double), cudaMemcpyHostToDevice));
    GJ_CUDA(err, cudaMemcpy(mh.as<double>() + mn, sig, mn * sizeof(double), cudaMemcpyHostToDevice));
    GJ_TRY(build<double>(err, c, mh.as<double>(), mh.as<double>() + mn, st));
    const int nrr = std::max(nr, 1), nt = g.nt;
    // e: host nt x nr -> device [r][t]
    std::vector<T> he(size_t(nrr) * nt, T(0));
    for (int r = 0; r < nrs[0]; ++r)
      for (int t = 0; t < nt; ++t) he[size_t(r) * nt + t] = T(e[size_t(r) * nt + t]);
    GJ_CUDA(err, cudaMemcpy(ebuf.p, he.data(), he.size() * sizeof(T), cudaMemcpyHostToDevice));
    // u: host m x n x nt -> device slots 1..nt (slot 0 unused)
    GJ_TRY(hist.alloc(err, size_t(nt + 1) * dn * sizeof(T)));
    {
      // host m x n x nt -> device slots 1..nt in the domain-node layout
      std::vector<T> hu(size_t(nt) * dn, T(0));
      for (int t = 0; t < nt; ++t)
        for (int b = 0; b < g.n; ++b)
          for (int a_ = 0; a_ < g.m; ++a_)
            hu[size_t(t) * dn + size_t(b) * hld + w.di0 - hr0 + a_] = T(u[size_t(t) * mn + size_t(b) * g.m + a_]);
      GJ_CUDA(err, cudaMemcpy(hist.as<T>() + dn, hu.data(), hu.size() * sizeof(T), cudaMemcpyHostToDevice));
    }
    GJ_TRY(adjA.alloc(err, sstride * sizeof(T)));
    GJ_TRY(adjB.alloc(err, sstride * sizeof(T)));
    GJ_TRY(acc.alloc(err, 4 * dn * sizeof(T)));
    GJ_CUDA(err, cudaMemset(adjA.p, 0, sstride * sizeof(T)));
    GJ_CUDA(err, cudaMemset(adjB.p, 0, sstride * sizeof(T)));
    GJ_CUDA(err, cudaMemset(acc.p, 0, 4 * dn * sizeof(T)));
    T* LA = adjA.as<T>() + ld;
    T* LB = adjB.as<T>() + ld;
    constexpr int V = VT<T>::V;
    const int tjf = tj_for(1);
    const dim3 grd((NX + 1 + 128 * V - 1) / (128 * V), (NY + 1 + tjf - 1) / tjf, 1);
    for (int k = nt; k >= 1; --k) {
      if (nr > 0)
        k_inject_set<T><<<dim3(1, 1), 128, 0, st>>>(LA, sstride, recbuf.as<long>(), selbuf.as<int>(), nrr,
                                                    nselbuf.as<int>(), ebuf.as<T>(), k - 1, nt, 1);
      StepArgs<T> a = step_args(LA, LB, k - 1);
      T* uk = hist.as<T>() + size_t(k) * dn;
      a.u0 = uk; a.u1 = uk; a.u2 = uk; a.c0 = T(0); a.c1 = T(0); a.c2 = T(0);
      a.uk = uk; a.hstride = dn;
      a.acc = acc.as<T>(); a.astride = 4 * dn; a.kahan = 1;
      a.tj = tjf;
      k_stepv<T, 1><<<grd, 128, 0, st>>>(wr, a);
      c.launches += 2;
      std::swap(LA, LB);
    }
    GJ_CUDA(err, cudaGetLastError());
    DevBuf gb;
    GJ_TRY(gb.alloc(err, 2 * mn * sizeof(double)));
    k_finish<T><<<256, 256, 0, st>>>(w, acc.as<T>(), 4 * dn, 1, 0, 0, g.dt, g.eps0, eps_m, sig_m,
                                     gb.as<double>(), gb.as<double>() + mn);
    GJ_CUDA(err, cudaGetLastError());
    GJ_CUDA(err, cudaDeviceSynchronize());
    std::vector<double> tmp(2 * mn);
    GJ_CUDA(err, cudaMemcpy(tmp.data(), gb.p, 2 * mn * sizeof(double), cudaMemcpyDeviceToHost));
    for (size_t p = 0; p < mn; ++p) gout[p] = tmp[mn + p];  // the u-correlation (sigma form)
    if (amax) {
      std::vector<T> hl(sstride);
      GJ_CUDA(err, cudaMemcpy(hl.data(), LA - ld, sstride * sizeof(T), cudaMemcpyDeviceToHost));
      for (int b = 0; b < g.n; ++b)
        for (int a_ = 0; a_ < g.m; ++a_)
          amax[size_t(a_) + size_t(b) * g.m] =
              std::fabs(double(hl[size_t(ld) + size_t(w.di0 + a_) + size_t(w.dj0 + b) * ld]));
    }
    return GJ_OK;
  }
};

template <class T>
static gj_status get_solver(Ctx& c, const gj_w_grid& g, const gj_w_shot* shots, int ns, WSolver<T>*& out) {
  c.dc_fac.release();  // the radar plan sizes itself from the free memory
  c.dc_vec.release();
  std::string k = std::string(sizeof(T) == 8 ? "d" : "f") + WSolver<T>::key(g, shots, ns);
  if (c.wsolver && c.wkey == k) {
    out = static_cast<WSolver<T>*>(c.wsolver.get());
    return GJ_OK;
  }
  c.wsolver.reset();
  auto s = std::make_unique<WSolver<T>>();
  GJ_TRY(s->setup(c.err, g, shots, ns));
  out = s.get();
  c.wsolver = std::move(s);
  c.wkey = k;
  return GJ_OK;
}

gj_status w_forward(Ctx& c, const gj_w_grid& g, gj_precision prec, const double* eps, const double* sig,
                    const gj_w_shot* shots, int nshots, double* d_out, double* jz_out, double* u_out) {
  if (!eps || !sig || !d_out) return c.err.set(GJ_EINVAL, "null model or output pointer");
  if (prec == GJ_F64) {
    WSolver<double>* s; GJ_TRY(get_solver(c, g, shots, nshots, s));
    return s->forward(c.err, c, eps, sig, d_out, jz_out, u_out);
  }
  WSolver<float>* s; GJ_TRY(get_solver(c, g, shots, nshots, s));
  return s->forward(c.err, c, eps, sig, d_out, jz_out, u_out);
}

gj_status w_gradient(Ctx& c, const gj_w_grid& g, gj_precision prec, const void* eps, const void* sig,
                     bool dev_in, const gj_w_shot* shots, int nshots, const void* dobs, bool dev_dobs,
                     gj_adj_mode mode, gj_misfit_kind mk, const gj_w_opts& o, void* geps, void* gsig,
                     bool dev_out, double* misfit_out, double* d_out, double* e_out, cudaStream_t st, bool e_given) {
  if (!eps || !sig || !dobs || !geps || !gsig) return c.err.set(GJ_EINVAL, "null input or output pointer");
  if (mode != GJ_ADJ_REFERENCE && mode != GJ_ADJ_EXACT) return c.err.set(GJ_EINVAL, "unknown adjoint mode");
  if (mk < GJ_MISFIT_L2 || mk > GJ_MISFIT_ENV_LOG) return c.err.set(GJ_EINVAL, "unknown misfit kind");
  if (prec == GJ_F64) {
    WSolver<double>* s; GJ_TRY(get_solver(c, g, shots, nshots, s));
    return s->gradient(c.err, c, eps, sig, dev_in, dobs, dev_dobs, mode, mk, o, geps, gsig, dev_out, misfit_out,
                       d_out, e_out, st, e_given);
  }
  WSolver<float>* s; GJ_TRY(get_solver(c, g, shots, nshots, s));
  return s->gradient(c.err, c, eps, sig, dev_in, dobs, dev_dobs, mode, mk, o, geps, gsig, dev_out, misfit_out,
                     d_out, e_out, st, e_given);
}

gj_status w_misfit(Ctx& c, const gj_w_grid& g, gj_precision prec, const double* eps, const double* sig,
                   const gj_w_shot* shots, int nshots, const double* dobs, gj_misfit_kind mk, double* misfit_out,
                   int ntrial, const gj_w_opts* opts) {
  if (!eps || !sig || !dobs || !misfit_out) return c.err.set(GJ_EINVAL, "null input or output pointer");
  if (mk < GJ_MISFIT_L2 || mk > GJ_MISFIT_ENV_LOG) return c.err.set(GJ_EINVAL, "unknown misfit kind");
  if (ntrial < 1) return c.err.set(GJ_EINVAL, "ntrial must be >= 1");
  const size_t mn = size_t(g.m) * size_t(g.n);
  if (ntrial > 1) {  // all models in one blocked run when the configuration allows it
    bool done = false;
    if (prec == GJ_F64) {
      WSolver<double>* s; GJ_TRY(get_solver(c, g, shots, nshots, s));
      GJ_TRY(s->misfit_trials(c.err, c, ntrial, eps, sig, dobs, mk, misfit_out, 0, opts, done));
    } else {
      WSolver<float>* s; GJ_TRY(get_solver(c, g, shots, nshots, s));
      GJ_TRY(s->misfit_trials(c.err, c, ntrial, eps, sig, dobs, mk, misfit_out, 0, opts, done));
    }
    if (done) return GJ_OK;
  }
  for (int t = 0; t < ntrial; ++t) {
    if (prec == GJ_F64) {
      WSolver<double>* s; GJ_TRY(get_solver(c, g, shots, nshots, s));
      GJ_TRY(s->misfit(c.err, c, eps + t * mn, sig + t * mn, dobs, mk, misfit_out + size_t(t) * nshots, 0, opts));
    } else {
      WSolver<float>* s; GJ_TRY(get_solver(c, g, shots, nshots, s));
      GJ_TRY(s->misfit(c.err, c, eps + t * mn, sig + t * mn, dobs, mk, misfit_out + size_t(t) * nshots, 0, opts));
    }
  }
  return GJ_OK;
}

gj_status w_grad_only(Ctx& c, const gj_w_grid& g, gj_precision prec, const double* eps, const double* sig,
                      const gj_w_shot& shot, const double* e, const double* u, double* gout, double* amax) {
  if (!eps || !sig || !e || !u || !gout) return c.err.set(GJ_EINVAL, "null input or output pointer");
  if (prec == GJ_F64) {
    WSolver<double>* s; GJ_TRY(get_solver(c, g, &shot, 1, s));
    return s->grad_only(c.err, c, eps, sig, e, u, gout, amax);
  }
  WSolver<float>* s; GJ_TRY(get_solver(c, g, &shot, 1, s));
  return s->grad_only(c.err, c, eps, sig, e, u, gout, amax);
}

// ------------------------------------------------------------------ batch
// gj_w_gradient_batch: many independent problems (grids, shots, step counts
// all different), their whole gradients run concurrently.  Each problem's
// plan is cached; its large buffers (adjoint states, u and band history,
// checkpoints, rings) are carved from one pool at offsets that repeat from
// call to call, so the captured graphs stay valid.  The problems are packed
// into waves by their smallest pool footprint (checkpointed at the interval
// of least memory); a wave's spare memory lets problems keep more history
// (the whole of it when it fits, which saves the recompute).  Every wave is
// one CUDA graph whose child graphs (one per problem: forward, residual,
// recompute, adjoint, imaging of all its shots) have no dependencies on one
// another, launched once.
template <class T>
struct WBatch : WBatchBase {
  std::vector<std::string> keys;
  std::vector<std::unique_ptr<WSolver<T>>> plans;
  std::vector<int> kc;  // checkpoint interval per problem (nt: whole history)
  std::vector<int> gs;  // shots per group per problem (0: all shots in one launch)
  DevBuf pool;
  std::vector<std::vector<int>> waves;
  cudaGraphExec_t exec = nullptr;  // every wave, one after the other, in one graph
  long launches = 0;               // kernel launches inside it
  int mode = -1, kahan = -1;
  size_t budget_opt = 0;  // opts.mem_budget_bytes the waves were planned for
  void drop_waves() {
    if (exec) cudaGraphExecDestroy(exec);
    exec = nullptr;
    waves.clear();
    launches = 0;
  }
  ~WBatch() override { drop_waves(); }
};

template <class T>
static gj_status gradient_batch_t(Ctx& c, const gj_w_problem* pr, int np, gj_adj_mode mode, const gj_w_opts& o0,
                                  int* nwaves_out) {
  Err& err = c.err;
  const int kahan = o0.no_kahan ? 0 : 1;
  c.wsolver.reset();  // the single-call plan and the DC buffers give their memory back
  c.wkey.clear();
  c.dc_fac.release();
  c.dc_vec.release();
  std::vector<std::string> keys(np);
  for (int p = 0; p < np; ++p)
    keys[p] = std::string(sizeof(T) == 8 ? "d" : "f") + WSolver<T>::key(pr[p].grid, pr[p].shots, pr[p].nshots);
  auto* B = dynamic_cast<WBatch<T>*>(c.wbatch.get());
  if (!B || B->keys != keys || B->mode != int(mode) || B->kahan != kahan) {
    c.wbatch.reset();
    auto nb = std::make_unique<WBatch<T>>();
    nb->keys = keys;
    nb->mode = int(mode);
    nb->kahan = kahan;
    for (int p = 0; p < np; ++p) {
      auto sv = std::make_unique<WSolver<T>>();
      gj_status r = sv->setup(err, pr[p].grid, pr[p].shots, pr[p].nshots);
      if (r != GJ_OK) return err.set(r, "problem %d: %s", p, err.msg.c_str());
      if (sv->ring_nth == 0) return err.set(GJ_EUNSUPPORTED, "problem %d: the batch runs the ring kernels only", p);
      sv->light_tune = true;
      nb->plans.push_back(std::move(sv));
    }
    B = nb.get();
    c.wbatch = std::move(nb);
  }
  if (B->budget_opt != o0.mem_budget_bytes) {
    B->drop_waves();
    B->budget_opt = o0.mem_budget_bytes;
  }
  cudaStream_t st = 0;
  for (int p = 0; p < np; ++p) {
    if (!pr[p].eps_r || !pr[p].sigma || !pr[p].d_obs || !pr[p].g_eps || !pr[p].g_sig)
      return err.set(GJ_EINVAL, "problem %d: null input or output pointer", p);
    gj_status r = B->plans[p]->stage_inputs(err, c, pr[p].eps_r, pr[p].sigma, false, pr[p].d_obs, false, st);
    if (r != GJ_OK) return r;
  }
  const bool exact = mode == GJ_ADJ_EXACT;
  if (B->waves.empty()) {
    // per-problem memory outside the pool (accumulators, forward states, final gradients) and the pool budget
    size_t owned = 0;
    for (auto& q : B->plans)
      owned += size_t(q->nshots) * (4 * q->dn + 2 * q->sstride + (exact ? 2 * size_t(q->w.bsz) : 0)) * sizeof(T) +
               4 * q->mn * sizeof(double);
    size_t free_b = 0, total_b = 0;
    GJ_CUDA(err, cudaMemGetInfo(&free_b, &total_b));
    const size_t avail = free_b > owned ? free_b - owned : 0;
    const size_t budget = o0.mem_budget_bytes ? o0.mem_budget_bytes : size_t(0.8 * double(avail));
    // Per problem, one of: (a) all shots in one launch, checkpointed (pool
    // nmin; the cheapest in memory, one recompute pass), upgraded to the whole
    // history when its wave has room; (b) the whole history in shot groups of
    // gs shots run one after the other (no recompute pass), for a problem whose
    // whole history takes more than a quarter of the budget, when groups of at
    // least 4 shots (or all) fit it.
    std::vector<size_t> nmin(np), nfull(np), need(np);
    std::vector<int> kmin(np);
    B->gs.assign(np, 0);
    for (int p = 0; p < np; ++p) {
      const WSolver<T>& q = *B->plans[p];
      kmin[p] = q.best_k(exact);
      nmin[p] = q.pool_need(kmin[p], exact);
      nfull[p] = q.pool_need(q.g.nt, exact);
      need[p] = nmin[p];
      if (nfull[p] > budget / 4) {
        const int ns = q.nshots;
        int G = 0;
        for (int t = ns; t >= std::min(ns, 4); --t)
          if (q.pool_need(q.g.nt, exact, t) <= budget) { G = t; break; }
        if (G > 0) {
          const int ng = (ns + G - 1) / G;  // balanced groups
          G = (ns + ng - 1) / ng;
          B->gs[p] = G;
          need[p] = q.pool_need(q.g.nt, exact, G);
        }
      }
      if (need[p] > budget) return err.set(GJ_ENOMEM, "problem %d needs %zu bytes, above the budget %zu", p, need[p], budget);
    }
    // pack by work, largest first
    std::vector<int> order(np);
    for (int p = 0; p < np; ++p) order[p] = p;
    auto work = [&](int p) {
      return double(B->plans[p]->nshots) * B->plans[p]->g.nt * double(B->plans[p]->NX) * B->plans[p]->NY;
    };
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return work(a) > work(b); });
    std::vector<int> cur;
    size_t used = 0;
    for (int p : order) {
      if (!cur.empty() && used + need[p] > budget) {
        B->waves.push_back(cur);
        cur.clear();
        used = 0;
      }
      cur.push_back(p);
      used += need[p];
    }
    if (!cur.empty()) B->waves.push_back(cur);
    // spare memory of a wave: whole histories for the checkpointed problems,
    // the cheapest upgrades first
    B->kc = kmin;
    for (int p = 0; p < np; ++p)
      if (B->gs[p] > 0) B->kc[p] = B->plans[p]->g.nt;
    size_t pool = 0;
    for (auto& wv : B->waves) {
      size_t u = 0;
      for (int p : wv) u += need[p];
      std::vector<int> up;
      for (int p : wv)
        if (B->gs[p] == 0) up.push_back(p);
      std::sort(up.begin(), up.end(), [&](int a, int b) { return nfull[a] - nmin[a] < nfull[b] - nmin[b]; });
      for (int p : up)
        if (u - nmin[p] + nfull[p] <= budget) { u += nfull[p] - nmin[p]; B->kc[p] = B->plans[p]->g.nt; }
      pool = std::max(pool, u);
    }
    GJ_TRY(B->pool.alloc(err, pool));
    if (getenv("GJ_BATCH_VERBOSE")) {
      for (size_t wi = 0; wi < B->waves.size(); ++wi)
        for (int p : B->waves[wi])
          fprintf(stderr, "gerjoii_b200 batch wave %zu problem %d: %d shots (groups of %d), %s, pool %.1f MB\n",
                  wi, p, B->plans[p]->nshots, B->gs[p] > 0 ? B->gs[p] : B->plans[p]->nshots,
                  B->gs[p] > 0 ? "whole history in shot groups"
                               : (B->kc[p] >= B->plans[p]->g.nt ? "whole history" : "checkpointed"),
                  double(B->gs[p] > 0 ? need[p] : (B->kc[p] >= B->plans[p]->g.nt ? nfull[p] : nmin[p])) / 1e6);
      fprintf(stderr, "gerjoii_b200 batch pool %.1f MB of budget %.1f MB\n", double(pool) / 1e6, double(budget) / 1e6);
    }
  }
  if (nwaves_out) *nwaves_out = int(B->waves.size());
  if (!B->exec) {
    // One graph: per wave, one child graph per problem (no dependencies
    // between them); each wave after the previous one, whose pool it reuses.
    cudaGraph_t all = nullptr;
    GJ_CUDA(err, cudaGraphCreate(&all, 0));
    struct GraphGuard { cudaGraph_t g; ~GraphGuard() { if (g) cudaGraphDestroy(g); } } ga{all};
    std::vector<cudaGraphNode_t> prev;  // the previous wave's nodes
    long nl = 0;
    for (size_t wi = 0; wi < B->waves.size(); ++wi) {
      const auto& wv = B->waves[wi];
      unsigned char* cursor = B->pool.template as<unsigned char>();
      std::vector<cudaGraphNode_t> cur;
      for (int p : wv) {
        WSolver<T>& q = *B->plans[p];
        gj_w_opts op = o0;
        op.shots_per_launch = B->gs[p] > 0 ? B->gs[p] : q.nshots;
        op.ckpt_every = B->kc[p] >= q.g.nt ? 0 : B->kc[p];
        op.mem_budget_bytes = B->kc[p] >= q.g.nt ? size_t(-1) / 4 : 0;
        q.pool_p = cursor;
        gj_status r = q.plan_buffers(err, op, size_t(1) << 62, mode, st);
        cursor = q.pool_p;
        q.pool_p = nullptr;
        if (r != GJ_OK) return r;
        if (size_t(cursor - B->pool.template as<unsigned char>()) > B->pool.bytes)
          return err.set(GJ_ENOMEM, "batch pool overrun (problem %d)", p);
        cudaStream_t cs;
        GJ_CUDA(err, cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
        GJ_CUDA(err, cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
        gj_status rs = q.enqueue_all(err, c, mode, kahan, cs, nl);
        cudaGraph_t pg = nullptr;
        cudaError_t ce = cudaStreamEndCapture(cs, &pg);
        cudaStreamDestroy(cs);
        if (rs != GJ_OK) { if (pg) cudaGraphDestroy(pg); return rs; }
        if (ce != cudaSuccess) return err.set(GJ_ECUDA, "graph capture failed: %s", cudaGetErrorString(ce));
        cudaGraphNode_t node;
        ce = cudaGraphAddChildGraphNode(&node, all, prev.data(), prev.size(), pg);
        cudaGraphDestroy(pg);
        if (ce != cudaSuccess) return err.set(GJ_ECUDA, "child graph: %s", cudaGetErrorString(ce));
        cur.push_back(node);
      }
      prev = std::move(cur);
    }
    cudaError_t ce = cudaGraphInstantiate(&B->exec, all, cudaGraphInstantiateFlagUseNodePriority);
    if (ce != cudaSuccess) {
      B->exec = nullptr;
      return err.set(GJ_ECUDA, "batch graph instantiate failed: %s", cudaGetErrorString(ce));
    }
    B->launches = nl;
  }
  GJ_CUDA(err, cudaGraphLaunch(B->exec, st));
  GJ_CUDA(err, cudaStreamSynchronize(st));
  c.launches += B->launches;
  // every problem's accumulators, sums and traces are its own (outside the
  // pool), so the finishing steps follow the whole graph
  for (int p = 0; p < np; ++p) {
    {
      WSolver<T>& q = *B->plans[p];
      std::vector<double> hs(2 * q.nshots);
      GJ_CUDA(err, cudaMemcpy(hs.data(), q.sums.p, hs.size() * sizeof(double), cudaMemcpyDeviceToHost));
      gj_w_opts op = o0;
      op.per_shot = 0;
      gj_status r = q.finish(err, c, mode, op, pr[p].g_eps, pr[p].g_sig, false, pr[p].misfit, nullptr, nullptr, hs, st);
      if (r != GJ_OK) return err.set(r, "problem %d: %s", p, err.msg.c_str());
    }
  }
  return GJ_OK;
}

gj_status w_gradient_batch(Ctx& c, gj_precision prec, const gj_w_problem* probs, int nprob, gj_adj_mode mode,
                           const gj_w_opts& o, int* nwaves_out) {
  if (nprob < 1 || !probs) return c.err.set(GJ_EINVAL, "need at least one problem");
  if (mode != GJ_ADJ_REFERENCE && mode != GJ_ADJ_EXACT) return c.err.set(GJ_EINVAL, "unknown adjoint mode");
  if (o.plain || o.no_ring || o.filt_high > o.filt_low || o.condition || o.per_shot)
    return c.err.set(GJ_EUNSUPPORTED, "the batch supports the default ring path with the L2 misfit, summed "
                                      "gradients and no residual filter or conditioning");
  if (prec == GJ_F64) return gradient_batch_t<double>(c, probs, nprob, mode, o, nwaves_out);
  return gradient_batch_t<float>(c, probs, nprob, mode, o, nwaves_out);
}

}  // namespace gj

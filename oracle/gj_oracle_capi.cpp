// ORACLE — TEST INFRASTRUCTURE ONLY.
// extern "C" wrappers around gj_oracle.hpp for ctypes (tests, smoke check and the
// benchmark's CPU-baseline leg).  Built by oracle/Makefile into oracle/_build/.
#include <atomic>
#include <thread>

#include "gj_oracle.hpp"

struct gjo_grid_c {
  int m, n, pml, pml_top, air, nt;
  double dx, dy, dt, eps0, mu0;
  int order;
  double R0;
};

static gjo::Grid to_grid(const gjo_grid_c* c) {
  gjo::Grid g;
  g.m = c->m; g.n = c->n; g.pml = c->pml; g.pml_top = c->pml_top; g.air = c->air; g.nt = c->nt;
  g.dx = c->dx; g.dy = c->dy; g.dt = c->dt; g.eps0 = c->eps0; g.mu0 = c->mu0;
  g.order = c->order; g.R0 = c->R0;
  return g;
}

// Dynamic parallel-for over [0, n) on `threads` std::threads (OpenMP is not in
// this toolchain).
template <class F>
static void parallel_for(int n, int threads, F&& f) {
  if (threads <= 0) threads = int(std::thread::hardware_concurrency());
  threads = std::max(1, std::min(threads, n));
  std::atomic<int> next{0};
  std::vector<std::thread> pool;
  for (int t = 0; t < threads; ++t)
    pool.emplace_back([&] {
      for (int i = next++; i < n; i = next++) f(i);
    });
  for (auto& th : pool) th.join();
}

static gjo::Shot to_shot(const gjo::Grid& g, int si, int sj, const double* w, int nr, const long* rec) {
  gjo::Shot s;
  s.src_i = si; s.src_j = sj;
  if (w) s.wavelet.assign(w, w + g.nt);
  s.rec.assign(rec, rec + nr);
  return s;
}

extern "C" {

#define GJO_FWD(SUF, T)                                                                          \
  int gjo_w_forward_##SUF(const gjo_grid_c* gc, const double* eps, const double* sig, int si,   \
                          int sj, const double* w, int nr, const long* rec, T* d, T* jz, T* u) { \
    gjo::Grid g = to_grid(gc);                                                                   \
    gjo::forward<T>(g, eps, sig, to_shot(g, si, sj, w, nr, rec), d, jz, u);                     \
    return 0;                                                                                    \
  }
GJO_FWD(f64, double)
GJO_FWD(f32, float)

#define GJO_GREF(SUF, T)                                                                          \
  int gjo_w_grad_reference_##SUF(const gjo_grid_c* gc, const double* eps, const double* sig,     \
                                 int si, int sj, int nr, const long* rec, const T* e, const T* u, \
                                 T* g_out, T* amax) {                                             \
    gjo::Grid g = to_grid(gc);                                                                    \
    gjo::grad_reference<T>(g, eps, sig, to_shot(g, si, sj, nullptr, nr, rec), e, u, g_out, amax); \
    return 0;                                                                                     \
  }
GJO_GREF(f64, double)
GJO_GREF(f32, float)

#define GJO_GEX(SUF, T)                                                                           \
  int gjo_w_grad_exact_##SUF(const gjo_grid_c* gc, const double* eps, const double* sig, int si, \
                             int sj, const double* w, int nr, const long* rec, const T* e,        \
                             double* geps, double* gsig) {                                        \
    gjo::Grid g = to_grid(gc);                                                                    \
    gjo::grad_exact<T>(g, eps, sig, to_shot(g, si, sj, w, nr, rec), e, geps, gsig);              \
    return 0;                                                                                     \
  }
GJO_GEX(f64, double)
GJO_GEX(f32, float)

int gjo_differentiate_cube_f64(double* v, long npix, int nt, double dt) {
  gjo::differentiate_cube<double>(v, size_t(npix), nt, dt);
  return 0;
}
int gjo_differentiate_cube_f32(float* v, long npix, int nt, double dt) {
  gjo::differentiate_cube<float>(v, size_t(npix), nt, dt);
  return 0;
}

}  // extern "C"

// Whole FWI gradient for a set of shots, one shot per host thread (the
// reference's parfor over shots, w_update_e_.m:32): forward, L2 residual,
// then the REFERENCE (mode 0: g_eps from d/dt u, g_sig from u, w_update_es.m)
// or EXACT (mode 1) gradient.  Gradients are summed over shots; misfit[s] is
// the per-shot normalised misfit.  All shots share nr receivers.
template <class T>
static int grad_batch(const gjo_grid_c* gc, const double* eps, const double* sig, int nshots,
                      const int* si, const int* sj, const double* wav, int nr, const long* rec,
                      const double* dobs, int mode, int threads, double* geps, double* gsig,
                      double* misfit) {
  gjo::Grid g = to_grid(gc);
  const size_t mn = size_t(g.m) * g.n, ntr = size_t(g.nt) * nr;
  std::vector<std::vector<double>> ge(nshots, std::vector<double>(mn)), gs(nshots, std::vector<double>(mn));
  parallel_for(nshots, threads, [&](int s) {
    gjo::Shot sh = to_shot(g, si[s], sj[s], wav + size_t(s) * g.nt, nr, rec + size_t(s) * nr);
    std::vector<T> d(ntr), e(ntr), dob(ntr);
    for (size_t i = 0; i < ntr; ++i) dob[i] = T(dobs[size_t(s) * ntr + i]);
    if (mode == 0) {
      std::vector<T> u(mn * g.nt);
      gjo::forward<T>(g, eps, sig, sh, d.data(), nullptr, u.data());
      misfit[s] = gjo::residual_l2<T>(d.data(), dob.data(), ntr, e.data());
      std::vector<T> gt(mn);
      gjo::grad_reference<T>(g, eps, sig, sh, e.data(), u.data(), gt.data(), nullptr);
      for (size_t p = 0; p < mn; ++p) gs[s][p] = gt[p];
      gjo::differentiate_cube<T>(u.data(), mn, g.nt, g.dt);
      gjo::grad_reference<T>(g, eps, sig, sh, e.data(), u.data(), gt.data(), nullptr);
      for (size_t p = 0; p < mn; ++p) ge[s][p] = gt[p];
    } else {
      gjo::forward<T>(g, eps, sig, sh, d.data(), nullptr, nullptr);
      misfit[s] = gjo::residual_l2<T>(d.data(), dob.data(), ntr, e.data());
      gjo::grad_exact<T>(g, eps, sig, sh, e.data(), ge[s].data(), gs[s].data());
    }
  });
  for (size_t p = 0; p < mn; ++p) {
    double a = 0, b = 0;
    for (int s = 0; s < nshots; ++s) { a += ge[s][p]; b += gs[s][p]; }
    geps[p] = a; gsig[p] = b;
  }
  return 0;
}

extern "C" {

int gjo_w_gradient_batch(const gjo_grid_c* gc, int precision, const double* eps, const double* sig,
                         int nshots, const int* si, const int* sj, const double* wav, int nr,
                         const long* rec, const double* dobs, int mode, int threads, double* geps,
                         double* gsig, double* misfit) {
  if (precision == 1)
    return grad_batch<double>(gc, eps, sig, nshots, si, sj, wav, nr, rec, dobs, mode, threads, geps, gsig, misfit);
  return grad_batch<float>(gc, eps, sig, nshots, si, sj, wav, nr, rec, dobs, mode, threads, geps, gsig, misfit);
}

// Forward traces for a set of shots in parallel (observed-data synthesis and the
// forward-only CPU baseline).  d is nt x nr x nshots.
int gjo_w_forward_batch(const gjo_grid_c* gc, int precision, const double* eps, const double* sig,
                        int nshots, const int* si, const int* sj, const double* wav, int nr,
                        const long* rec, int threads, double* d) {
  gjo::Grid g = to_grid(gc);
  const size_t ntr = size_t(g.nt) * nr;
  parallel_for(nshots, threads, [&](int s) {
    gjo::Shot sh = to_shot(g, si[s], sj[s], wav + size_t(s) * g.nt, nr, rec + size_t(s) * nr);
    if (precision == 1) {
      gjo::forward<double>(g, eps, sig, sh, d + size_t(s) * ntr, nullptr, nullptr);
    } else {
      std::vector<float> df(ntr);
      gjo::forward<float>(g, eps, sig, sh, df.data(), nullptr, nullptr);
      for (size_t i = 0; i < ntr; ++i) d[size_t(s) * ntr + i] = df[i];
    }
  });
  return 0;
}

}  // extern "C"

// ORACLE — TEST INFRASTRUCTURE ONLY.
//
// CPU restatement of the reference's radar (GPR) FDTD forward solve, its two
// adjoints and the imaging condition.  Only the test suite, the smoke check and
// the CPU-baseline leg of the benchmark may call this code, and only as the
// checker: the product path is the CUDA library under gerjoii_b200/csrc.
//
// Each function names the reference file:line it restates (paths inside the
// diegozain/gerjoii project).  Parity status: the reference is MATLAB and cannot
// run here; this restatement is pinned against the numpy twin (oracle/np_oracle.py,
// which follows the MATLAB strip-by-strip slicing literally), against the
// reference's known answers, and (exact adjoint) against central differences.
//
// Conventions (0-based, column-major, fastest index = depth i, as in MATLAB):
//   NX = pml_top + air + m + pml   (depth incl. PML; "nx" in wdc_geom.m:70)
//   NY = n + 2*pml                 (lateral incl. PML; "ny" in wdc_geom.m:69)
//   Ez (NX+1)x(NY+1), Hx (NX+1)xNY, Hy NXx(NY+1) (w_solve.m:70-72); here all
//   three live in (NX+1)x(NY+1) arrays with leading dimension NX+1.
//   eps_r_z / sigma_e_z are NX x NY cells; Ez node (I,J) uses cell (I,J).
#pragma once
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <stdexcept>
#include <vector>

namespace gjo {

struct Grid {
  int m = 0, n = 0;     // model rows (depth) and columns (lateral)
  int pml = 0;          // PML cells bottom/left/right (pml_w == pml_d)
  int pml_top = 0;      // PML rows on top: pml (reference layout) or 0 (free top)
  int air = 0;          // air rows (eps_r=1, sigma=0) above the model
  int nt = 0;
  double dx = 0, dy = 0, dt = 0;
  double eps0 = 8.854187817e-12, mu0 = 4e-7 * M_PI;  // param_wdc.m:28-29
  int order = 2;                                     // wdc_geom.m:98
  double R0 = 1e-8;                                  // wdc_geom.m:99
  int NX() const { return pml_top + air + m + pml; }
  int NY() const { return n + 2 * pml; }
};

// Index ranges of w_solve.m in 0-based form.
// pis = pml_top+1, pie = NX-pml+1, pjs = pml+1, pje = NY-pml+1 (wdc_geom.m:100-103).
struct Layout {
  int NX, NY, P, Pt, air, m, n, ld;
  int ez_i0, ez_i1, ez_j0, ez_j1;  // interior Ez nodes, inclusive (w_solve.m:201)
  int hy_i0, hy_i1;                // interior Hy rows (w_solve.m:146)
  int hx_j0, hx_j1;                // interior Hx cols (w_solve.m:144)
  int dom_i0, dom_j0;              // domain origin (wdc_geom.m:107-110)
  explicit Layout(const Grid& g) {
    P = g.pml; Pt = g.pml_top; air = g.air; m = g.m; n = g.n;
    NX = g.NX(); NY = g.NY(); ld = NX + 1;
    ez_i0 = Pt + 1; ez_i1 = NX - P - 1;
    ez_j0 = P + 1;  ez_j1 = NY - P - 1;
    hy_i0 = Pt;     hy_i1 = NX - P - 1;
    hx_j0 = P;      hx_j1 = NY - P - 1;
    dom_i0 = Pt + air; dom_j0 = P;
  }
  size_t nodes() const { return size_t(NX + 1) * size_t(NY + 1); }
  size_t at(int I, int J) const { return size_t(I) + size_t(J) * size_t(ld); }
  bool ez_interior(int I, int J) const {
    return I >= ez_i0 && I <= ez_i1 && J >= ez_j0 && J <= ez_j1;
  }
  bool ez_boundary(int I, int J) const { return I == 0 || J == 0 || I == NX || J == NY; }
  bool ez_band(int I, int J) const { return !ez_boundary(I, J) && !ez_interior(I, J); }
  bool x_top(int I) const { return I >= 1 && I <= Pt; }
  bool x_bot(int I) const { return I >= NX - P && I <= NX - 1; }
  bool y_strip(int J) const { return (J >= 1 && J <= P) || (J >= NY - P && J <= NY - 1); }
};

// w_exp2pml.m:19-34 generalised to pml_top rows on top: air rows on top, then
// edge-replicated eps_r in the PML (sides first, then top/bottom rows of the
// side-padded array), zero sigma outside the model.
inline void exp2pml(const Grid& g, const double* eps, const double* sig,
                    std::vector<double>& epsr, std::vector<double>& sigz) {
  const int NX = g.NX(), NY = g.NY(), P = g.pml, Pt = g.pml_top, air = g.air;
  const int rows_mid = air + g.m;  // [air; model]
  std::vector<double> e_side(size_t(rows_mid) * NY), s_side(size_t(rows_mid) * NY, 0.0);
  for (int J = 0; J < NY; ++J) {
    int jm = std::min(std::max(J - P, 0), g.n - 1);
    for (int r = 0; r < rows_mid; ++r) {
      double e = 1.0, s = 0.0;
      if (r >= air) {
        e = eps[size_t(r - air) + size_t(jm) * g.m];
        if (J >= P && J < P + g.n) s = sig[size_t(r - air) + size_t(J - P) * g.m];
      }
      e_side[size_t(r) + size_t(J) * rows_mid] = e;
      s_side[size_t(r) + size_t(J) * rows_mid] = s;
    }
  }
  epsr.assign(size_t(NX) * NY, 0.0);
  sigz.assign(size_t(NX) * NY, 0.0);
  for (int J = 0; J < NY; ++J)
    for (int I = 0; I < NX; ++I) {
      int r = std::min(std::max(I - Pt, 0), rows_mid - 1);
      epsr[size_t(I) + size_t(J) * NX] = e_side[size_t(r) + size_t(J) * rows_mid];
      bool in_mid = I >= Pt && I < Pt + rows_mid;
      sigz[size_t(I) + size_t(J) * NX] = in_mid ? s_side[size_t(I - Pt) + size_t(J) * rows_mid] : 0.0;
    }
}

// Per-node update coefficients, double precision (w_cpml.m, w_coeff.m).
struct Coefs {
  std::vector<double> ce, chy, chx;    // interior Ez: Ceze, Cezhy, Cezhx (w_coeff.m:28-30)
  std::vector<double> ax, bx, ay, by;  // band Ez: split-field Ezx/Ezy coefficients (w_cpml.m)
  std::vector<double> hxa, hxb, hya, hyb;  // H: 1/scalar in the interior, graded in strips
  double cezj = 0;                     // source coefficient (w_coeff.m:44-45)
  // PML profiles kept for the exact adjoint's eps-derivatives.
  std::vector<double> sex, smx, sey, smy;  // graded sigma_e / sigma_m per row (x) / column (y)
};

inline double sigma_max(const Grid& g, double d) {
  // w_cpml.m:47-48: -(order+1)*eps0*c*log(R0)/(2*d*pml)
  const double c = 1.0 / std::sqrt(g.mu0 * g.eps0);
  return -(g.order + 1) * g.eps0 * c * std::log(g.R0) / (2.0 * d * g.pml);
}

// Graded PML conductivity profiles, rho_e = (k-0.75)/P, rho_m = (k-0.25)/P
// counted from the interface (w_cpml.m:49-50, 72-73, 112-113, 153-154).
inline void pml_profiles(const Grid& g, const Layout& L, Coefs& c) {
  const double P = g.pml, smx_ = sigma_max(g, g.dx), smy_ = sigma_max(g, g.dy);
  c.sex.assign(L.NX + 1, 0.0); c.smx.assign(L.NX + 1, 0.0);
  c.sey.assign(L.NY + 1, 0.0); c.smy.assign(L.NY + 1, 0.0);
  for (int I = 1; I <= L.Pt; ++I) {  // top strip Ez rows: ind = I (w_cpml.m:49)
    double r = (P - I + 1 - 0.75) / P;
    c.sex[I] = smx_ * std::pow(r, g.order);
  }
  for (int I = 0; I <= L.Pt - 1; ++I) {  // top strip Hy rows: ind = I+1 (w_cpml.m:50)
    double r = (P - (I + 1) + 1 - 0.25) / P;
    c.smx[I] = (g.mu0 / g.eps0) * smx_ * std::pow(r, g.order);
  }
  for (int I = L.NX - L.P; I <= L.NX - 1; ++I) {  // bottom strip (w_cpml.m:72-73)
    double k = I - (L.NX - L.P) + 1;
    c.sex[I] = smx_ * std::pow((k - 0.75) / P, g.order);
    c.smx[I] = (g.mu0 / g.eps0) * smx_ * std::pow((k - 0.25) / P, g.order);
  }
  for (int J = 1; J <= L.P; ++J) {  // left strip Ez cols: ind = J (w_cpml.m:112)
    double r = (P - J + 1 - 0.75) / P;
    c.sey[J] = smy_ * std::pow(r, g.order);
  }
  for (int J = 0; J <= L.P - 1; ++J) {  // left strip Hx cols: ind = J+1 (w_cpml.m:113)
    double r = (P - (J + 1) + 1 - 0.25) / P;
    c.smy[J] = (g.mu0 / g.eps0) * smy_ * std::pow(r, g.order);
  }
  for (int J = L.NY - L.P; J <= L.NY - 1; ++J) {  // right strip (w_cpml.m:153-154)
    double k = J - (L.NY - L.P) + 1;
    c.sey[J] = smy_ * std::pow((k - 0.75) / P, g.order);
    c.smy[J] = (g.mu0 / g.eps0) * smy_ * std::pow((k - 0.25) / P, g.order);
  }
}

// Builds every coefficient for the padded materials.  sign_sigma = -1 gives the
// reference adjoint's "dt <- -dt" coefficients (w_grad.m:21-27).
inline Coefs build_coefs(const Grid& g, const std::vector<double>& epsr,
                         const std::vector<double>& sigz, int src_i, int src_j,
                         double sign_sigma = 1.0) {
  Layout L(g);
  Coefs c;
  pml_profiles(g, L, c);
  const size_t N = L.nodes();
  const double dt = g.dt, dx = g.dx, dy = g.dy, e0 = g.eps0, u0 = g.mu0;
  c.ce.assign(N, 0); c.chy.assign(N, 0); c.chx.assign(N, 0);
  c.ax.assign(N, 0); c.bx.assign(N, 0); c.ay.assign(N, 0); c.by.assign(N, 0);
  c.hxa.assign(N, 1); c.hxb.assign(N, 0); c.hya.assign(N, 1); c.hyb.assign(N, 0);
  auto EPS = [&](int I, int J) { return epsr[size_t(I) + size_t(J) * L.NX]; };
  auto SIG = [&](int I, int J) { return sign_sigma * sigz[size_t(I) + size_t(J) * L.NX]; };
  for (int J = 0; J <= L.NY; ++J)
    for (int I = 0; I <= L.NX; ++I) {
      const size_t k = L.at(I, J);
      // ---- Hx (rows 0..NX, cols 0..NY-1) ----
      if (J <= L.NY - 1) {
        if (J >= L.hx_j0 && J <= L.hx_j1) {  // interior (w_solve.m:144, w_coeff.m:34-35)
          c.hxa[k] = 1.0; c.hxb[k] = -(2 * dt / dy) / (2 * u0);
        } else if (I >= 1 && I <= L.NX - 1) {  // y strips (w_solve.m:180-186, w_cpml.m:123-126,164-167)
          double s = c.smy[J] / EPS(I, J);
          c.hxa[k] = (2 * u0 - dt * s) / (2 * u0 + dt * s);
          c.hxb[k] = -(2 * dt / dy) / (2 * u0 + dt * s);
        }
      }
      // ---- Hy (rows 0..NX-1, cols 0..NY) ----
      if (I <= L.NX - 1) {
        if (I >= L.hy_i0 && I <= L.hy_i1) {  // interior (w_solve.m:146, w_coeff.m:39-40)
          c.hya[k] = 1.0; c.hyb[k] = (2 * dt / dx) / (2 * u0);
        } else if (J >= 1 && J <= L.NY - 1) {
          double s = c.smx[I];
          if (I >= L.NX - L.P) s /= EPS(I, J);  // bottom (xp) strip divides by eps_r (w_cpml.m:83)
          c.hya[k] = (2 * u0 - dt * s) / (2 * u0 + dt * s);
          c.hyb[k] = (2 * dt / dx) / (2 * u0 + dt * s);
        }
      }
      // ---- Ez ----
      if (L.ez_interior(I, J)) {  // w_coeff.m:28-30
        double D = 2 * EPS(I, J) * e0 + dt * SIG(I, J);
        c.ce[k] = (2 * EPS(I, J) * e0 - dt * SIG(I, J)) / D;
        c.chy[k] = (2 * dt / dx) / D;
        c.chx[k] = -(2 * dt / dy) / D;
      } else if (L.ez_band(I, J)) {
        const double e = EPS(I, J);
        // Ezx
        if (L.x_top(I)) {  // w_cpml.m:60-61 (no eps_r)
          double s = c.sex[I];
          c.ax[k] = (2 * e0 - dt * s) / (2 * e0 + dt * s);
          c.bx[k] = (2 * dt / dx) / (2 * e0 + dt * s);
        } else if (L.x_bot(I)) {  // w_cpml.m:93-96
          double s = c.sex[I];
          c.ax[k] = (2 * e0 * e - dt * s) / (2 * e0 * e + dt * s);
          c.bx[k] = (2 * dt / dx) / (2 * e0 * e + dt * s);
        } else {  // y strips, rows pis+1..pie-1 (w_cpml.m:133-134, 174-175)
          c.ax[k] = 1.0;
          c.bx[k] = dt / (dx * e0 * e);
        }
        // Ezy
        if (L.y_strip(J)) {  // w_cpml.m:141-144, 182-185
          double s = c.sey[J];
          c.ay[k] = (2 * e0 * e - dt * s) / (2 * e0 * e + dt * s);
          c.by[k] = -(2 * dt / dy) / (2 * e0 * e + dt * s);
        } else if (L.x_top(I)) {  // w_cpml.m:63-64
          c.ay[k] = 1.0;
          c.by[k] = -dt / (dy * e0);
        } else {  // x bottom strip, cols pjs+1..pje-1 (w_cpml.m:103-104)
          c.ay[k] = 1.0;
          c.by[k] = -dt / (dy * e0 * e);
        }
      }
    }
  if (src_i >= 0 && src_j >= 0) {  // w_coeff.m:44-45
    c.cezj = -(2 * dt) / (2 * EPS(src_i, src_j) * e0 + dt * SIG(src_i, src_j));
  }
  return c;
}

template <class T>
struct State {
  std::vector<T> Ez, Hx, Hy, Ezx, Ezy;
  explicit State(size_t N = 0) : Ez(N, T(0)), Hx(N, T(0)), Hy(N, T(0)), Ezx(N, T(0)), Ezy(N, T(0)) {}
};

// Coefficients rounded to the field precision (the reference keeps them in single).
template <class T>
struct CoefT {
  std::vector<T> ce, chy, chx, ax, bx, ay, by, hxa, hxb, hya, hyb;
  T cezj;
  explicit CoefT(const Coefs& c) {
    auto cv = [](const std::vector<double>& v) { return std::vector<T>(v.begin(), v.end()); };
    ce = cv(c.ce); chy = cv(c.chy); chx = cv(c.chx); ax = cv(c.ax); bx = cv(c.bx);
    ay = cv(c.ay); by = cv(c.by); hxa = cv(c.hxa); hxb = cv(c.hxb); hya = cv(c.hya); hyb = cv(c.hyb);
    cezj = T(c.cezj);
  }
};

// One Yee step of w_solve.m:80-94 (new_H, new_H_pml, new_Ez, source, new_Ez_pml).
// src < 0: no source (the adjoint of w_grad.m:77-83 has none).
template <class T>
inline void step(const Layout& L, const CoefT<T>& c, State<T>& s, long src, T srcval) {
  const int NX = L.NX, NY = L.NY;
  for (int J = 0; J <= NY - 1; ++J)
    for (int I = 0; I <= NX; ++I) {
      size_t k = L.at(I, J);
      s.Hx[k] = c.hxa[k] * s.Hx[k] + c.hxb[k] * (s.Ez[k + L.ld] - s.Ez[k]);
    }
  for (int J = 0; J <= NY; ++J)
    for (int I = 0; I <= NX - 1; ++I) {
      size_t k = L.at(I, J);
      s.Hy[k] = c.hya[k] * s.Hy[k] + c.hyb[k] * (s.Ez[k + 1] - s.Ez[k]);
    }
  for (int J = 1; J <= NY - 1; ++J)
    for (int I = 1; I <= NX - 1; ++I) {
      size_t k = L.at(I, J);
      T dhy = s.Hy[k] - s.Hy[k - 1];
      T dhx = s.Hx[k] - s.Hx[k - L.ld];
      if (L.ez_interior(I, J)) {
        s.Ez[k] = c.ce[k] * s.Ez[k] + c.chy[k] * dhy + c.chx[k] * dhx;
        if (long(k) == src) s.Ez[k] += c.cezj * srcval;  // w_solve.m:92
      } else {
        s.Ezx[k] = c.ax[k] * s.Ezx[k] + c.bx[k] * dhy;  // w_solve.m:232-256
        s.Ezy[k] = c.ay[k] * s.Ezy[k] + c.by[k] * dhx;
        s.Ez[k] = s.Ezx[k] + s.Ezy[k];                  // w_solve.m:260-267
      }
    }
}

struct Shot {
  int src_i = -1, src_j = -1;        // source Ez node (0-based)
  std::vector<double> wavelet;       // nt samples
  std::vector<long> rec;             // receiver Ez linear indices (0-based)
};

// w_fwd.m:18-24 + w_solve.m: forward model, traces d (nt x nr), source trace Jz
// (nt), optional domain history u (m x n x nt).
template <class T>
inline void forward(const Grid& g, const double* eps, const double* sig, const Shot& sh,
                    T* d, T* jz, T* u) {
  Layout L(g);
  std::vector<double> epsr, sigz;
  exp2pml(g, eps, sig, epsr, sigz);
  CoefT<T> c(build_coefs(g, epsr, sigz, sh.src_i, sh.src_j));
  State<T> s(L.nodes());
  const long src = long(L.at(sh.src_i, sh.src_j));
  const int nr = int(sh.rec.size());
  for (int it = 0; it < g.nt; ++it) {
    step<T>(L, c, s, src, T(sh.wavelet[it]));
    for (int r = 0; r < nr; ++r) d[size_t(it) + size_t(r) * g.nt] = s.Ez[sh.rec[r]];  // w_solve.m:100
    if (jz) jz[it] = s.Ez[src];                                                      // w_solve.m:104
    if (u)                                                                            // w_solve.m:102
      for (int b = 0; b < g.n; ++b)
        for (int a = 0; a < g.m; ++a)
          u[size_t(a) + size_t(b) * g.m + size_t(it) * g.m * g.n] = s.Ez[L.at(L.dom_i0 + a, L.dom_j0 + b)];
  }
}

// differentiate_cube.m:23-51: second-order time derivative, one-sided 3-point
// stencils at both ends, applied per pixel along the last axis.
template <class T>
inline void differentiate_cube(T* v, size_t npix, int nt, double dt) {
  std::vector<T> tmp(nt);
  for (size_t p = 0; p < npix; ++p) {
    for (int t = 0; t < nt; ++t) tmp[t] = v[p + size_t(t) * npix];
    for (int t = 0; t < nt; ++t) {
      double r;
      if (t == 0) r = (-1.5 * tmp[0] + 2.0 * tmp[1] - 0.5 * tmp[2]) / dt;
      else if (t == nt - 1) r = (0.5 * tmp[nt - 3] - 2.0 * tmp[nt - 2] + 1.5 * tmp[nt - 1]) / dt;
      else r = (tmp[t + 1] - tmp[t - 1]) * (0.5 / dt);
      v[p + size_t(t) * npix] = T(r);
    }
  }
}

// w_grad.m:24-108 (REFERENCE adjoint): sigma flipped, receivers hard-set to the
// time-reversed residual before each step, g -= u(nt-it) .* a, g *= dt.
// Returns a_max = |a| of the final step (w_grad.m:110-112).
template <class T>
inline void grad_reference(const Grid& g, const double* eps, const double* sig, const Shot& sh,
                           const T* e /*nt x nr*/, const T* u /*m x n x nt*/, T* gout, T* amax) {
  Layout L(g);
  std::vector<double> epsr, sigz;
  exp2pml(g, eps, sig, epsr, sigz);
  CoefT<T> c(build_coefs(g, epsr, sigz, sh.src_i, sh.src_j, -1.0));
  State<T> s(L.nodes());
  const int nr = int(sh.rec.size());
  const size_t mn = size_t(g.m) * g.n;
  std::vector<T> acc(mn, T(0));
  for (int it = 0; it < g.nt; ++it) {
    const int k = g.nt - 1 - it;  // 0-based forward step index of e(nt-it) / u(:,:,nt-it)
    for (int r = 0; r < nr; ++r) s.Ez[sh.rec[r]] = e[size_t(k) + size_t(r) * g.nt];  // w_grad.m:72
    step<T>(L, c, s, -1, T(0));
    for (int b = 0; b < g.n; ++b)
      for (int a = 0; a < g.m; ++a) {
        size_t p = size_t(a) + size_t(b) * g.m;
        T av = s.Ez[L.at(L.dom_i0 + a, L.dom_j0 + b)];
        acc[p] = acc[p] - u[p + size_t(k) * mn] * av;  // w_grad.m:87
        if (it == g.nt - 1 && amax) amax[p] = std::abs(av);
      }
  }
  for (size_t p = 0; p < mn; ++p) gout[p] = T(g.dt) * acc[p];  // w_grad.m:108
}

// Residual and misfit for the L2 objective (w_bozdag.m:48-50, w_E.m:7-16 with
// N = identity, normalised as w_update_e.m:75-76).
template <class T>
inline double residual_l2(const T* d, const T* dobs, size_t n, T* e) {
  double num = 0, den = 0;
  for (size_t i = 0; i < n; ++i) {
    T r = d[i] - dobs[i];
    e[i] = r;
    num += double(r) * double(r);
    den += double(dobs[i]) * double(dobs[i]);
  }
  return den > 0 ? 0.5 * num / den : 0.5 * num;
}

// ---------------------------------------------------------------------------
// EXACT adjoint: transpose of the discrete update of step<T>, run backwards,
// giving dJ/d(eps_r) and dJ/d(sigma) of J = 0.5*sum_t sum_r (d - d_obs)^2 with
// respect to the padded material cells, then mapped to the model through the
// transpose of exp2pml.  Contributions through the eps-dependent PML
// coefficients (bottom, left and right strips) are included.
// ---------------------------------------------------------------------------
template <class T>
struct AdjState {
  std::vector<T> lE, lHx, lHy, lEzx, lEzy;
  explicit AdjState(size_t N) : lE(N, T(0)), lHx(N, T(0)), lHy(N, T(0)), lEzx(N, T(0)), lEzy(N, T(0)) {}
};

// Reverse of one step.  s1 = forward state after the step, s0 = before it.
// ge/gs accumulate into padded-cell gradients (NX x NY, leading dimension NX).
template <class T>
struct AdjScratch {
  std::vector<T> px, py, lEmid, qx, qy;
  explicit AdjScratch(size_t N) : px(N), py(N), lEmid(N), qx(N), qy(N) {}
};

template <class T>
inline void adjoint_step(const Grid& g, const Layout& L, const CoefT<T>& c, const Coefs& cd,
                         const std::vector<double>& epsr, const std::vector<double>& sigz,
                         const State<T>& s0, const State<T>& s1, AdjState<T>& a,
                         std::vector<double>& ge, std::vector<double>& gs, AdjScratch<T>& w) {
  const int NX = L.NX, NY = L.NY;
  std::vector<T>& px = w.px;
  std::vector<T>& py = w.py;
  std::vector<T>& lEmid = w.lEmid;
  std::fill(px.begin(), px.end(), T(0));
  std::fill(py.begin(), py.end(), T(0));
  std::fill(lEmid.begin(), lEmid.end(), T(0));
  const double e0 = g.eps0, u0 = g.mu0, dt = g.dt;
  auto cell = [&](int I, int J) { return size_t(I) + size_t(J) * NX; };
  // E part (transpose of new_Ez / new_Ez_pml)
  for (int J = 1; J <= NY - 1; ++J)
    for (int I = 1; I <= NX - 1; ++I) {
      size_t k = L.at(I, J);
      double eps = epsr[cell(I, J)];
      if (L.ez_interior(I, J)) {
        T l = a.lE[k];
        double D = 2 * eps * e0 + dt * sigz[cell(I, J)];
        ge[cell(I, J)] += double(l) * (-2 * e0 / D) * (double(s1.Ez[k]) - double(s0.Ez[k]));
        gs[cell(I, J)] += double(l) * (-dt / D) * (double(s1.Ez[k]) + double(s0.Ez[k]));
        lEmid[k] = c.ce[k] * l;
        px[k] = c.chy[k] * l;
        py[k] = c.chx[k] * l;
      } else {
        T lx = a.lEzx[k] + a.lE[k], ly = a.lEzy[k] + a.lE[k];
        double dEzx = double(s1.Ezx[k]) - double(s0.Ezx[k]);
        double dEzy = double(s1.Ezy[k]) - double(s0.Ezy[k]);
        if (L.x_bot(I)) {
          double D = 2 * e0 * eps + dt * cd.sex[I];
          ge[cell(I, J)] += double(lx) * (-2 * e0 / D) * dEzx;
        } else if (!L.x_top(I)) {
          ge[cell(I, J)] += double(lx) * (-1.0 / eps) * dEzx;
        }
        if (L.y_strip(J)) {
          double D = 2 * e0 * eps + dt * cd.sey[J];
          ge[cell(I, J)] += double(ly) * (-2 * e0 / D) * dEzy;
        } else if (L.x_bot(I)) {
          ge[cell(I, J)] += double(ly) * (-1.0 / eps) * dEzy;
        }
        a.lEzx[k] = c.ax[k] * lx;
        a.lEzy[k] = c.ay[k] * ly;
        px[k] = c.bx[k] * lx;
        py[k] = c.by[k] * ly;
      }
    }
  // H part (transpose of new_H / new_H_pml)
  std::vector<T>& qx = w.qx;
  std::vector<T>& qy = w.qy;
  std::fill(qx.begin(), qx.end(), T(0));
  std::fill(qy.begin(), qy.end(), T(0));
  for (int J = 0; J <= NY - 1; ++J)
    for (int I = 0; I <= NX; ++I) {
      size_t k = L.at(I, J);
      T lt = a.lHx[k] + py[k] - py[k + L.ld];
      bool strip = !(J >= L.hx_j0 && J <= L.hx_j1) && I >= 1 && I <= NX - 1;
      if (strip) {
        double eps = epsr[cell(I, J)];
        double sm = cd.smy[J] / eps, Dm = 2 * u0 + dt * sm;
        ge[cell(I, J)] += double(lt) * (dt * sm / (eps * Dm)) * (double(s1.Hx[k]) + double(s0.Hx[k]));
      }
      a.lHx[k] = c.hxa[k] * lt;
      qx[k] = c.hxb[k] * lt;
    }
  for (int J = 0; J <= NY; ++J)
    for (int I = 0; I <= NX - 1; ++I) {
      size_t k = L.at(I, J);
      T lt = a.lHy[k] + px[k] - px[k + 1];
      bool strip = !(I >= L.hy_i0 && I <= L.hy_i1) && J >= 1 && J <= NY - 1;
      if (strip && L.x_bot(I)) {
        double eps = epsr[cell(I, J)];
        double sm = cd.smx[I] / eps, Dm = 2 * u0 + dt * sm;
        ge[cell(I, J)] += double(lt) * (dt * sm / (eps * Dm)) * (double(s1.Hy[k]) + double(s0.Hy[k]));
      }
      a.lHy[k] = c.hya[k] * lt;
      qy[k] = c.hyb[k] * lt;
    }
  for (int J = 0; J <= NY; ++J)
    for (int I = 0; I <= NX; ++I) {
      size_t k = L.at(I, J);
      if (L.ez_boundary(I, J)) { a.lE[k] = T(0); continue; }
      a.lE[k] = lEmid[k] + qx[k - L.ld] - qx[k] + qy[k - 1] - qy[k];
    }
}

// Maps padded-cell gradients back to the model through the transpose of exp2pml.
inline void pad_to_model(const Grid& g, const std::vector<double>& ge, const std::vector<double>& gs,
                         double* geps, double* gsig) {
  const int NX = g.NX(), NY = g.NY(), P = g.pml, Pt = g.pml_top, air = g.air;
  for (size_t p = 0; p < size_t(g.m) * g.n; ++p) { geps[p] = 0; gsig[p] = 0; }
  const int rows_mid = air + g.m;
  for (int J = 0; J < NY; ++J)
    for (int I = 0; I < NX; ++I) {
      int r = std::min(std::max(I - Pt, 0), rows_mid - 1);  // row of [air; model]
      if (r < air) continue;                                // air is not a model parameter
      int a = r - air;
      int b = std::min(std::max(J - P, 0), g.n - 1);
      geps[size_t(a) + size_t(b) * g.m] += ge[size_t(I) + size_t(J) * NX];
      bool in_model = I >= Pt + air && I < Pt + rows_mid && J >= P && J < P + g.n;
      if (in_model) gsig[size_t(a) + size_t(b) * g.m] += gs[size_t(I) + size_t(J) * NX];
    }
}

// Exact gradient for one shot with segment checkpointing (every K steps).
// e is the adjoint source dJ/dd (nt x nr).
template <class T>
inline void grad_exact(const Grid& g, const double* eps, const double* sig, const Shot& sh,
                       const T* e, double* geps, double* gsig) {
  Layout L(g);
  std::vector<double> epsr, sigz;
  exp2pml(g, eps, sig, epsr, sigz);
  Coefs cd = build_coefs(g, epsr, sigz, sh.src_i, sh.src_j);
  CoefT<T> c(cd);
  const long src = long(L.at(sh.src_i, sh.src_j));
  const int nt = g.nt;
  const int K = std::max(1, int(std::sqrt(double(nt))));
  std::vector<State<T>> ckpt;  // state before step k0 = s*K (0-based steps)
  State<T> s(L.nodes());
  for (int it = 0; it < nt; ++it) {
    if (it % K == 0) ckpt.push_back(s);
    step<T>(L, c, s, src, T(sh.wavelet[it]));
  }
  std::vector<double> ge(size_t(L.NX) * L.NY, 0.0), gs(size_t(L.NX) * L.NY, 0.0);
  AdjState<T> a(L.nodes());
  AdjScratch<T> scratch(L.nodes());
  const int nr = int(sh.rec.size());
  std::vector<State<T>> buf(K + 1, State<T>(L.nodes()));  // reused by every segment
  for (int seg = int(ckpt.size()) - 1; seg >= 0; --seg) {
    const int k0 = seg * K, k1 = std::min(nt, k0 + K);
    buf[0] = ckpt[seg];
    for (int it = k0; it < k1; ++it) {
      buf[it - k0 + 1] = buf[it - k0];
      step<T>(L, c, buf[it - k0 + 1], src, T(sh.wavelet[it]));
    }
    for (int it = k1 - 1; it >= k0; --it) {
      for (int r = 0; r < nr; ++r) a.lE[sh.rec[r]] += e[size_t(it) + size_t(r) * nt];
      adjoint_step<T>(g, L, c, cd, epsr, sigz, buf[it - k0], buf[it - k0 + 1], a, ge, gs, scratch);
    }
  }
  pad_to_model(g, ge, gs, geps, gsig);
}

}  // namespace gjo

// Robin coefficients of a DC source on the host (gj_dc_alphas): the private
// alphas of dc_Lk.m:820-960 in the compact layout of gj_dc_src.alpha, so that
// callers without the reference's MATLAB (or whose MATLAB cannot reach a
// private function) can fill gj_dc_src.alpha.
//
// For boundary node e and the two surface electrodes c (beta = +1 at A, -1 at
// B), with co / ca the distances of dc_Lk.m built from the spacings (signs
// kept) and r = hypot(co, ca):
//   alpha_e = sum_c beta_c ky K1(ky r) ca / r  /  sum_c beta_c K0(ky r),
// on the left side, the bottom and the right side, in the order
// [left h = 2..m-1 | bottom l = 2..n-1 | right h = 2..m-1 | c11 c21 c12 c22].
// K0 and K1 are taken exponentially scaled relative to the nearer electrode,
// so the ratio keeps its limit where the reference's besselk underflows (0/0).
#include <cmath>
#include <vector>

#include "../../include/gerjoii_gpu.h"

namespace {

// e^x K_nu(x) for nu = 0, 1 and x > 0: from std::cyl_bessel_k below x = 600,
// above it (where K_nu underflows) from the large-argument expansion
// sqrt(pi / 2x) sum_k prod_{j<=k} (4 nu^2 - (2j-1)^2) / (k! (8x)^k)
// (Abramowitz and Stegun 9.7.2; eight terms are below 1e-20 there).
double bessel_k_scaled(int nu, double x) {
  if (x < 600.0) return std::cyl_bessel_k(double(nu), x) * std::exp(x);
  const double mu = 4.0 * nu * nu;
  double term = 1.0, sum = 1.0;
  for (int k = 1; k <= 8; ++k) {
    const double odd = 2.0 * k - 1.0;
    term *= (mu - odd * odd) / (8.0 * k * x);
    sum += term;
  }
  return std::sqrt(M_PI / (2.0 * x)) * sum;
}

}  // namespace

extern "C" gj_status gj_dc_alphas(const gj_dc_grid* grid, long a_node, long b_node, const double* ky,
                                  double* alpha_out) {
  if (!grid || !ky || !alpha_out) return GJ_EINVAL;
  const int n = grid->n, m = grid->m, nky = grid->n_ky;
  if (n < 3 || m < 3 || nky < 1) return GJ_EINVAL;
  const long N = long(n) * m;
  if (a_node < 0 || a_node >= N || b_node < 0 || b_node >= N) return GJ_EINVAL;
  const double DX = grid->dx, DZ = grid->dz;
  const int col[2] = {int(a_node % n), int(b_node % n)};
  const double beta[2] = {1.0, -1.0};
  const int rows = 2 * m + n - 2;  // left side (m - 1), bottom (n), right side (m - 1)
  const int na = GJ_DC_NALPHA(n, m);
  std::vector<double> a(rows);
  for (int k = 0; k < nky; ++k) {
    for (int i = 0; i < rows; ++i) {
      double co[2], ca[2], x[2];
      for (int c = 0; c < 2; ++c) {
        if (i < m - 1) {  // left side, depth h = i + 1
          co[c] = (i + 1) * DZ;
          ca[c] = col[c] * DX;
        } else if (i < m - 1 + n) {  // bottom row, lateral l
          co[c] = std::abs((i - (m - 1)) - col[c]) * DX;
          ca[c] = (m - 1) * DZ;
        } else {  // right side, depth m - 1 - j
          co[c] = ((m - 1) - (i - (m - 1 + n))) * DZ;
          ca[c] = (n - 1 - col[c]) * DX;
        }
        x[c] = ky[k] * std::sqrt(co[c] * co[c] + ca[c] * ca[c]);
      }
      const double x0 = std::fmin(x[0], x[1]);
      double num = 0.0, den = 0.0;
      for (int c = 0; c < 2; ++c) {
        const double r = std::sqrt(co[c] * co[c] + ca[c] * ca[c]);
        const double sc = std::exp(-(x[c] - x0));
        num += beta[c] * ky[k] * bessel_k_scaled(1, x[c]) * sc * (ca[c] / r);
        den += beta[c] * bessel_k_scaled(0, x[c]) * sc;
      }
      a[i] = num / den;
    }
    double* out = alpha_out + size_t(k) * na;
    int o = 0;
    for (int i = 0; i < m - 2; ++i) out[o++] = a[i];                       // left, h = 2..m-1
    for (int i = m; i < m + n - 2; ++i) out[o++] = a[i];                   // bottom, l = 2..n-1
    for (int i = rows - 1; i >= m + n; --i) out[o++] = a[i];               // right, h = 2..m-1
    out[o++] = a[m - 2];                                                   // c11
    out[o++] = a[m - 1];                                                   // c21
    out[o++] = a[m + n - 2];                                               // c12
    out[o++] = a[m + n - 1];                                               // c22
  }
  return GJ_OK;
}

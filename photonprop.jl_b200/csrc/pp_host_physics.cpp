// Host-side (FP64) physics of PhotonProp.jl: the seawater medium, the
// Frank-Tamm spectrum tables and the PMT acceptance.  These build the small
// tables that a context keeps resident on the device; they run once per
// context, not per photon.
#include <cmath>
#include <vector>

#include "pp_internal.h"

namespace {

constexpr double kPi = 3.14159265358979323846;
constexpr double kAlpha = 7.2973525693e-3;  // CODATA2018 fine-structure constant (src/spectrum.jl:33)

// Quan & Fry refractive-index coefficients with the pressure term,
// src/medium.jl:131-154: n(x) = a01 + x (a2 + x (a3 + x a4)), x = 1 / wl[nm].
void fry(const pp_medium_desc* m, double& a01, double& a2, double& a3, double& a4) {
  const double n0 = 1.31405, n1 = 1.45e-5, n2 = 1.779e-4, n3 = 1.05e-6, n4 = 1.6e-8;
  const double n5 = 2.02e-6, n6 = 15.868, n7 = 0.01155, n8 = 0.00423, n9 = 4382.0, n10 = 1.1455e6;
  const double T = m->temperature, S = m->salinity, P = m->pressure;
  a01 = n0 + (n2 - n3 * T + n4 * T * T) * S - n5 * T * T + n1 * P;
  a2 = n6 + n7 * S - n8 * T;
  a3 = -n9;
  a4 = n10;
}

// Reference absorption-length knots, src/medium.jl:245-246.
const double kAbsWl[6] = {300.0, 365.0, 400.0, 450.0, 585.0, 800.0};
const double kAbsLen[6] = {10.4, 10.4, 14.5, 27.7, 7.1, 7.1};

// Linear interpolation on sorted knots, clamped at both ends (fast_linear_interp,
// src/utils.jl:10-34, with the lower index clamped).
double interp_sorted(double x, const double* xs, const double* ys, int n) {
  if (n <= 0) return 1.0;
  if (n == 1) return ys[0];
  x = std::min(std::max(x, xs[0]), xs[n - 1]);
  int hi = 0;
  while (hi < n && xs[hi] < x) ++hi;
  hi = std::min(std::max(hi, 1), n - 1);
  const int lo = hi - 1;
  const double along = (x - xs[lo]) / (xs[hi] - xs[lo]);
  return ys[lo] + (ys[hi] - ys[lo]) * along;
}

// Gauss-Legendre nodes/weights by Newton iteration on P_n (the three-term
// recurrence (j) P_j = (2j-1) x P_{j-1} - (j-1) P_{j-2} and
// P_n' = n (x P_n - P_{n-1}) / (x^2 - 1)); w = 2 / ((1 - x^2) P_n'^2).
void gauss_legendre(int n, std::vector<double>& x, std::vector<double>& w) {
  x.assign(n, 0.0);
  w.assign(n, 0.0);
  for (int i = 0; i < (n + 1) / 2; ++i) {
    double z = std::cos(kPi * (i + 0.75) / (n + 0.5));
    double dp = 0.0;
    for (int it = 0; it < 100; ++it) {
      double p0 = 1.0, p1 = z;
      for (int j = 2; j <= n; ++j) {
        const double p2 = ((2.0 * j - 1.0) * z * p1 - (j - 1.0) * p0) / j;
        p0 = p1;
        p1 = p2;
      }
      dp = n * (z * p1 - p0) / (z * z - 1.0);
      const double dz = p1 / dp;
      z -= dz;
      if (std::fabs(dz) < 1e-16) break;
    }
    {
      double p0 = 1.0, p1 = z;
      for (int j = 2; j <= n; ++j) {
        const double p2 = ((2.0 * j - 1.0) * z * p1 - (j - 1.0) * p0) / j;
        p0 = p1;
        p1 = p2;
      }
      dp = n * (z * p1 - p0) / (z * z - 1.0);
    }
    x[i] = -z;
    x[n - 1 - i] = z;
    w[i] = w[n - 1 - i] = 2.0 / ((1.0 - z * z) * dp * dp);
  }
}

// Photons per cm in [a, b]: GL-50 quadrature of the Frank-Tamm formula
// 2 pi alpha / wl^2 (1 - 1/n^2) (frank_tamm / frank_tamm_norm,
// src/spectrum.jl:32-45; integrate_gauss_quad, src/utils.jl:63-78).
double frank_tamm_norm(const pp_medium_desc* m, double a, double b, const std::vector<double>& x,
                       const std::vector<double>& w) {
  double a01, a2, a3, a4;
  fry(m, a01, a2, a3, a4);
  const double half = (b - a) / 2.0, mid = (a + b) / 2.0;
  double s = 0.0;
  for (size_t i = 0; i < x.size(); ++i) {
    const double wl = half * x[i] + mid;
    const double xi = 1.0 / wl;
    const double n = a01 + xi * (a2 + xi * (a3 + xi * a4));
    s += w[i] * (2.0 * kPi * kAlpha / (wl * wl) * (1.0 - 1.0 / (n * n))) * half;
  }
  return s * 1e7;
}

}  // namespace

namespace pp {

void medium_coeffs(const pp_medium_desc* m, double out[11]) {
  double a01, a2, a3, a4;
  fry(m, a01, a2, a3, a4);
  out[0] = a01;
  out[1] = a2;
  out[2] = a3;
  out[3] = a4;
  // get_sca_len_part_conc, src/medium.jl:206-210
  out[4] = 0.0017;
  out[5] = 1.34 * m->vol_conc_small_part;
  out[6] = 0.312 * m->vol_conc_large_part;
  out[7] = out[8] = out[9] = out[10] = 0.0;
}

void default_abs_table(double* wl, double* len, int* n) {
  for (int i = 0; i < 6; ++i) {
    wl[i] = kAbsWl[i];
    len[i] = kAbsLen[i];
  }
  *n = 6;
}

}  // namespace pp

extern "C" {

double pp_refractive_index(const pp_medium_desc* m, double wl) {
  double a01, a2, a3, a4;
  fry(m, a01, a2, a3, a4);
  const double x = 1.0 / wl;
  return a01 + x * (a2 + x * (a3 + x * a4));
}

double pp_group_index(const pp_medium_desc* m, double wl) {
  double a01, a2, a3, a4;
  fry(m, a01, a2, a3, a4);
  const double x = 1.0 / wl;
  return a01 + x * (2.0 * a2 + x * (3.0 * a3 + x * 4.0 * a4));
}

double pp_scattering_length(const pp_medium_desc* m, double wl) {
  const double x = 550.0 / wl;
  const double c = 0.0017 * std::pow(x, 4.3) + 1.34 * m->vol_conc_small_part * std::pow(x, 1.7) +
                   0.312 * m->vol_conc_large_part * std::pow(x, 0.3);
  return 1.0 / c;
}

double pp_absorption_length(const pp_medium_desc* m, double wl) {
  if (m->n_abs > 0) return interp_sorted(wl, m->abs_wl, m->abs_len, m->n_abs);
  return interp_sorted(wl, kAbsWl, kAbsLen, 6);
}

double pp_pmt_acceptance(const pp_pmt_desc* p, double wl) {
  if (!p || p->n <= 0) return 1.0;
  return interp_sorted(wl, p->wavelength, p->acceptance, p->n);
}

// CherenkovSpectrum knots: the CDF on a 1 nm grid (frank_tamm_inverted_cdf,
// src/spectrum.jl:54-70), inverted by piecewise-linear interpolation and
// sampled at n equidistant CDF values (src/spectrum.jl:77-82,96-101).
pp_status pp_cherenkov_knots(const pp_medium_desc* m, double wl_min, double wl_max, int32_t n_knots,
                             double* out) {
  if (!m || !out || n_knots < 2 || n_knots > PP_MAX_KNOTS || !(wl_max > wl_min) || !(wl_min > 0.0))
    return PP_ERR_ARG;
  std::vector<double> x, w;
  gauss_legendre(50, x, w);
  const int n_grid = (int)std::floor(wl_max - wl_min + 1e-9) + 1;
  std::vector<double> wl(n_grid), cdf(n_grid);
  const double full = frank_tamm_norm(m, wl_min, wl_max, x, w);
  for (int i = 0; i < n_grid; ++i) {
    wl[i] = wl_min + (double)i;
    cdf[i] = i == 0 ? 0.0 : frank_tamm_norm(m, wl_min, wl[i], x, w) / full;
  }
  for (int j = 0; j < n_knots; ++j) {
    const double u = (double)j / (double)(n_knots - 1);
    if (u <= cdf[0]) {
      out[j] = wl[0];
      continue;
    }
    if (u >= cdf[n_grid - 1]) {
      out[j] = wl[n_grid - 1];
      continue;
    }
    int k = 1;
    while (k < n_grid - 1 && cdf[k] < u) ++k;
    const double f = (u - cdf[k - 1]) / (cdf[k] - cdf[k - 1]);
    out[j] = wl[k - 1] + f * (wl[k] - wl[k - 1]);
  }
  return PP_OK;
}

}  // extern "C"

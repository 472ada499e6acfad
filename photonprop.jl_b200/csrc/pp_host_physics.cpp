// Host-side (FP64) physics of PhotonProp.jl: the seawater medium, the
// Frank-Tamm spectrum tables and the PMT acceptance.  These build the small
// tables that a context keeps resident on the device; they run once per
// context, not per photon.
#include <cmath>
#include <mutex>
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

void gl_nodes(int n, double* x, double* w) {
  std::vector<double> xv, wv;
  gauss_legendre(n, xv, wv);
  for (int i = 0; i < n; ++i) {
    x[i] = xv[i];
    w[i] = wv[i];
  }
}

double frank_tamm_norm_cm(const pp_medium_desc* m, double wl_min, double wl_max) {
  std::vector<double> x, w;
  gauss_legendre(50, x, w);
  return frank_tamm_norm(m, wl_min, wl_max, x, w);
}

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

namespace pp {

// Gamma(s, z), the upper incomplete gamma function, for s > 0, z >= 0.  Below
// z = s + 1 it is Gamma(s) minus the lower function, whose power series
// gamma(s, z) = z^s e^-z sum_k z^k / (s (s+1) ... (s+k)) converges fast there;
// above, Legendre's continued fraction
// Gamma(s, z) = e^-z z^s / (z + 1 - s - 1 (1 - s) / (z + 3 - s - 2 (2 - s) / ...))
// evaluated by the modified Lentz method.
double upper_incomplete_gamma(double s, double z) {
  if (!(s > 0.0) || !(z >= 0.0)) return NAN;
  if (z == 0.0) return std::tgamma(s);
  const double lpre = s * std::log(z) - z;
  if (z < s + 1.0) {
    double term = 1.0 / s, sum = term;
    for (int k = 1; k < 1000; ++k) {
      term *= z / (s + k);
      sum += term;
      if (std::fabs(term) < std::fabs(sum) * 1e-17) break;
    }
    return std::tgamma(s) - std::exp(lpre) * sum;
  }
  const double tiny = 1e-300;
  double b = z + 1.0 - s, c = 1.0 / tiny, d = 1.0 / b, f = d;
  for (int k = 1; k < 1000; ++k) {
    const double an = -k * (k - s);
    b += 2.0;
    d = an * d + b;
    if (std::fabs(d) < tiny) d = tiny;
    c = b + an / c;
    if (std::fabs(c) < tiny) c = tiny;
    d = 1.0 / d;
    const double delta = d * c;
    f *= delta;
    if (std::fabs(delta - 1.0) < 1e-16) break;
  }
  return std::exp(lpre) * f;
}

// gamma(s, z), the lower incomplete gamma function: the power series below
// z = s + 1, Gamma(s) - Gamma(s, z) above.
double lower_incomplete_gamma(double s, double z) {
  if (!(z > 0.0)) return 0.0;
  if (z < s + 1.0) {
    double term = 1.0 / s, sum = term;
    for (int k = 1; k < 1000; ++k) {
      term *= z / (s + k);
      sum += term;
      if (std::fabs(term) < std::fabs(sum) * 1e-17) break;
    }
    return std::exp(s * std::log(z) - z) * sum;
  }
  return std::tgamma(s) - upper_incomplete_gamma(s, z);
}

// Antiderivative of a exp(b |v|^c) + d: with k = -b,
// sign(v) (a/c) k^(-1/c) gamma(1/c, k |v|^c) + d v.
double cascade_G(double v) {
  const double k = -kAngB, s = 1.0 / kAngC;
  const double p = (kAngA / kAngC) * std::pow(k, -s) * lower_incomplete_gamma(s, k * std::pow(std::fabs(v), kAngC));
  return (v < 0.0 ? -p : p) + kAngD * v;
}

void cascade_tables(double* fwd, double* inv) {
  const double dv = (kCascVMax - kCascVMin) / kCascNF;
  for (int i = 0; i <= kCascNF; ++i) fwd[i] = cascade_G(kCascVMin + dv * i);
  const double g0 = fwd[0], g1 = fwd[kCascNF];
  inv[0] = kCascVMin;
  inv[kCascNI] = kCascVMax;
  for (int j = 1; j < kCascNI; ++j) {
    const double level = g0 + (g1 - g0) * j / kCascNI;
    double lo = kCascVMin, hi = kCascVMax;
    for (int it = 0; it < 64; ++it) {
      const double mid = 0.5 * (lo + hi);
      if (cascade_G(mid) < level) lo = mid; else hi = mid;
    }
    inv[j] = 0.5 * (lo + hi);
  }
}

// Inverse-CDF sample of cos(theta) at refractive index n: G at the ends of
// [-1 - 1/n, 1 - 1/n] from the forward table, the level u of the way between
// them, v from the inverse table (linear interpolation throughout).
double cascade_sample(const double* fwd, const double* inv, double u, double n) {
  const double c0 = 1.0 / n;
  auto lerp_tab = [](const double* t, int cells, double x) {
    x = std::min(std::max(x, 0.0), (double)cells);
    int i = std::min((int)x, cells - 1);
    return t[i] + (x - i) * (t[i + 1] - t[i]);
  };
  const double inv_dv = kCascNF / (kCascVMax - kCascVMin);
  const double gl = lerp_tab(fwd, kCascNF, (-1.0 - c0 - kCascVMin) * inv_dv);
  const double gh = lerp_tab(fwd, kCascNF, (1.0 - c0 - kCascVMin) * inv_dv);
  const double g0 = fwd[0], g1 = fwd[kCascNF];
  const double v = lerp_tab(inv, kCascNI, (gl + u * (gh - gl) - g0) * kCascNI / (g1 - g0));
  return std::min(std::max(v + c0, -1.0), 1.0);
}

// The reference's antiderivative of a exp(b |x - cos_c|^c) + d
// (src/emission.jl:65-81): with u = |x - cos_c| and k = -b,
// F(x) = d x + (a / c) (cos_c - x) Gamma(1/c, k u^c) (k u^c)^(-1/c); above the
// peak the reference adds twice its value just below the peak
// (peak_val = F(cos_c - 1e-5)), which is what joins the two branches in its
// closed form.  Kept as the reference has it, including the d cos_c share of
// peak_val, so that the normalisation matches.
namespace {
double ang_branch(double x, double cos_c, double u) {
  const double k = -kAngB;
  const double ku = k * std::pow(u, kAngC);
  return (1.0 / kAngC) * (kAngC * kAngD * x +
                          kAngA * (cos_c - x) * upper_incomplete_gamma(1.0 / kAngC, ku) * std::pow(ku, -1.0 / kAngC));
}
double ang_indef(double x, double cos_c) {
  const double peak_val = ang_branch(cos_c - 1e-5, cos_c, 1e-5);
  if (x <= cos_c) return ang_branch(x, cos_c, cos_c - x);
  return ang_branch(x, cos_c, x - cos_c) + 2.0 * peak_val;
}
}  // namespace

double cherenkov_ang_dist_int_closed(double ref_index, double lower, double upper) {
  const double cos_c = 1.0 / ref_index;
  return ang_indef(upper, cos_c) - ang_indef(lower, cos_c);
}

void cherenkov_ang_dist_int_table(double* out) {
  for (int i = 0; i < kAngIntN; ++i) out[i] = cherenkov_ang_dist_int_closed(kAngIntN0 + kAngIntDn * i, -1.0, 1.0);
}

// LinearInterpolation(1.1:0.01:1.5, table) inside the range, NaN outside
// (the reference's interpolation throws there).
double ang_int_interp(const double* table, double n) {
  const double x = (n - kAngIntN0) / kAngIntDn;
  if (!(x >= -1e-9) || !(x <= kAngIntN - 1 + 1e-9)) return NAN;
  int i = (int)std::floor(x);
  i = std::min(std::max(i, 0), kAngIntN - 2);
  const double f = x - i;
  return table[i] + f * (table[i + 1] - table[i]);
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

// ---- Cherenkov angular distribution of EM cascades (src/emission.jl:19-99) ----

double pp_cherenkov_ang_dist(double costheta, double ref_index) {
  const double cos_c = 1.0 / ref_index;
  return pp::kAngA * std::exp(pp::kAngB * std::pow(std::fabs(costheta - cos_c), pp::kAngC)) + pp::kAngD;
}

double pp_cherenkov_ang_dist_int_exact(double ref_index, double lower, double upper) {
  return pp::cherenkov_ang_dist_int_closed(ref_index, lower, upper);
}

double pp_cherenkov_ang_dist_int(double ref_index) {
  double table[pp::kAngIntN];
  pp::cherenkov_ang_dist_int_table(table);
  return pp::ang_int_interp(table, ref_index);
}

double pp_cascade_cos_theta(double u, double n) {
  static std::vector<double> fwd, inv;
  static std::once_flag once;
  std::call_once(once, [] {
    fwd.resize(pp::kCascNF + 1);
    inv.resize(pp::kCascNI + 1);
    pp::cascade_tables(fwd.data(), inv.data());
  });
  if (!(n > 0.0)) return NAN;
  return pp::cascade_sample(fwd.data(), inv.data(), u, n);
}

pp_status pp_dir_reweight(const double* thetas, double obs_angle, const double* ref_ixs, double* out, int64_t n) {
  if (n < 0 || (n > 0 && (!thetas || !ref_ixs || !out))) return PP_ERR_ARG;
  double table[pp::kAngIntN];
  pp::cherenkov_ang_dist_int_table(table);
  for (int64_t i = 0; i < n; ++i)
    out[i] = pp_cherenkov_ang_dist(std::cos(thetas[i] - obs_angle), ref_ixs[i]) /
             (2.0 * pp::ang_int_interp(table, ref_ixs[i]));
  return PP_OK;
}

}  // extern "C"

"""FP64 numpy/scipy restatement of the reference's fit stage.  TEST
INFRASTRUCTURE ONLY: the checker of the library's reweighting and Gamma-fit
kernels and of its host functions.

Follows:
  cherenkov_ang_dist              src/emission.jl:32-44 (e- parameters, :19)
  _cherenkov_ang_dist_int         src/emission.jl:52-86 (closed form with the
                                  upper incomplete gamma function, including
                                  the reference's peak_val join)
  cherenkov_ang_dist_int          src/emission.jl:88-99 (linear interpolation
                                  on 1.1:0.01:1.5)
  get_dir_reweight                src/modelling.jl:46-49
  fit_photon_dist                 src/modelling.jl:52-79
The weighted Gamma fit (Distributions.jl 0.25.62 fit_mle(Gamma, x, w), not
vendored) is restated as Minka's generalised Newton iteration on the
sufficient statistics (sum w, sum w x, sum w ln x); tests pin it against
scipy.stats.gamma.fit, an independent optimiser.
"""
from __future__ import annotations

import numpy as np
from scipy import special

A, B, C, D = 4.27033, -6.02527, 0.29887, -0.00103
INT_N0, INT_DN, INT_N = 1.1, 0.01, 41


def cherenkov_ang_dist(costheta, ref_index):
    cos_c = 1.0 / np.asarray(ref_index, dtype=np.float64)
    return A * np.exp(B * np.abs(np.asarray(costheta, dtype=np.float64) - cos_c) ** C) + D


def upper_gamma(s, z):
    return special.gammaincc(s, z) * special.gamma(s)


def _branch(x, cos_c, u):
    ku = -B * u ** C
    return (1.0 / C) * (C * D * x + A * (cos_c - x) * upper_gamma(1.0 / C, ku) * ku ** (-1.0 / C))


def _indef(x, cos_c):
    peak_val = _branch(cos_c - 1e-5, cos_c, 1e-5)
    if x <= cos_c:
        return _branch(x, cos_c, cos_c - x)
    return _branch(x, cos_c, x - cos_c) + 2.0 * peak_val


def cherenkov_ang_dist_int_exact(ref_index, lower=-1.0, upper=1.0):
    cos_c = 1.0 / ref_index
    return _indef(upper, cos_c) - _indef(lower, cos_c)


def join_offset(ref_index):
    """What the reference's peak_val join adds to the true integral:
    2 peak_val - 2 (a/c) k^(-1/c) Gamma(1/c), k = -b."""
    cos_c = 1.0 / ref_index
    k = -B
    true_jump = 2.0 * (A / C) * k ** (-1.0 / C) * special.gamma(1.0 / C)
    return 2.0 * _branch(cos_c - 1e-5, cos_c, 1e-5) - true_jump


def int_table():
    return np.array([cherenkov_ang_dist_int_exact(INT_N0 + INT_DN * i) for i in range(INT_N)])


def cherenkov_ang_dist_int(ref_index, table=None):
    t = int_table() if table is None else table
    x = (np.asarray(ref_index, dtype=np.float64) - INT_N0) / INT_DN
    i = np.clip(np.floor(x).astype(np.int64), 0, INT_N - 2)
    f = x - i
    out = t[i] + f * (t[i + 1] - t[i])
    return np.where((x >= -1e-9) & (x <= INT_N - 1 + 1e-9), out, np.nan)


def get_dir_reweight(thetas, obs_angle, ref_ixs, table=None):
    norm = cherenkov_ang_dist_int(ref_ixs, table) * 2.0
    return cherenkov_ang_dist(np.cos(np.asarray(thetas) - obs_angle), ref_ixs) / norm


def gamma_fit_moments(sw, swx, swlx, tol=1e-14, maxiter=100):
    """(alpha, theta) maximising the weighted Gamma likelihood."""
    if not sw > 0:
        return np.nan, np.nan
    mx = swx / sw
    ml = swlx / sw
    lmx = np.log(mx)
    s = lmx - ml
    if not (s > 0 and np.isfinite(s)):
        return np.nan, np.nan
    a = (3.0 - s + np.sqrt((s - 3.0) ** 2 + 24.0 * s)) / (12.0 * s)
    with np.errstate(all="ignore"):
        a = _newton(a, ml, lmx, tol, maxiter)
    if not (a > 0 and np.isfinite(a)):
        return np.nan, np.nan
    return a, mx / a


def _newton(a, ml, lmx, tol, maxiter):
    for _ in range(maxiter):
        ia = 1.0 / a
        z = ia + (ml - lmx + np.log(a) - special.digamma(a)) / (a * a * (ia - special.polygamma(1, a)))
        an = 1.0 / z
        done = abs(an - a) <= tol * a
        a = an
        if done or not a > 0:
            break
    return a


def gamma_fit(x, w):
    x = np.asarray(x, dtype=np.float64)
    w = np.asarray(w, dtype=np.float64)
    return gamma_fit_moments(w.sum(), (w * x).sum(), (w * np.log(x)).sum())


def moments(tres, weight):
    """[sum w (all), sum w, sum w tres, sum w ln tres] over tres > 0 (the
    reference masks tres >= 0; an exact 0 has no Gamma likelihood)."""
    tres = np.asarray(tres, dtype=np.float64)
    w = np.asarray(weight, dtype=np.float64)
    m = tres > 0
    with np.errstate(divide="ignore", invalid="ignore"):
        lt = np.where(m, np.log(np.where(m, tres, 1.0)), 0.0)
    return np.array([w.sum(), w[m].sum(), (w[m] * tres[m]).sum(), (w[m] * lt[m]).sum()])


def fit_photon_dist(obs_angles, tres, thetas, ref_ix, abs_weight, pmt_weight, n_ph_gen, table=None):
    """Rows (obs_angle, fit_alpha, fit_theta, det_fraction), moments."""
    rows, mom = [], []
    for a in obs_angles:
        w = get_dir_reweight(thetas, a, ref_ix, table) * abs_weight * pmt_weight
        m = moments(tres, w)
        al, th = gamma_fit_moments(m[1], m[2], m[3])
        rows.append((a, al, th, m[0] / n_ph_gen))
        mom.append(m)
    return np.array(rows), np.array(mom)


# ---- cascade emitter: inverse-CDF sampling of the angular profile --------
CASC_NF, CASC_NI, CASC_VMIN, CASC_VMAX = 2048, 8192, -1.85, 0.35
_CASC = None


def cascade_G(v):
    """Antiderivative of a exp(b |v|^c) + d: sign(v) (a/c) k^(-1/c) gamma(1/c, k |v|^c) + d v
    (k = -b; scipy's regularised lower incomplete gamma times Gamma(1/c))."""
    v = np.asarray(v, dtype=np.float64)
    k, s = -B, 1.0 / C
    p = (A / C) * k ** (-s) * special.gammainc(s, k * np.abs(v) ** C) * special.gamma(s)
    return np.sign(v) * p + D * v


def cascade_tables():
    """(forward G table, inverse v table, vmin, dv, gmin, dg), FP64."""
    global _CASC
    if _CASC is None:
        v = CASC_VMIN + (CASC_VMAX - CASC_VMIN) / CASC_NF * np.arange(CASC_NF + 1)
        fwd = cascade_G(v)
        levels = fwd[0] + (fwd[-1] - fwd[0]) * np.arange(CASC_NI + 1) / CASC_NI
        lo = np.full_like(levels, CASC_VMIN)
        hi = np.full_like(levels, CASC_VMAX)
        for _ in range(64):
            mid = 0.5 * (lo + hi)
            below = cascade_G(mid) < levels
            lo = np.where(below, mid, lo)
            hi = np.where(below, hi, mid)
        inv = 0.5 * (lo + hi)
        inv[0], inv[-1] = CASC_VMIN, CASC_VMAX
        _CASC = (np.ascontiguousarray(fwd), np.ascontiguousarray(inv), CASC_VMIN,
                 (CASC_VMAX - CASC_VMIN) / CASC_NF, float(fwd[0]), float(fwd[-1] - fwd[0]) / CASC_NI)
    return _CASC


def cascade_cos_theta(u, n):
    """cos(theta) sampled from the profile at refractive index n for uniform u."""
    fwd, inv, vmin, dv, gmin, dg = cascade_tables()

    def lerp(t, x):
        cells = len(t) - 1
        x = np.clip(x, 0.0, cells)
        i = np.minimum(np.floor(x).astype(np.int64), cells - 1)
        return t[i] + (x - i) * (t[i + 1] - t[i])
    c0 = 1.0 / np.asarray(n, dtype=np.float64)
    gl = lerp(fwd, (-1.0 - c0 - vmin) / dv)
    gh = lerp(fwd, (1.0 - c0 - vmin) / dv)
    v = lerp(inv, (gl + np.asarray(u, dtype=np.float64) * (gh - gl) - gmin) / dg)
    return np.clip(v + c0, -1.0, 1.0)


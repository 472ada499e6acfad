"""FP64 CPU restatement of PhotonProp.jl's physics tables.

TEST INFRASTRUCTURE ONLY.  This module is the oracle's half of the medium,
spectrum and detection physics; only ``tests/``, ``__graft_entry__.smoke()``
and ``bench.py``'s CPU-baseline leg may import it, and only as the checker.
The product (``photonprop.jl_b200``) has its own C++ implementation of the
same formulas and never imports anything under ``oracle/``.

Parity status: the helper known-answer tests of the reference
(``src/tests/test_photon_prob.jl``) pin the interpolators; the medium and
spectrum formulas are restated from the reference source (no reference run is
possible here: Julia is absent), so their spot values are pinned only by the
reference's own constants.

Every function cites the reference file:line it restates.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

# PhysicalConstants CODATA2018 (src/photon_prop_cuda.jl:635, src/spectrum.jl:33)
C_VACUUM_M_PER_NS = 0.299792458
FINE_STRUCTURE = 7.2973525693e-3
BAR_PER_ATM = 1.01325

# Absorption-length knots, src/medium.jl:245-246
ABS_WL = np.array([300.0, 365.0, 400.0, 450.0, 585.0, 800.0])
ABS_LEN = np.array([10.4, 10.4, 14.5, 27.7, 7.1, 7.1])


@dataclass
class Water:
    """WaterProperties, src/medium.jl:23-50 (salinity permille, pressure atm,
    temperature degC, particle concentrations ppm, X0 g/cm^2)."""

    salinity: float
    pressure: float
    temperature: float
    vol_conc_small_part: float
    vol_conc_large_part: float
    radiation_length: float = 36.08


def cascadia(salinity=34.82, temperature=1.8) -> Water:
    """make_cascadia_medium_properties, src/medium.jl:52-58 (269.44088 bar)."""
    return Water(salinity, 269.44088 / BAR_PER_ATM, temperature, 0.0075, 0.0075, 36.08)


def _fry_coeffs(m: Water):
    """Quan-Fry coefficients, src/medium.jl:131-154."""
    n0, n1, n2, n3, n4 = 1.31405, 1.45e-5, 1.779e-4, 1.05e-6, 1.6e-8
    n5, n6, n7, n8, n9, n10 = 2.02e-6, 15.868, 0.01155, 0.00423, 4382.0, 1.1455e6
    t, s, p = m.temperature, m.salinity, m.pressure
    a01 = n0 + (n2 - n3 * t + n4 * t * t) * s - n5 * t * t + n1 * p
    a2 = n6 + n7 * s - n8 * t
    return a01, a2, -n9, n10


def refractive_index(wl, m: Water):
    """get_refractive_index_fry, src/medium.jl:125-158 (phase index)."""
    a01, a2, a3, a4 = _fry_coeffs(m)
    x = 1.0 / np.asarray(wl, dtype=np.float64)
    return a01 + x * (a2 + x * (a3 + x * a4))


def group_index(wl, m: Water):
    """Group index n - lambda dn/dlambda of the Quan-Fry polynomial
    (src/medium.jl:143-157 differentiated analytically; the reference itself
    only uses the phase index, src/photon_prop_cuda.jl:634-638)."""
    a01, a2, a3, a4 = _fry_coeffs(m)
    x = 1.0 / np.asarray(wl, dtype=np.float64)
    return a01 + x * (2.0 * a2 + x * (3.0 * a3 + x * 4.0 * a4))


def scattering_length(wl, m: Water):
    """get_sca_len_part_conc, src/medium.jl:201-214."""
    x = 550.0 / np.asarray(wl, dtype=np.float64)
    coeff = (0.0017 * x ** 4.3 + 1.34 * m.vol_conc_small_part * x ** 1.7
             + 0.312 * m.vol_conc_large_part * x ** 0.3)
    return 1.0 / coeff


def interp_sorted(x, xs, ys):
    """fast_linear_interp(x, xs, ys), src/utils.jl:10-34: clamp, then linear
    interpolation on the segment found by searchsortedfirst.  The reference
    reads xs[0] when x == xs[1] (1-based); the lower index is clamped here,
    which gives the same value ys[1]."""
    xs = np.asarray(xs, dtype=np.float64)
    ys = np.asarray(ys, dtype=np.float64)
    x = np.clip(np.asarray(x, dtype=np.float64), xs[0], xs[-1])
    hi = np.searchsorted(xs, x, side="left")  # searchsortedfirst, 0-based
    hi = np.clip(hi, 1, len(xs) - 1)
    lo = hi - 1
    along = (x - xs[lo]) / (xs[hi] - xs[lo])
    return ys[lo] + (ys[hi] - ys[lo]) * along


def interp_equidistant(x, knots, lower, upper):
    """fast_linear_interp(x, knots, lower, upper), src/utils.jl:37-60."""
    knots = np.asarray(knots, dtype=np.float64)
    x = np.clip(np.asarray(x, dtype=np.float64), lower, upper)
    n = len(knots)
    step = (upper - lower) / (n - 1)
    along = (x - lower) / step
    fl = np.floor(along)
    i = fl.astype(np.int64)
    last = i >= n - 1
    i = np.minimum(i, n - 2)
    frac = along - fl
    val = knots[i] + (knots[i + 1] - knots[i]) * frac
    return np.where(last, knots[-1], val)


def absorption_length(wl, m: Water | None = None):
    """get_absorption_length, src/medium.jl:243-251."""
    return interp_sorted(wl, ABS_WL, ABS_LEN)


def gauss_legendre(order=50):
    """FastGaussQuadrature.gausslegendre(50), src/utils.jl:8."""
    return np.polynomial.legendre.leggauss(order)


def integrate_gauss_quad(f, a, b, order=50):
    """integrate_gauss_quad + transform_integral_range, src/utils.jl:63-78."""
    nodes, weights = gauss_legendre(order)
    half = (b - a) / 2.0
    u = half * nodes + (a + b) / 2.0
    return float(np.dot(weights, f(u) * half))


def frank_tamm(wl, n):
    """frank_tamm, src/spectrum.jl:32-34."""
    return 2.0 * math.pi * FINE_STRUCTURE / wl ** 2 * (1.0 - 1.0 / n ** 2)


def frank_tamm_norm(wl_range, m: Water):
    """frank_tamm_norm, src/spectrum.jl:42-45 (cm^-1)."""
    f = lambda wl: frank_tamm(wl, refractive_index(wl, m))
    return integrate_gauss_quad(f, wl_range[0], wl_range[1]) * 1e7


def frank_tamm_inverted_cdf(wl_range, m: Water, step=1.0):
    """frank_tamm_inverted_cdf, src/spectrum.jl:54-70."""
    wl_steps = np.arange(wl_range[0], wl_range[1] + step / 2, step)
    full = frank_tamm_norm(wl_range, m)
    norms = np.zeros(len(wl_steps))
    for i in range(1, len(wl_steps)):
        norms[i] = frank_tamm_norm((wl_range[0], wl_steps[i]), m) / full
    order = np.argsort(norms, kind="stable")
    return norms[order], wl_steps[order]


def cherenkov_spectrum_knots(wl_range, n_knots, m: Water):
    """CherenkovSpectrum(wl_range, interp_steps, medium).knots,
    src/spectrum.jl:77-82,96-101: the gridded linear interpolation of
    (CDF -> wavelength) evaluated at n equidistant CDF values."""
    norms, wls = frank_tamm_inverted_cdf(wl_range, m)
    return np.interp(np.linspace(0.0, 1.0, n_knots), norms, wls)


def load_pmt_table(path):
    """PMTAcc.csv as read by src/detection.jl:31-33 (wavelength, acceptance)."""
    d = np.loadtxt(path, delimiter=",")
    return d[:, 0].copy(), d[:, 1].copy()


def pmt_acceptance(wl, table):
    """p_one_pmt_acc, src/detection.jl:18-33: gridded linear interpolation
    (Interpolations.jl LinearInterpolation; clamped here at the table ends)."""
    xs, ys = table
    return np.interp(np.asarray(wl, dtype=np.float64), xs, ys)


# Cherenkov angular profile, src/emission.jl:32-44 (e- parameters :23)
ANG_A, ANG_B, ANG_C, ANG_D = 4.27033, -6.02527, 0.29887, -0.00103


def cherenkov_ang_dist(costheta, ref_index):
    """cherenkov_ang_dist, src/emission.jl:32-44."""
    ctc = 1.0 / np.asarray(ref_index, dtype=np.float64)
    return ANG_A * np.exp(ANG_B * np.abs(np.asarray(costheta) - ctc) ** ANG_C) + ANG_D

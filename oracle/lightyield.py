"""FP64 numpy/scipy restatement of the reference's light-yield module.  TEST
INFRASTRUCTURE ONLY: the checker of the library's light-yield host functions
and of its particle -> source kernel.

Follows src/lightyield.jl:
  parameters                     :35-37, :46-69
  longitudinal_profile           :116-140 (L_rad = X0 / density x 1000 cm, :121-122)
  fractional_contrib_long!       :143-169 (50-point Gauss-Legendre, numpy's nodes)
  cherenkov_track_length(_dev)   :186-198
  particle_to_elongated_lightsource! :229-262
and the water density of src/medium.jl:60-78 (DIPPR105), both the
reference's expression (temperature in degC, (1 - T)/C) and the DIPPR105
form with the temperature in kelvin.
"""
from __future__ import annotations

import numpy as np
from scipy import special

from . import tables as tb

LONG = {11: (2.01849, 1.45469, 0.63207), -11: (2.00035, 1.45501, 0.63008), 22: (2.83923, 1.34031, 0.64526)}
TRACK = {11: (532.07078881, 1.00000211, 5.78170887, 0.5), -11: (532.11320598, 0.99999254, 5.73419669, 0.5),
         22: (532.08540905, 0.99999877, 5.78170887, 5.66586567)}
DA, DB, DC, DD = 0.14395, 0.0112, 649.727, 0.05107
C_VAC = 0.299792458
GL_X, GL_W = np.polynomial.legendre.leggauss(50)


def density(m: tb.Water, mode="reference"):
    T = m.temperature
    if mode == "reference":
        return DA / DB ** ((1 + (1 - T) / DC) ** DD)
    return DA / DB ** (1 + (1 - (T + 273.15) / DC) ** DD)


def rad_length_cm(m: tb.Water, mode="reference"):
    return m.radiation_length / density(m, mode) * 1000.0


def longitudinal_profile(energy, z_cm, m: tb.Water, ptype, mode="reference"):
    alpha, beta, b = LONG[int(ptype)]
    t = np.asarray(z_cm, dtype=np.float64) / rad_length_cm(m, mode)
    a = alpha + beta * np.log10(energy)
    return b * ((t * b) ** (a - 1.0) * np.exp(-(t * b)) / special.gamma(a))


def gl(f, lo, hi):
    half, mid = (hi - lo) / 2.0, (hi + lo) / 2.0
    return float(np.sum(GL_W * f(half * GL_X + mid)) * half)


def fractional_contrib_long(energy, z_grid, m, ptype, mode="reference"):
    z = np.asarray(z_grid, dtype=np.float64)
    f = lambda x: longitudinal_profile(energy, x, m, ptype, mode)
    norm = gl(f, z.min(), z.max())
    out = np.zeros_like(z)
    for i in range(len(z) - 1):
        out[i + 1] = gl(f, z[i], z[i + 1]) / norm
    return out


def cherenkov_track_length(energy, ptype):
    a, b, _, _ = TRACK[int(ptype)]
    return a * energy ** b


def cherenkov_track_length_dev(energy, ptype):
    _, _, a, b = TRACK[int(ptype)]
    return a * energy ** b


def elongated_sources(pos, direction, time, energy, ptype, grid, m, wl_range, mode="reference"):
    """[(position, time, photons)] of the grid intervals; the grid values are
    centimetres in the profile (times 100 in mode "metres") and metres along
    the particle."""
    g = np.asarray(grid, dtype=np.float64)
    zc = g * (1.0 if mode == "reference" else 100.0)
    frac = fractional_contrib_long(energy, zc, m, ptype, mode)
    total = tb.frank_tamm_norm(wl_range, m) * cherenkov_track_length(energy, ptype)
    out = []
    for i in range(1, len(g)):
        mid = 0.5 * (g[i - 1] + g[i])
        out.append((np.asarray(pos, dtype=np.float64) + mid * np.asarray(direction, dtype=np.float64),
                    time + mid / C_VAC, int(np.rint(total * frac[i]))))
    return out

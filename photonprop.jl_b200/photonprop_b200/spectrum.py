"""Spectral module of PhotonProp.jl (src/spectrum.jl)."""
from __future__ import annotations

import numpy as np

from . import _lib
from .medium import WaterProperties


class Spectrum:
    pass


class Monochromatic(Spectrum):
    """Monochromatic(wavelength), src/spectrum.jl:14-16."""

    def __init__(self, wavelength: float):
        self.wavelength = float(wavelength)

    def desc(self):
        d = _lib.SpectrumDesc()
        d.kind = _lib.SPECTRUM_MONOCHROMATIC
        d.n_knots = 1
        d.wl_min = d.wl_max = self.wavelength
        return d

    @property
    def knots(self):
        return np.array([self.wavelength])


class CherenkovSpectrum(Spectrum):
    """CherenkovSpectrum(wl_range, interp_steps, medium), src/spectrum.jl:90-103:
    `knots` are the inverse Frank-Tamm CDF at interp_steps equidistant points."""

    def __init__(self, wl_range=(300.0, 800.0), interp_steps: int = 20,
                 medium: WaterProperties | None = None):
        if medium is None:
            raise ValueError("CherenkovSpectrum needs a medium")
        self.wl_range = (float(wl_range[0]), float(wl_range[1]))
        self.interp_steps = int(interp_steps)
        self.medium = medium
        out = np.zeros(self.interp_steps)
        _lib.check(_lib.load().pp_cherenkov_knots(medium.desc(), self.wl_range[0], self.wl_range[1],
                                                  self.interp_steps, out.ctypes.data))
        self.knots = out

    def desc(self):
        d = _lib.SpectrumDesc()
        d.kind = _lib.SPECTRUM_CHERENKOV
        d.n_knots = self.interp_steps
        d.wl_min, d.wl_max = self.wl_range
        return d

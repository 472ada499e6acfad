"""Medium module of PhotonProp.jl (src/medium.jl), evaluated by the library.

WaterProperties stores the reference's unit-stripped values (permille, atm,
degC, ppm, ppm, g/cm^2).  The functions evaluate the library's FP64 host
implementation of the same formulas.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from . import _lib

BAR_PER_ATM = 1.01325


@dataclass
class WaterProperties:
    """WaterProperties, src/medium.jl:23-50."""

    salinity: float            # permille
    pressure: float            # atm
    temperature: float         # degC
    vol_conc_small_part: float  # ppm
    vol_conc_large_part: float  # ppm
    radiation_length: float = 36.08  # g/cm^2
    absorption_table: tuple | None = field(default=None)  # (wl, len); None = src/medium.jl:245-246

    @classmethod
    def from_units(cls, salinity_permille, pressure_bar, temperature_c, small_ppm, large_ppm,
                   radiation_length=36.08):
        """The reference's unitful constructor with pressure given in bar."""
        return cls(float(salinity_permille), float(pressure_bar) / BAR_PER_ATM, float(temperature_c),
                   float(small_ppm), float(large_ppm), float(radiation_length))

    def desc(self) -> _lib.MediumDesc:
        d = _lib.MediumDesc()
        d.salinity = self.salinity
        d.pressure = self.pressure
        d.temperature = self.temperature
        d.vol_conc_small_part = self.vol_conc_small_part
        d.vol_conc_large_part = self.vol_conc_large_part
        d.radiation_length = self.radiation_length
        if self.absorption_table is not None:
            wl, ln = (np.asarray(x, dtype=np.float64) for x in self.absorption_table)
            if len(wl) != len(ln) or not 2 <= len(wl) <= _lib.MAX_ABS or np.any(np.diff(wl) <= 0):
                raise ValueError("absorption table: 2..32 strictly increasing wavelengths")
            d.n_abs = len(wl)
            d.abs_wl[:len(wl)] = list(wl)
            d.abs_len[:len(ln)] = list(ln)
        return d


def make_cascadia_medium_properties(salinity=34.82, temperature=1.8) -> WaterProperties:
    """make_cascadia_medium_properties, src/medium.jl:52-58 (269.44088 bar)."""
    return WaterProperties.from_units(salinity, 269.44088, temperature, 0.0075, 0.0075, 36.08)


def make_seawater(salinity=35.0, temperature=2.0) -> WaterProperties:
    """The repo's seawater model at the given salinity/temperature, with the
    Cascadia pressure and particle concentrations."""
    return make_cascadia_medium_properties(salinity, temperature)


def _vec(fn, wl, medium):
    d = medium.desc()
    L = _lib.load()
    f = getattr(L, fn)
    w = np.asarray(wl, dtype=np.float64)
    out = np.array([f(d, float(x)) for x in w.ravel()]).reshape(w.shape)
    return out if out.ndim else float(out)


def get_refractive_index(wavelength, medium: WaterProperties):
    """Phase refractive index, src/medium.jl:125-158,179-183."""
    return _vec("pp_refractive_index", wavelength, medium)


def get_group_index(wavelength, medium: WaterProperties):
    """Group index n - lambda dn/dlambda of the same model."""
    return _vec("pp_group_index", wavelength, medium)


def get_scattering_length(wavelength, medium: WaterProperties):
    """Scattering length in m, src/medium.jl:201-235."""
    return _vec("pp_scattering_length", wavelength, medium)


def get_absorption_length(wavelength, medium: WaterProperties):
    """Absorption length in m, src/medium.jl:243-251."""
    return _vec("pp_absorption_length", wavelength, medium)

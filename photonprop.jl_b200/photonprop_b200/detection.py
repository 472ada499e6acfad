"""Detection module of PhotonProp.jl (src/detection.jl)."""
from __future__ import annotations

import os
from dataclasses import dataclass

import numpy as np

from . import _lib

DATA = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data")


@dataclass
class DetectionSphere:
    """DetectionSphere(position, radius), src/detection.jl:10-15."""

    position: tuple
    radius: float


class PMTWavelengthAcceptance:
    """PMTWavelengthAcceptance(xs, ys), src/detection.jl:18-28: linear
    interpolation of a tabulated acceptance, evaluated by the library."""

    def __init__(self, wavelengths, acceptance):
        xs = np.asarray(wavelengths, dtype=np.float64)
        ys = np.asarray(acceptance, dtype=np.float64)
        if len(xs) != len(ys) or not 2 <= len(xs) <= _lib.MAX_PMT or np.any(np.diff(xs) <= 0):
            raise ValueError("PMT table: 2..256 strictly increasing wavelengths")
        self.wavelengths, self.acceptance = xs, ys

    def desc(self) -> _lib.PmtDesc:
        d = _lib.PmtDesc()
        d.n = len(self.wavelengths)
        d.wavelength[:d.n] = list(self.wavelengths)
        d.acceptance[:d.n] = list(self.acceptance)
        return d

    def __call__(self, wavelength):
        d = self.desc()
        L = _lib.load()
        w = np.asarray(wavelength, dtype=np.float64)
        out = np.array([L.pp_pmt_acceptance(d, float(x)) for x in w.ravel()]).reshape(w.shape)
        return out if out.ndim else float(out)


def _load_table(name):
    d = np.loadtxt(os.path.join(DATA, name), delimiter=",", comments="#")
    return PMTWavelengthAcceptance(d[:, 0], d[:, 1])


# p_one_pmt_acc, src/detection.jl:31-33 (PMTAcc.csv)
p_one_pmt_acc = _load_table("pmt_acceptance.csv")
# the same curve tabulated at 5 nm over 300-700 nm
p_one_pmt_acc_5nm = _load_table("pmt_acceptance_5nm.csv")

"""Emission module of PhotonProp.jl (src/emission.jl)."""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from . import _lib
from .spectrum import Spectrum


@dataclass(frozen=True)
class AngularEmissionProfile:
    """AngularEmissionProfile{U,T}, src/emission.jl:13: a tag for the angular
    emission model: "IsotropicEmission", "CherenkovEmission" (a track emitting
    on the Cherenkov cone) or "CherenkovAngularEmission" (a point emitting
    with the EM-cascade profile cherenkov_ang_dist about its direction)."""

    kind: str = "IsotropicEmission"

    @property
    def emitter(self) -> int:
        if self.kind == "IsotropicEmission":
            return _lib.EMITTER_ISOTROPIC
        if self.kind == "CherenkovEmission":
            return _lib.EMITTER_CHERENKOV_CONE
        if self.kind == "CherenkovAngularEmission":
            return _lib.EMITTER_CASCADE
        raise ValueError(f"Cannot initialize {self.kind}")


IsotropicEmission = AngularEmissionProfile("IsotropicEmission")
CherenkovEmission = AngularEmissionProfile("CherenkovEmission")
CherenkovAngularEmission = AngularEmissionProfile("CherenkovAngularEmission")


@dataclass
class PhotonSource:
    """PhotonSource, src/emission.jl:102-109.  For a Cherenkov emitter the
    photons start on a track of `track_length` m from `position` along
    `direction`."""

    position: tuple
    direction: tuple
    time: float
    photons: int
    spectrum: Spectrum
    emission_profile: AngularEmissionProfile = IsotropicEmission
    track_length: float = 1.0


# Cherenkov angular profile of EM cascades, src/emission.jl:20-44 (e- parameters)
ANG_DIST_PARS = (4.27033, -6.02527, 0.29887, -0.00103)


def cherenkov_ang_dist(costheta, ref_index, pars=ANG_DIST_PARS):
    """cherenkov_ang_dist, src/emission.jl:32-44 (arXiv:1210.5140); the
    library's FP64 host function for the e- parameters, the same formula for
    other parameters."""
    if tuple(pars) == ANG_DIST_PARS:
        L = _lib.load()
        out = np.vectorize(lambda c, n: L.pp_cherenkov_ang_dist(float(c), float(n)), otypes=[np.float64])(
            costheta, ref_index)
        return float(out) if np.ndim(out) == 0 else out
    a, b, c, d = pars
    ctc = 1.0 / np.asarray(ref_index, dtype=np.float64)
    return a * np.exp(b * np.abs(np.asarray(costheta, dtype=np.float64) - ctc) ** c) + d

"""LightYield module of PhotonProp.jl (src/lightyield.jl): electromagnetic
cascades as Cherenkov light sources.

The shower profile, track length and Frank-Tamm normalisation are the
library's FP64 host functions; particle_to_elongated_lightsource and
particles_to_sources run on the device (one thread per particle interval)
and write pp_pair records that cross_pairs combines with target spheres for
the batched propagation kernel, so a batch can be driven by physical events.

Length units: mode "reference" reproduces the reference's arithmetic (grid
values are centimetres in the shower profile and are used unchanged as
metres for positions and times; the reference's water-density expression
with the temperature in degC).  Mode "metres" takes the grid in metres and
the DIPPR105 density at the temperature in kelvin.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass
from enum import IntEnum

import numpy as np

from . import _lib
from .emission import CherenkovEmission, IsotropicEmission, PhotonSource
from .medium import WaterProperties
from .spectrum import Spectrum


class ParticleType(IntEnum):
    """ParticleType, src/lightyield.jl:24-28."""
    EMinus = 11
    EPlus = -11
    Gamma = 22


@dataclass(frozen=True)
class LongitudinalParameters:
    alpha: float
    beta: float
    b: float


@dataclass(frozen=True)
class CherenkovTrackLengthParameters:
    alpha: float  # cm
    beta: float
    alpha_dev: float  # cm
    beta_dev: float


# src/lightyield.jl:35-37, 46-69 (the library holds the same values)
LongitudinalParametersEMinus = LongitudinalParameters(2.01849, 1.45469, 0.63207)
LongitudinalParametersEPlus = LongitudinalParameters(2.00035, 1.45501, 0.63008)
LongitudinalParametersGamma = LongitudinalParameters(2.83923, 1.34031, 0.64526)
CherenkovTrackLengthParametersEMinus = CherenkovTrackLengthParameters(532.07078881, 1.00000211, 5.78170887, 0.5)
CherenkovTrackLengthParametersEPlus = CherenkovTrackLengthParameters(532.11320598, 0.99999254, 5.73419669, 0.5)
CherenkovTrackLengthParametersGamma = CherenkovTrackLengthParameters(532.08540905, 0.99999877, 5.78170887,
                                                                     5.66586567)

_MODES = {"reference": _lib.LY_REFERENCE, "metres": _lib.LY_METRES}


def _mode(mode):
    try:
        return _MODES[mode]
    except KeyError:
        raise ValueError(f"unknown length mode {mode!r} (reference or metres)") from None


@dataclass
class Particle:
    """Particle, src/lightyield.jl:201-207 (m, unit vector, ns, GeV)."""
    position: tuple
    direction: tuple
    time: float
    energy: float
    type: ParticleType


def particles_array(particles) -> np.ndarray:
    out = np.zeros(len(particles), dtype=_lib.PARTICLE_DTYPE)
    for i, p in enumerate(particles):
        out[i]["pos"] = p.position
        out[i]["dir"] = p.direction
        out[i]["time"] = p.time
        out[i]["energy"] = p.energy
        out[i]["type"] = int(p.type)
    return out


def medium_density(medium: WaterProperties, mode="reference") -> float:
    return _lib.load().pp_medium_density(medium.desc(), _mode(mode))


def longitudinal_profile(energy, z, medium: WaterProperties, ptype, mode="reference"):
    """longitudinal_profile(energy, z, medium, ptype), src/lightyield.jl:116-140
    (energy in GeV, z in cm)."""
    L = _lib.load()
    d = medium.desc()
    m = _mode(mode)
    f = np.vectorize(lambda e, zz: L.pp_longitudinal_profile(d, m, int(ptype), float(e), float(zz)),
                     otypes=[np.float64])
    out = f(energy, z)
    return float(out) if np.ndim(out) == 0 else out


def cherenkov_track_length(energy, ptype):
    """cherenkov_track_length(energy, ptype), src/lightyield.jl:194-198 (cm)."""
    L = _lib.load()
    out = np.vectorize(lambda e: L.pp_cherenkov_track_length(int(ptype), float(e)), otypes=[np.float64])(energy)
    return float(out) if np.ndim(out) == 0 else out


def cherenkov_track_length_dev(energy, ptype):
    L = _lib.load()
    out = np.vectorize(lambda e: L.pp_cherenkov_track_length_dev(int(ptype), float(e)), otypes=[np.float64])(energy)
    return float(out) if np.ndim(out) == 0 else out


def frank_tamm_norm(wl_range, medium: WaterProperties) -> float:
    """frank_tamm_norm(wl_range, wl -> n(wl, medium)), src/spectrum.jl:41-45 (per cm)."""
    return _lib.load().pp_frank_tamm_norm(medium.desc(), float(wl_range[0]), float(wl_range[1]))


def fractional_contrib_long(energy, z_grid, medium: WaterProperties, ptype, mode="reference"):
    """fractional_contrib_long(energy, z_grid, medium, ptype), src/lightyield.jl:143-181 (z in cm)."""
    z = np.ascontiguousarray(z_grid, dtype=np.float64)
    out = np.zeros_like(z)
    _lib.check(_lib.load().pp_fractional_contrib_long(medium.desc(), _mode(mode), int(ptype), float(energy),
                                                      z.ctypes.data, len(z), out.ctypes.data))
    return out


def particle_to_lightsource(particle: Particle, medium: WaterProperties, wl_range, spectrum: Spectrum | None = None):
    """particle_to_lightsource, src/lightyield.jl:209-227: one source with
    frank_tamm_norm(wl_range) x cherenkov_track_length(E) photons.  (The
    reference reads a refractive-index field the medium does not have; the
    medium's n(wl) is used.)"""
    n = frank_tamm_norm(wl_range, medium) * cherenkov_track_length(particle.energy, particle.type)
    return PhotonSource(tuple(particle.position), tuple(particle.direction), float(particle.time), int(round(n)),
                        spectrum, CherenkovEmission, 0.0)


def particles_to_sources(propagator, particles, len_range, precision, wl_range=(300.0, 800.0), *, mode="reference",
                         emitter="isotropic"):
    """particle_to_elongated_lightsource for every particle at once on the
    device: (sources [n_particles * (n_grid - 1)] pp_pair records, n_grid)."""
    import torch
    parts = particles if isinstance(particles, np.ndarray) else particles_array(particles)
    parts = np.ascontiguousarray(parts, dtype=_lib.PARTICLE_DTYPE)
    em = {"isotropic": _lib.EMITTER_ISOTROPIC, "cone": _lib.EMITTER_CHERENKOV_CONE,
          "cascade": _lib.EMITTER_CASCADE}[emitter]
    dev = torch.device("cuda", propagator.device)
    n_grid_est = int(np.floor((len_range[1] - len_range[0]) / precision * (1 + 1e-12) + 1e-9)) + 1
    cap = max(1, len(parts) * max(n_grid_est - 1, 0))
    d_parts = torch.from_numpy(parts.view(np.uint8).copy()).to(dev)
    d_src = torch.zeros(cap * _lib.PAIR_DTYPE.itemsize, dtype=torch.uint8, device=dev)
    ng = ctypes.c_int64(0)
    stream = torch.cuda.current_stream(dev)
    _lib.check(_lib.load().pp_particles_to_sources_device(
        propagator.handle, d_parts.data_ptr(), len(parts), float(len_range[0]), float(len_range[1]),
        float(precision), _mode(mode), float(wl_range[0]), float(wl_range[1]), em, d_src.data_ptr(), cap,
        ctypes.byref(ng), stream.cuda_stream), propagator.handle)
    n_src = len(parts) * (ng.value - 1)
    out = d_src[: n_src * _lib.PAIR_DTYPE.itemsize].cpu().numpy().view(_lib.PAIR_DTYPE)
    return out, int(ng.value)


def particle_to_elongated_lightsource(particle: Particle, len_range, precision, medium: WaterProperties,
                                      spectrum: Spectrum, wl_range, *, propagator=None, mode="reference"):
    """particle_to_elongated_lightsource(particle, len_range, precision,
    medium, spectrum, wl_range), src/lightyield.jl:264-285: the PhotonSource
    of every grid interval (computed on the device of `propagator`, whose
    medium is used)."""
    from .propagation import Propagator
    prop = propagator or Propagator(medium, spectrum)
    src, _ = particles_to_sources(prop, [particle], len_range, precision, wl_range, mode=mode)
    return [PhotonSource(tuple(float(x) for x in s["pos"]), tuple(float(x) for x in s["dir"]), float(s["t0"]),
                         int(s["n_photons"]), spectrum, IsotropicEmission, 0.0) for s in src]


def cross_pairs(propagator, sources, targets, seed=0) -> np.ndarray:
    """Every source with every target sphere ((x, y, z, r) rows) on the
    device: pairs[s * n_targets + t] with seed pp_pair_seed(seed, index)."""
    import torch
    src = np.ascontiguousarray(sources, dtype=_lib.PAIR_DTYPE)
    tg = np.ascontiguousarray(np.asarray(targets, dtype=np.float32).reshape(-1, 4))
    dev = torch.device("cuda", propagator.device)
    d_src = torch.from_numpy(src.view(np.uint8).copy()).to(dev)
    d_tg = torch.from_numpy(tg.copy()).to(dev)
    n = len(src) * len(tg)
    d_out = torch.zeros(max(n, 1) * _lib.PAIR_DTYPE.itemsize, dtype=torch.uint8, device=dev)
    _lib.check(_lib.load().pp_cross_pairs_device(propagator.handle, d_src.data_ptr(), len(src), d_tg.data_ptr(),
                                                 len(tg), seed & (2**64 - 1), d_out.data_ptr(),
                                                 torch.cuda.current_stream(dev).cuda_stream), propagator.handle)
    return d_out[: n * _lib.PAIR_DTYPE.itemsize].cpu().numpy().view(_lib.PAIR_DTYPE)

"""Synthetic source-target workloads (pp_pair arrays).

point_source_pair      one isotropic point source and one sphere
cone_grid_pairs        a 1 m Cherenkov-cone track along +z and spheres on a grid of
                       distances x polar angles relative to the track
mixed_batch            many pairs with log-uniform photon counts, 50/50 isotropic /
                       cone emitters with random directions, sphere centres at a
                       uniform distance in a random direction; per-pair seeds from
                       pp_pair_seed(global seed, index)
"""
from __future__ import annotations

import numpy as np

from . import _lib
from .propagation import pair_seed


def point_source_pair(n_photons=100_000, target=(10.0, 0.0, 0.0), radius=0.21, seed=0):
    p = np.zeros(1, dtype=_lib.PAIR_DTYPE)
    p["dir"] = (0.0, 0.0, 1.0)
    p["target"] = target
    p["radius"] = radius
    p["n_photons"] = int(n_photons)
    p["seed"] = seed
    p["emitter"] = _lib.EMITTER_ISOTROPIC
    return p


def cone_grid_pairs(n_photons=100_000_000, distances=(5.0, 10.0, 20.0, 50.0, 100.0),
                    polar_deg=(0.0, 45.0, 90.0, 135.0, 180.0), track_len=1.0, radius=0.21, seed=0):
    """Track from the origin along +z; sphere centres at distance d from the
    track midpoint at polar angle theta from the track axis (x-z plane)."""
    out = np.zeros(len(distances) * len(polar_deg), dtype=_lib.PAIR_DTYPE)
    i = 0
    for d in distances:
        for th in polar_deg:
            t = np.radians(th)
            out[i]["dir"] = (0.0, 0.0, 1.0)
            out[i]["track_len"] = track_len
            out[i]["target"] = (d * np.sin(t), 0.0, 0.5 * track_len + d * np.cos(t))
            out[i]["radius"] = radius
            out[i]["n_photons"] = int(n_photons)
            out[i]["seed"] = pair_seed(seed, i)
            out[i]["emitter"] = _lib.EMITTER_CHERENKOV_CONE
            i += 1
    return out


def _unit_vectors(rng, n):
    z = rng.uniform(-1.0, 1.0, n)
    phi = rng.uniform(0.0, 2 * np.pi, n)
    s = np.sqrt(1.0 - z * z)
    return np.stack([s * np.cos(phi), s * np.sin(phi), z], axis=1)


def mixed_batch(n_pairs=4096, seed=0, n_min=1e4, n_max=1e7, d_min=2.0, d_max=150.0, radius=0.21,
                track_len=1.0, cone_fraction=0.5, distance_law="uniform"):
    rng = np.random.Generator(np.random.PCG64(seed))
    out = np.zeros(n_pairs, dtype=_lib.PAIR_DTYPE)
    n = np.exp(rng.uniform(np.log(n_min), np.log(n_max), n_pairs))
    out["n_photons"] = np.round(n).astype(np.int64)
    cone = rng.uniform(size=n_pairs) < cone_fraction
    out["emitter"] = np.where(cone, _lib.EMITTER_CHERENKOV_CONE, _lib.EMITTER_ISOTROPIC)
    out["dir"] = _unit_vectors(rng, n_pairs)
    out["track_len"] = np.where(cone, track_len, 0.0)
    if distance_law == "loguniform":
        dist = np.exp(rng.uniform(np.log(d_min), np.log(d_max), n_pairs))
    else:
        dist = rng.uniform(d_min, d_max, n_pairs)
    out["target"] = _unit_vectors(rng, n_pairs) * dist[:, None]
    out["radius"] = radius
    out["seed"] = [pair_seed(seed, i) for i in range(n_pairs)]
    return out


def total_photons(pairs) -> int:
    return int(np.asarray(pairs["n_photons"], dtype=np.int64).sum())

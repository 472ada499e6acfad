"""Synthetic source-target batches for the CPU side, without the product.

TEST INFRASTRUCTURE ONLY: ``bench.py``'s reference arm and CPU-baseline leg
build their batch here so that the process timing the oracle never loads the
product library.  ``mixed_batch`` draws exactly the numbers that
``photonprop_b200.batches.mixed_batch`` draws (same PCG64 calls in the same
order, positions rounded to FP32 as the product's 80-byte pair record stores
them) and ``pair_seed`` is splitmix64 (Steele, Lea, Flood, OOPSLA 2014) of
seed + golden-ratio * (index + 1), the product's per-pair seed; a CPU test
checks both against the product field by field.

The workload is the 4096-pair mixed-batch benchmark: photon
counts log-uniform in [1e4, 1e7], 50/50 isotropic point / 1 m Cherenkov-cone
emitters with directions uniform on the sphere, sphere centres at a uniform
distance in [2, 150] m in a random direction, radius 0.21 m.  The reference
(PhotonProp.jl) has no batched entry point; its propagation of one
source-target pair is ``propagate_distance`` (src/photon_prop_cuda.jl:588-644).
"""
from __future__ import annotations

import os

import numpy as np

from .oracle import PAIR_DTYPE

EMITTER_ISOTROPIC, EMITTER_CHERENKOV_CONE = 0, 1

_PMT_CSV = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "photonprop.jl_b200",
                        "photonprop_b200", "data", "pmt_acceptance.csv")

_M64 = np.uint64(0xFFFFFFFFFFFFFFFF)


def pair_seed(global_seed: int, index) -> np.ndarray:
    """splitmix64 of global_seed + 0x9E3779B97F4A7C15 * (index + 1), modulo 2^64."""
    idx = np.asarray(index, dtype=np.uint64)
    with np.errstate(over="ignore"):
        z = np.uint64(global_seed & 0xFFFFFFFFFFFFFFFF) + np.uint64(0x9E3779B97F4A7C15) * (idx + np.uint64(1))
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        return z ^ (z >> np.uint64(31))


def _unit_vectors(rng, n):
    z = rng.uniform(-1.0, 1.0, n)
    phi = rng.uniform(0.0, 2 * np.pi, n)
    s = np.sqrt(1.0 - z * z)
    return np.stack([s * np.cos(phi), s * np.sin(phi), z], axis=1)


def _f32(x):
    return np.asarray(x, dtype=np.float64).astype(np.float32).astype(np.float64)


def mixed_batch(n_pairs=4096, seed=0, n_min=1e4, n_max=1e7, d_min=2.0, d_max=150.0, radius=0.21,
                track_len=1.0, cone_fraction=0.5):
    """The mixed benchmark batch as oracle pairs (FP64 fields holding the
    FP32 values the product's pair records carry)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    out = np.zeros(n_pairs, dtype=PAIR_DTYPE)
    n = np.exp(rng.uniform(np.log(n_min), np.log(n_max), n_pairs))
    out["n_photons"] = np.round(n).astype(np.int64)
    cone = rng.uniform(size=n_pairs) < cone_fraction
    out["emitter"] = np.where(cone, EMITTER_CHERENKOV_CONE, EMITTER_ISOTROPIC)
    out["dir"] = _f32(_unit_vectors(rng, n_pairs))
    out["track_len"] = _f32(np.where(cone, track_len, 0.0))
    dist = rng.uniform(d_min, d_max, n_pairs)
    out["target"] = _f32(_unit_vectors(rng, n_pairs) * dist[:, None])
    out["radius"] = _f32(radius)
    out["seed"] = pair_seed(seed, np.arange(n_pairs, dtype=np.uint64))
    return out


def pmt_table():
    """PMTAcc.csv of the reference (src/detection.jl:31-33) as the package
    data file stores it: (wavelengths nm, acceptance)."""
    d = np.loadtxt(_PMT_CSV, delimiter=",", comments="#")
    return d[:, 0].copy(), d[:, 1].copy()


def sampled(pairs, fraction):
    """The first ceil(fraction * N_i) photons of every pair (at least one of a
    non-empty pair): a sample whose photon mix follows the batch's."""
    out = pairs.copy()
    n = np.asarray(pairs["n_photons"], dtype=np.int64)
    out["n_photons"] = np.where(n > 0, np.maximum(1, np.ceil(n * float(fraction))).astype(np.int64), 0)
    out["n_photons"] = np.minimum(out["n_photons"], n)
    return out

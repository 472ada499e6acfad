"""Modelling module of PhotonProp.jl (src/modelling.jl:33-190): Cherenkov
reweighting of isotropic photons, Gamma fits of their arrival-time
residuals, the fit table and its Parquet I/O.

The per-hit work runs on the device (pp_propagate_fit, pp_fit_photon_dist_device):
every hit is reweighted for every observation angle, the weighted moments are
accumulated in FP64 and a Gamma distribution is fitted per (distance, angle)
by maximum likelihood, without the hits leaving the GPU.  make_photon_fits
propagates all distances in one batched launch.  The scalar helpers
(cherenkov_ang_dist, get_dir_reweight) are the library's FP64 host functions.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass
from typing import Callable

import numpy as np

from . import _lib
from .batches import point_source_pair
from .detection import p_one_pmt_acc
from .medium import make_cascadia_medium_properties
from .propagation import Propagator, RunOptions, pair_seed
from .spectrum import CherenkovSpectrum

STD_ANG_DIST_PARS = (4.27033, -6.02527, 0.29887, -0.00103)  # a, b, c, d for e- (src/emission.jl:19)


def cherenkov_ang_dist(costheta, ref_index):
    """cherenkov_ang_dist, src/emission.jl:32-44 (FP64, elementwise)."""
    L = _lib.load()
    f = np.vectorize(lambda c, n: L.pp_cherenkov_ang_dist(float(c), float(n)), otypes=[np.float64])
    out = f(costheta, ref_index)
    return float(out) if np.ndim(out) == 0 else out


def cherenkov_ang_dist_int(ref_index, lower=None, upper=None):
    """cherenkov_ang_dist_int, src/emission.jl:88-99: the interpolated [-1, 1]
    integral; with lower/upper, the closed form _cherenkov_ang_dist_int over
    [lower, upper] (src/emission.jl:52-86)."""
    L = _lib.load()
    if lower is None and upper is None:
        f = np.vectorize(lambda n: L.pp_cherenkov_ang_dist_int(float(n)), otypes=[np.float64])
        out = f(ref_index)
    else:
        lo = -1.0 if lower is None else lower
        hi = 1.0 if upper is None else upper
        f = np.vectorize(lambda n: L.pp_cherenkov_ang_dist_int_exact(float(n), lo, hi), otypes=[np.float64])
        out = f(ref_index)
    if np.ndim(out) == 0:
        v = float(out)
        if np.isnan(v) and lower is None and upper is None:
            raise ValueError(f"ref_index {ref_index} outside the tabulated range 1.1-1.5")
        return v
    return out


def get_dir_reweight(thetas, obs_angle, ref_ixs):
    """get_dir_reweight(thetas, obs_angle, ref_ixs), src/modelling.jl:46-49."""
    t = np.ascontiguousarray(thetas, dtype=np.float64)
    n = np.ascontiguousarray(np.broadcast_to(np.asarray(ref_ixs, dtype=np.float64), t.shape))
    out = np.empty_like(t)
    _lib.check(_lib.load().pp_dir_reweight(t.ctypes.data, float(obs_angle), n.ctypes.data, out.ctypes.data, t.size))
    return out


class SobolSeq:
    """One-dimensional Sobol sequence scaled to [lb, ub]: the first dimension
    of Sobol.jl 1.5.0's SobolSeq (not vendored), whose direction numbers are
    all 1, so point k (k = 1, 2, ...; the initial 0 is skipped) is the
    bit-reversed Gray code of k, 0.5, 0.75, 0.25, 0.375, 0.875, ..."""

    def __init__(self, lb, ub):
        self.lb, self.ub, self.n = float(lb), float(ub), 0

    def next(self) -> float:
        self.n += 1
        g = self.n ^ (self.n >> 1)
        r = int(f"{g:032b}"[::-1], 2)
        return self.lb + (self.ub - self.lb) * r / 2.0 ** 32


_default_prop = None


def _default_propagator():
    global _default_prop
    if _default_prop is None:
        m = make_cascadia_medium_properties()
        _default_prop = Propagator(m, CherenkovSpectrum((300.0, 800.0), 20, m), p_one_pmt_acc)
    return _default_prop


def fit_photon_dist(obs_angles, obs_photon_df, n_ph_gen, *, propagator: Propagator | None = None):
    """fit_photon_dist(obs_angles, obs_photon_df, n_ph_gen), src/modelling.jl:52-79,
    on the device: the DataFrame's columns tres, initial_theta, ref_ix,
    abs_weight and wavelength are reweighted for each observation angle
    (times the PMT acceptance of the propagator's table) and fitted.
    Returns a DataFrame (obs_angle, fit_alpha, fit_theta, det_fraction)."""
    import pandas as pd
    import torch
    prop = propagator or _default_propagator()
    angles = np.ascontiguousarray(np.ravel(obs_angles), dtype=np.float64)
    n = len(obs_photon_df)
    dev = torch.device("cuda", prop.device)
    cols = [torch.from_numpy(np.array(obs_photon_df[k].to_numpy(), dtype=np.float64, copy=True)).to(dev)
            if n else torch.zeros(1, dtype=torch.float64, device=dev)
            for k in ("tres", "initial_theta", "ref_ix", "abs_weight", "wavelength")]
    d_m = torch.zeros((len(angles), _lib.FIT_MOMENTS), dtype=torch.float64, device=dev)
    d_f = torch.zeros((len(angles), _lib.FIT_OUT), dtype=torch.float64, device=dev)
    L = _lib.load()
    stream = torch.cuda.current_stream(dev).cuda_stream
    st = L.pp_fit_photon_dist_device(prop.handle, n, *[c.data_ptr() for c in cols], angles.ctypes.data,
                                     len(angles), int(n_ph_gen), d_m.data_ptr(), d_f.data_ptr(), stream)
    _lib.check(st, prop.handle)
    f = d_f.cpu().numpy()
    return pd.DataFrame({"obs_angle": angles, "fit_alpha": f[:, 0], "fit_theta": f[:, 1], "det_fraction": f[:, 2]})


@dataclass
class FitResult:
    fits: np.ndarray      # [n_pairs, n_angles, 3]: fit_alpha, fit_theta, det_fraction
    moments: np.ndarray   # [n_pairs, n_angles, 4]
    stats: np.ndarray     # [n_pairs, 8]
    n_hits: int


def propagate_fit(propagator: Propagator, pairs, obs_angles, opts: RunOptions | None = None,
                  hit_capacity: int | None = None) -> FitResult:
    """Propagates a batch and fits every (pair, observation angle) on the
    device (pp_propagate_fit).  hit_capacity sizes the device hit buffer
    (96 bytes per hit with the fit records); the library runs the pairs in
    waves that fit it, planned from a pilot launch of the first photons of
    every pair.  The default is the batch's photon count (every photon hits
    at most once), between 2^16 and 2^27 (at most 12.9 GB of device memory)."""
    opts = opts or RunOptions(mode="compat", pmt_weight=True)
    o = opts.to_c()
    o.hist_bins = 0
    pairs = np.ascontiguousarray(pairs)
    angles = np.ascontiguousarray(np.ravel(obs_angles), dtype=np.float64)
    n_p, n_a = len(pairs), len(angles)
    if hit_capacity is None:
        hit_capacity = int(min(max(int(pairs["n_photons"].sum()), 1 << 16), 1 << 27))
    fits = np.zeros((n_p, n_a, _lib.FIT_OUT))
    mom = np.zeros((n_p, n_a, _lib.FIT_MOMENTS))
    stats = np.zeros((n_p, 8))
    n_hits = ctypes.c_int64(0)
    L = _lib.load()
    while True:
        st = L.pp_propagate_fit(propagator.handle, pairs.ctypes.data, n_p, ctypes.byref(o), angles.ctypes.data, n_a,
                                hit_capacity, ctypes.byref(n_hits), fits.ctypes.data, mom.ctypes.data,
                                stats.ctypes.data, None)
        if st == _lib.PP_ERR_OVERFLOW:  # one pair alone has more hits than the buffer
            hit_capacity = int(n_hits.value * 1.1) + 1
            continue
        _lib.check(st, propagator.handle)
        return FitResult(fits, mom, stats, int(n_hits.value))


def fit_pairs(n_photons_per_dist: int, n_distances: int, n_angles: int, max_dist: float = 300.0, seed: int = 0):
    """The sample points of make_photon_fits (src/modelling.jl:88-95):
    (pairs, distances, obs_angles).  Distances are 10^Sobol([0, log10 max_dist])
    rounded to Float32 like propagate_distance's argument; one isotropic
    source at the origin and a 0.21 m sphere at (0, 0, distance) per distance."""
    s = SobolSeq(0.0, np.pi)
    s2 = SobolSeq(0.0, float(np.float32(np.log10(np.float32(max_dist)))))
    distances = np.array([np.float32(10.0 ** s2.next()) for _ in range(n_distances)], dtype=np.float32)
    obs_angles = np.array([s.next() for _ in range(n_angles)])
    pairs = np.concatenate([point_source_pair(n_photons_per_dist, target=(0.0, 0.0, float(d)), radius=0.21,
                                              seed=pair_seed(seed, i)) for i, d in enumerate(distances)])
    return pairs, distances, obs_angles


def make_photon_fits(n_photons_per_dist: int, n_distances: int, n_angles: int, max_dist: float = 300.0, *,
                     propagator: Propagator | None = None, mode: str = "compat", seed: int = 0,
                     g: float | None = None):
    """make_photon_fits(n_photons_per_dist, n_distances, n_angles, max_dist),
    src/modelling.jl:86-111: distances 10^Sobol([0, log10 max_dist]) and
    observation angles Sobol([0, pi]) (fit_pairs); all distances propagate in
    one batched launch and every (distance, angle) is fitted on the device.
    Returns the DataFrame (obs_angle, fit_alpha, fit_theta, det_fraction,
    distance), distances outer, angles inner, as the reference's
    vcat(..., source=:distance)."""
    import pandas as pd
    prop = propagator or _default_propagator()
    pairs, distances, obs_angles = fit_pairs(n_photons_per_dist, n_distances, n_angles, max_dist, seed)
    res = propagate_fit(prop, pairs, obs_angles, RunOptions(mode=mode, g=g, pmt_weight=True, hist_bins=0))
    f = res.fits.reshape(-1, _lib.FIT_OUT)
    return pd.DataFrame({"obs_angle": np.tile(obs_angles, n_distances), "fit_alpha": f[:, 0], "fit_theta": f[:, 1],
                         "det_fraction": f[:, 2],
                         "distance": np.repeat(distances.astype(np.float64), n_angles)})


# ---- fit table I/O (src/modelling.jl:119-172) ------------------------------
FIT_TABLE_COLUMNS = ("obs_angle", "fit_alpha", "fit_theta", "det_fraction", "distance")


def write_fit_table(df, path):
    """write_parquet(path, results_df) of the reference's workflow
    (example_full.jl:136-137): the five FP64 columns of make_photon_fits."""
    import pyarrow as pa
    import pyarrow.parquet as pq
    table = pa.table({k: np.asarray(df[k], dtype=np.float64) for k in FIT_TABLE_COLUMNS})
    pq.write_table(table, path)


def read_parquet(path):
    import pyarrow.parquet as pq
    return pq.read_table(path).to_pandas()


@dataclass
class FeatureTransformation:
    """FeatureTransformation, src/modelling.jl:128-131."""
    forward: Callable
    backward: Callable


def apply_transformation(x, t: FeatureTransformation):
    return t.forward(x)


def reverse_transformation(x, t: FeatureTransformation):
    return t.backward(x)


def default_trafos():
    """The feature/target transformations of get_data, src/modelling.jl:176-183."""
    return {
        ("det_fraction", "log_det_fraction"): FeatureTransformation(lambda x: -np.log10(x), lambda x: 10.0 ** (-x)),
        ("det_fraction", "log_det_fraction_scaled"): FeatureTransformation(lambda x: (-np.log10(x) - 3) / 10,
                                                                           lambda x: 10.0 ** (-(x * 10 + 3))),
        ("obs_angle", "cos_obs_angle"): FeatureTransformation(np.cos, np.arccos),
        ("fit_alpha", "log_fit_alpha"): FeatureTransformation(np.log10, lambda x: 10.0 ** x),
        ("fit_theta", "log_fit_theta"): FeatureTransformation(np.log10, lambda x: 10.0 ** x),
        ("distance", "log_distance"): FeatureTransformation(np.log10, lambda x: 10.0 ** x),
    }


def splitdf(df, pct, rng=None):
    """splitdf(df, pct), src/modelling.jl:119-125: a random pct / (1 - pct) row split."""
    assert 0 <= pct <= 1
    rng = rng or np.random.default_rng()
    ids = np.arange(1, len(df) + 1)
    rng.shuffle(ids)
    sel = ids <= len(df) * pct
    return df[sel], df[~sel]


def read_from_parquet(filename, trafos=None, rng=None):
    """read_from_parquet(filename, trafos), src/modelling.jl:145-172: Float32
    columns, transformed features and targets, an 80/20 split; returns
    (features_train, targets_train, features_test, targets_test) as
    [n_features, n] arrays like the reference's transposed matrices."""
    df = read_parquet(filename).astype(np.float32)
    for (src, dst), t in (trafos or default_trafos()).items():
        df[dst] = np.asarray(apply_transformation(df[src].to_numpy(), t), dtype=np.float32)
    feature_names = ["log_distance", "cos_obs_angle"]
    target_names = ["log_fit_alpha", "log_fit_theta", "log_det_fraction_scaled"]
    train, test = splitdf(df, 0.8, rng)
    return (train[feature_names].to_numpy(np.float32).T, train[target_names].to_numpy(np.float32).T,
            test[feature_names].to_numpy(np.float32).T, test[target_names].to_numpy(np.float32).T)

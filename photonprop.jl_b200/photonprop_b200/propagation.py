"""PhotonPropagationCuda module of PhotonProp.jl (src/photon_prop_cuda.jl) on
the B200 library.

Propagator owns one library context (device-resident medium, spectrum and
PMT tables) and exposes the batched, plain, device-buffer and
reference-layout entry points.  propagate_distance, cuda_propagate_photons_,
initialize_photon_arrays and process_output mirror the reference functions of
the same names.
"""
from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass

import numpy as np

from . import _lib
from .detection import DetectionSphere, PMTWavelengthAcceptance, p_one_pmt_acc
from .emission import IsotropicEmission, PhotonSource
from .medium import WaterProperties, get_absorption_length, get_refractive_index
from .spectrum import CherenkovSpectrum, Spectrum

C_VACUUM_M_PER_NS = 0.299792458  # CODATA2018, src/photon_prop_cuda.jl:635


@dataclass
class RunOptions:
    """pp_run_opts.  mode "compat" reproduces the reference kernel's arithmetic
    (theta drawn in radians, 10 fixed steps, no move when the line meets the
    sphere beyond the step, phase-velocity time, absorption-only weight);
    "physical" is the physical model (isotropic cos(theta), Cherenkov cone,
    group-velocity time, photons end at t_max, absorption x PMT weight)."""

    mode: str = "physical"
    g: float | None = None
    max_steps: int | None = None
    t_max: float = 500.0
    hist_t0: float = 0.0
    hist_bin_width: float = 1.0
    hist_bins: int | None = None
    pmt_weight: bool | None = None
    normalize: bool = False
    write_hits: bool = True
    cascade: bool = False  # the device entry points' pairs may include cascade emitters
    block_size: int = 0
    blocks_per_sm: int = 0
    chunk_photons: int = 0

    def to_c(self) -> _lib.RunOpts:
        m = {"compat": _lib.MODE_COMPAT, "physical": _lib.MODE_PHYSICAL}.get(self.mode)
        if m is None:
            raise ValueError(f"unknown mode {self.mode!r}")
        o = _lib.RunOpts()
        _lib.check(_lib.load().pp_default_opts(m, ctypes.byref(o)))
        if self.g is not None:
            o.g = self.g
        if self.max_steps is not None:
            o.max_steps = self.max_steps
        if m == _lib.MODE_PHYSICAL:
            o.t_max = self.t_max
        o.hist_t0 = self.hist_t0
        o.hist_bin_width = self.hist_bin_width
        if self.hist_bins is not None:
            o.hist_bins = self.hist_bins
        flags = o.flags
        if self.pmt_weight is not None:
            flags = (flags | _lib.OPT_PMT_WEIGHT) if self.pmt_weight else (flags & ~_lib.OPT_PMT_WEIGHT)
        if self.normalize:
            flags |= _lib.OPT_NORMALIZE
        if not self.write_hits:
            flags |= _lib.OPT_NO_HITS
        if self.cascade:
            flags |= _lib.OPT_CASCADE
        o.flags = flags
        o.block_size, o.blocks_per_sm, o.chunk_photons = self.block_size, self.blocks_per_sm, self.chunk_photons
        return o


@dataclass
class PropagationResult:
    hits: np.ndarray   # HIT_DTYPE records (at most the capacity)
    n_hits: int        # true number of hits
    stats: np.ndarray  # [n_pairs, 8]: hits, sum w, sum w^2, sum w t, sum w t^2, sum w ln t, photons, 0
    hist: np.ndarray   # [n_pairs, bins] FP64 arrival-time histogram
    overflow: bool = False

    def sorted_hits(self):
        h = self.hits
        return h[np.lexsort((h["photon"], h["pair"]))]


def pair_seed(global_seed: int, index: int) -> int:
    return int(_lib.load().pp_pair_seed(global_seed & (2**64 - 1), index))


def make_pair(source: PhotonSource, target: DetectionSphere, seed: int = 0) -> np.ndarray:
    """One pp_pair record from a PhotonSource and a DetectionSphere."""
    p = np.zeros(1, dtype=_lib.PAIR_DTYPE)
    p["pos"] = source.position
    p["t0"] = source.time
    d = np.asarray(source.direction, dtype=np.float64)
    nrm = np.linalg.norm(d)
    p["dir"] = d / nrm if nrm > 0 else (0.0, 0.0, 1.0)
    p["track_len"] = source.track_length
    p["target"] = target.position
    p["radius"] = target.radius
    p["n_photons"] = int(source.photons)
    p["seed"] = seed & (2**64 - 1)
    p["emitter"] = source.emission_profile.emitter
    return p


class Propagator:
    """One library context on `device` with the medium, spectrum and PMT
    tables resident on the device."""

    def __init__(self, medium: WaterProperties, spectrum: Spectrum,
                 pmt: PMTWavelengthAcceptance | None = p_one_pmt_acc, device: int = 0):
        L = _lib.load()
        self.medium, self.spectrum, self.pmt, self.device = medium, spectrum, pmt, device
        h = ctypes.c_void_p()
        st = L.pp_create(ctypes.byref(h), device, medium.desc(), spectrum.desc(),
                         pmt.desc() if pmt is not None else None)
        if st != _lib.PP_OK:
            raise _lib.PPError(st, L.pp_last_error(None).decode())
        self._h = h
        self._L = L

    def close(self):
        if getattr(self, "_h", None):
            self._L.pp_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @property
    def handle(self):
        return self._h

    def knots(self) -> np.ndarray:
        out = np.zeros(_lib.MAX_KNOTS, dtype=np.float32)
        n = ctypes.c_int32()
        _lib.check(self._L.pp_get_knots(self._h, out.ctypes.data, _lib.MAX_KNOTS, ctypes.byref(n)), self._h)
        return out[:n.value].copy()

    def _run(self, fn, pairs, opts: RunOptions, hit_capacity):
        pairs = np.ascontiguousarray(pairs, dtype=_lib.PAIR_DTYPE)
        o = opts.to_c()
        n = len(pairs)
        bins = o.hist_bins
        hits = np.zeros(max(hit_capacity, 1), dtype=_lib.HIT_DTYPE)
        stats = np.zeros((max(n, 1), _lib.N_STATS))
        hist = np.zeros((max(n, 1), max(bins, 1)))
        nh = ctypes.c_int64()
        st = fn(self._h, pairs.ctypes.data if n else None, n, ctypes.byref(o), hits.ctypes.data,
                hit_capacity, ctypes.byref(nh), stats.ctypes.data, hist.ctypes.data if bins > 0 else None)
        overflow = st == _lib.PP_ERR_OVERFLOW
        if not overflow:
            _lib.check(st, self._h)
        k = 0 if (o.flags & _lib.OPT_NO_HITS) else min(nh.value, hit_capacity)
        return PropagationResult(hits[:k].copy(), nh.value, stats[:n], hist[:n, :bins], overflow)

    def propagate_into(self, pairs, opts: RunOptions, hits, stats, hist, plain: bool = False) -> tuple:
        """pp_propagate (or pp_propagate_plain) into caller-owned host arrays
        (e.g. pinned).  Returns (n_hits, overflow)."""
        o = opts.to_c()
        n = len(pairs)
        nh = ctypes.c_int64()
        fn = self._L.pp_propagate_plain if plain else self._L.pp_propagate
        st = fn(self._h, _lib.ptr(pairs) if n else None, n, ctypes.byref(o), _lib.ptr(hits), len(hits),
                ctypes.byref(nh), _lib.ptr(stats), _lib.ptr(hist) if o.hist_bins > 0 else None)
        if st != _lib.PP_ERR_OVERFLOW:
            _lib.check(st, self._h)
        return nh.value, st == _lib.PP_ERR_OVERFLOW

    def propagate(self, pairs, opts: RunOptions | None = None, hit_capacity: int = 1 << 20):
        """Batched persistent kernel over all pairs (pp_propagate)."""
        return self._run(self._L.pp_propagate, pairs, opts or RunOptions(), hit_capacity)

    def propagate_plain(self, pairs, opts: RunOptions | None = None, hit_capacity: int = 1 << 20):
        """One launch per pair with host synchronisation (pp_propagate_plain)."""
        return self._run(self._L.pp_propagate_plain, pairs, opts or RunOptions(), hit_capacity)

    def propagate_device(self, d_pairs, n_pairs, opts: RunOptions, d_hits, hit_capacity, d_counters,
                         d_stats, d_hist, stream=None):
        """pp_propagate_device on torch CUDA tensors; asynchronous on `stream`
        (a torch.cuda.Stream or a raw handle)."""
        o = opts.to_c()
        s = getattr(stream, "cuda_stream", stream)
        _lib.check(self._L.pp_propagate_device(
            self._h, _lib.ptr(d_pairs), n_pairs, ctypes.byref(o), _lib.ptr(d_hits), hit_capacity,
            _lib.ptr(d_counters), _lib.ptr(d_stats), _lib.ptr(d_hist) if o.hist_bins > 0 else None,
            s), self._h)

    def propagate_device_noalloc(self, d_pairs, n_pairs, opts: RunOptions, d_hits, hit_capacity, d_counters,
                                 d_stats, d_hist, stream=None):
        """pp_propagate_device_noalloc: like propagate_device, for callers whose
        device memory is all owned by their own pool; the library allocates
        nothing (its work-queue scratch is a fixed static device array, at most
        NOALLOC_MAX_PAIRS pairs per call).  Make the first call on a device
        before any stream capture, and do not overlap calls on the GPU."""
        o = opts.to_c()
        s = getattr(stream, "cuda_stream", stream)
        _lib.check(self._L.pp_propagate_device_noalloc(
            self._h, _lib.ptr(d_pairs), n_pairs, ctypes.byref(o), _lib.ptr(d_hits), hit_capacity,
            _lib.ptr(d_counters), _lib.ptr(d_stats), _lib.ptr(d_hist) if o.hist_bins > 0 else None,
            s), self._h)

    def propagate_plain_device(self, d_pair, h_pair, pair_index, opts: RunOptions, d_hits, hit_capacity,
                               d_counters, d_stats, d_hist, stream=None):
        o = opts.to_c()
        s = getattr(stream, "cuda_stream", stream)
        hp = np.ascontiguousarray(h_pair, dtype=_lib.PAIR_DTYPE)
        _lib.check(self._L.pp_propagate_plain_device(
            self._h, _lib.ptr(d_pair), hp.ctypes.data, pair_index, ctypes.byref(o), _lib.ptr(d_hits),
            hit_capacity, _lib.ptr(d_counters), _lib.ptr(d_stats),
            _lib.ptr(d_hist) if o.hist_bins > 0 else None, s), self._h)

    def autotune(self, pairs, opts: RunOptions, cache_path: str | None = None):
        pairs = np.ascontiguousarray(pairs, dtype=_lib.PAIR_DTYPE)
        o = opts.to_c()
        best = _lib.RunOpts()
        rate = ctypes.c_double()
        _lib.check(self._L.pp_autotune(self._h, pairs.ctypes.data, len(pairs), ctypes.byref(o),
                                       cache_path.encode() if cache_path else None, ctypes.byref(best),
                                       ctypes.byref(rate)), self._h)
        return {"block_size": best.block_size, "blocks_per_sm": best.blocks_per_sm,
                "chunk_photons": best.chunk_photons, "photons_per_s": rate.value}

    def device_eval(self, op: int, inputs) -> np.ndarray:
        out_w = {0: 4, 3: 3, 4: 3, 12: 5}.get(op, 1)
        x = np.ascontiguousarray(inputs, dtype=np.float64)
        n = x.shape[0] if x.ndim > 0 else 1
        out = np.zeros((n, out_w))
        _lib.check(self._L.pp_device_eval(self._h, op, x.ctypes.data, out.ctypes.data, n), self._h)
        return out

    def cuda_propagate_photons(self, out_positions, out_directions, out_wavelengths, out_dist_travelled,
                               out_stack_pointers, out_n_ph_simulated, stack_len, pair, opts: RunOptions,
                               threads: int, stream=None):
        o = opts.to_c()
        s = getattr(stream, "cuda_stream", stream)
        pr = np.ascontiguousarray(pair, dtype=_lib.PAIR_DTYPE)
        _lib.check(self._L.pp_cuda_propagate_photons(
            self._h, _lib.ptr(out_positions), _lib.ptr(out_directions), _lib.ptr(out_wavelengths),
            _lib.ptr(out_dist_travelled), _lib.ptr(out_stack_pointers), _lib.ptr(out_n_ph_simulated),
            int(stack_len), int(out_stack_pointers.shape[0]), int(threads), pr.ctypes.data, ctypes.byref(o),
            s), self._h)


# ---------------------------------------------------------------------------
# Reference-shaped functions

def initialize_photon_arrays(stack_length: int, blocks: int, dtype=None, device="cuda"):
    """initialize_photon_arrays, src/photon_prop_cuda.jl:414-422: zeroed
    device arrays (positions, directions, wavelengths, dist_travelled,
    per-block stack pointers, photons simulated)."""
    import torch
    dt = dtype or torch.float32
    n = int(stack_length) * int(blocks)
    return (torch.zeros((n, 3), dtype=dt, device=device), torch.zeros((n, 3), dtype=dt, device=device),
            torch.zeros(n, dtype=dt, device=device), torch.zeros(n, dtype=dt, device=device),
            torch.zeros(int(blocks), dtype=torch.int32, device=device),
            torch.zeros(1, dtype=torch.int64, device=device))


def process_output(output, stack_pointers):
    """process_output, src/photon_prop_cuda.jl:390-411: concatenates the used
    part of every block's stack (1-based stack pointers, 0 = empty)."""
    output = np.asarray(output)
    sp = np.asarray(stack_pointers, dtype=np.int64)
    stack_len = output.shape[0] // sp.shape[0]
    parts = []
    for i, p in enumerate(sp):
        if p == 0:
            continue
        start = i * stack_len  # 0-based start of block i
        parts.append(output[start:int(p)])
    if not parts:
        return output[:0]
    return np.concatenate(parts, axis=0)


def cuda_propagate_photons_(out_positions, out_directions, out_wavelengths, out_dist_travelled,
                            out_stack_pointers, out_n_ph_simulated, stack_len, seed, source: PhotonSource,
                            target_pos, target_r, medium: WaterProperties, *, threads=1024, mode="compat",
                            g=0.99, propagator: Propagator | None = None):
    """cuda_propagate_photons!, src/photon_prop_cuda.jl:262-386, with the same
    arguments (device arrays from initialize_photon_arrays; the grid has one
    block per stack pointer and `threads` threads per block)."""
    prop = propagator or Propagator(medium, source.spectrum)
    pair = make_pair(source, DetectionSphere(tuple(target_pos), float(target_r)), seed)
    prop.cuda_propagate_photons(out_positions, out_directions, out_wavelengths, out_dist_travelled,
                                out_stack_pointers, out_n_ph_simulated, stack_len, pair,
                                RunOptions(mode=mode, g=g, hist_bins=0), threads)


def propagate_distance(distance: float, medium: WaterProperties, n_ph_gen: int, *, seed: int = 0,
                       mode: str = "compat", g: float | None = None, propagator: Propagator | None = None,
                       target_radius: float = 0.21, hit_capacity: int | None = None):
    """propagate_distance, src/photon_prop_cuda.jl:588-644: an isotropic
    source at the origin (Cherenkov spectrum 300-800 nm, 20 knots) and a
    0.21 m sphere at (0, 0, distance); returns the DataFrame
    (tres, initial_theta, ref_ix, abs_weight, dist_travelled, wavelength),
    empty if nothing was detected.  The host finish (absorption weight, times,
    residuals, theta) is FP64 as in the reference."""
    import pandas as pd
    distance = float(distance)
    spectrum = CherenkovSpectrum((300.0, 800.0), 20, medium)
    prop = propagator or Propagator(medium, spectrum)
    source = PhotonSource((0.0, 0.0, 0.0), (0.0, 0.0, 1.0), 0.0, int(n_ph_gen), spectrum, IsotropicEmission)
    target = DetectionSphere((0.0, 0.0, distance), target_radius)
    pair = make_pair(source, target, seed)
    opts = RunOptions(mode=mode, g=g, hist_bins=0, pmt_weight=False)
    cap = hit_capacity or max(1024, int(n_ph_gen * 0.05) + 1024)
    res = prop.propagate(pair, opts, hit_capacity=cap)
    if res.overflow:
        raise _lib.PPError(_lib.PP_ERR_OVERFLOW, "hit capacity too small")
    h = res.sorted_hits()
    if len(h) == 0:
        return pd.DataFrame()
    n_ph_sim = int(res.stats[0, 6])
    distt = h["dist"].astype(np.float32)
    wls = h["wavelength"].astype(np.float32)
    dirs = h["dir0"].astype(np.float32)
    abs_weight = np.exp(-distt.astype(np.float64) / get_absorption_length(wls, medium))
    if n_ph_sim > n_ph_gen:  # downsampling of src/photon_prop_cuda.jl:624-631
        k = int(math.ceil(len(abs_weight) * n_ph_gen / n_ph_sim))
        distt, wls, dirs, abs_weight = distt[:k], wls[:k], dirs[:k], abs_weight[:k]
    ref_ix = get_refractive_index(wls, medium)
    c_n = C_VACUUM_M_PER_NS / ref_ix
    photon_times = distt / c_n
    tgeo = (distance - target_radius) / (C_VACUUM_M_PER_NS / get_refractive_index(800.0, medium))
    tres = photon_times - tgeo
    thetas = np.arccos(np.clip(dirs[:, 2].astype(np.float64), -1.0, 1.0))
    return pd.DataFrame({"tres": tres, "initial_theta": thetas, "ref_ix": ref_ix, "abs_weight": abs_weight,
                         "dist_travelled": distt, "wavelength": wls})

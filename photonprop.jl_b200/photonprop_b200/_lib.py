"""ctypes binding of libphotonprop_b200.so (include/photonprop_b200.h).

The library is the product: every propagation goes through its CUDA kernels.
If it is missing, loading raises; there is no CPU fallback.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from . import _build

LIB_PATH = _build.LIB_PATH

PP_OK, PP_ERR_ARG, PP_ERR_OOM, PP_ERR_OVERFLOW, PP_ERR_TIMEOUT, PP_ERR_CUDA, PP_ERR_STATE, PP_ERR_BUSY = range(8)
STATUS_NAMES = {0: "PP_OK", 1: "PP_ERR_ARG", 2: "PP_ERR_OOM", 3: "PP_ERR_OVERFLOW", 4: "PP_ERR_TIMEOUT",
                5: "PP_ERR_CUDA", 6: "PP_ERR_STATE", 7: "PP_ERR_BUSY"}
MODE_COMPAT, MODE_PHYSICAL = 0, 1
EMITTER_ISOTROPIC, EMITTER_CHERENKOV_CONE, EMITTER_CASCADE = 0, 1, 2
SPECTRUM_CHERENKOV, SPECTRUM_MONOCHROMATIC = 0, 1
OPT_PMT_WEIGHT, OPT_NORMALIZE, OPT_NO_HITS, OPT_COMPACT_HITS, OPT_CASCADE = 1, 2, 4, 8, 16
MAX_KNOTS, MAX_ABS, MAX_PMT, N_STATS = 64, 32, 256, 8
NOALLOC_MAX_PAIRS = 65536

PAIR_DTYPE = np.dtype([
    ("pos", "<f4", 3), ("t0", "<f4"), ("dir", "<f4", 3), ("track_len", "<f4"),
    ("target", "<f4", 3), ("radius", "<f4"), ("n_photons", "<i8"), ("seed", "<u8"),
    ("emitter", "<i4"), ("reserved", "<i4", 3)])
assert PAIR_DTYPE.itemsize == 80

HIT_DTYPE = np.dtype([
    ("pos", "<f4", 3), ("time", "<f4"), ("dir0", "<f4", 3), ("weight", "<f4"),
    ("dir", "<f4", 3), ("wavelength", "<f4"), ("dist", "<f4"), ("pair", "<u4"),
    ("photon", "<u8")])
assert HIT_DTYPE.itemsize == 64

HIT32_DTYPE = np.dtype([
    ("pos", "<f4", 3), ("time", "<f4"), ("weight", "<f4"), ("wavelength", "<f4"), ("photon_lo", "<u4"),
    ("pair", "<u4")])
assert HIT32_DTYPE.itemsize == 32


class MediumDesc(ctypes.Structure):
    _fields_ = [("salinity", ctypes.c_double), ("pressure", ctypes.c_double),
                ("temperature", ctypes.c_double), ("vol_conc_small_part", ctypes.c_double),
                ("vol_conc_large_part", ctypes.c_double), ("radiation_length", ctypes.c_double),
                ("n_abs", ctypes.c_int32), ("pad", ctypes.c_int32),
                ("abs_wl", ctypes.c_double * MAX_ABS), ("abs_len", ctypes.c_double * MAX_ABS)]


class SpectrumDesc(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int32), ("n_knots", ctypes.c_int32),
                ("wl_min", ctypes.c_double), ("wl_max", ctypes.c_double)]


class PmtDesc(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int32), ("pad", ctypes.c_int32),
                ("wavelength", ctypes.c_double * MAX_PMT), ("acceptance", ctypes.c_double * MAX_PMT)]


class RunOpts(ctypes.Structure):
    _fields_ = [("mode", ctypes.c_int32), ("max_steps", ctypes.c_int32), ("g", ctypes.c_float),
                ("t_max", ctypes.c_float), ("hist_t0", ctypes.c_float),
                ("hist_bin_width", ctypes.c_float), ("hist_bins", ctypes.c_int32),
                ("flags", ctypes.c_uint32), ("block_size", ctypes.c_int32),
                ("blocks_per_sm", ctypes.c_int32), ("chunk_photons", ctypes.c_int32),
                ("reserved", ctypes.c_int32)]


class ServerConfig(ctypes.Structure):
    _fields_ = [("max_inflight", ctypes.c_int32), ("max_pairs_per_batch", ctypes.c_int32),
                ("hbm_budget_bytes", ctypes.c_int64), ("bytes_per_hit", ctypes.c_int32),
                ("hit_safety", ctypes.c_float), ("max_queued", ctypes.c_int32), ("reserved", ctypes.c_int32),
                ("opts", RunOpts)]


class ServerCounters(ctypes.Structure):
    _fields_ = [("submitted", ctypes.c_int64), ("completed", ctypes.c_int64), ("batches", ctypes.c_int64),
                ("pairs", ctypes.c_int64), ("in_flight_batches", ctypes.c_int64), ("waiting", ctypes.c_int64),
                ("reserved_bytes", ctypes.c_int64), ("photons", ctypes.c_double)]


class PPError(RuntimeError):
    """A non-OK pp_status; .status holds the code."""

    def __init__(self, status, msg):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


_lib = None

# (name, restype, argtypes) for every declaration of include/photonprop_b200.h
_VP, _D, _I64, _I32 = ctypes.c_void_p, ctypes.c_double, ctypes.c_int64, ctypes.c_int32
_SIGS = [
    ("pp_abi_version", ctypes.c_int, []),
    ("pp_version", ctypes.c_char_p, []),
    ("pp_launch_count", ctypes.c_uint64, []),
    ("pp_pair_seed", ctypes.c_uint64, [ctypes.c_uint64, ctypes.c_uint64]),
    ("pp_refractive_index", _D, [ctypes.POINTER(MediumDesc), _D]),
    ("pp_group_index", _D, [ctypes.POINTER(MediumDesc), _D]),
    ("pp_scattering_length", _D, [ctypes.POINTER(MediumDesc), _D]),
    ("pp_absorption_length", _D, [ctypes.POINTER(MediumDesc), _D]),
    ("pp_pmt_acceptance", _D, [ctypes.POINTER(PmtDesc), _D]),
    ("pp_cherenkov_knots", ctypes.c_int, [ctypes.POINTER(MediumDesc), _D, _D, _I32, _VP]),
    ("pp_default_opts", ctypes.c_int, [_I32, ctypes.POINTER(RunOpts)]),
    ("pp_create", ctypes.c_int, [ctypes.POINTER(_VP), ctypes.c_int, ctypes.POINTER(MediumDesc),
                                 ctypes.POINTER(SpectrumDesc), ctypes.POINTER(PmtDesc)]),
    ("pp_destroy", None, [_VP]),
    ("pp_last_error", ctypes.c_char_p, [_VP]),
    ("pp_device", ctypes.c_int, [_VP]),
    ("pp_get_knots", ctypes.c_int, [_VP, _VP, _I32, ctypes.POINTER(_I32)]),
    ("pp_propagate", ctypes.c_int, [_VP, _VP, _I64, ctypes.POINTER(RunOpts), _VP, _I64,
                                    ctypes.POINTER(_I64), _VP, _VP]),
    ("pp_propagate_plain", ctypes.c_int, [_VP, _VP, _I64, ctypes.POINTER(RunOpts), _VP, _I64,
                                          ctypes.POINTER(_I64), _VP, _VP]),
    ("pp_propagate_device", ctypes.c_int, [_VP, _VP, _I64, ctypes.POINTER(RunOpts), _VP, _I64,
                                           _VP, _VP, _VP, _VP]),
    ("pp_propagate_device_noalloc", ctypes.c_int, [_VP, _VP, _I64, ctypes.POINTER(RunOpts), _VP, _I64,
                                                   _VP, _VP, _VP, _VP]),
    ("pp_propagate_plain_device", ctypes.c_int, [_VP, _VP, _VP, _I64, ctypes.POINTER(RunOpts), _VP,
                                                 _I64, _VP, _VP, _VP, _VP]),
    ("pp_cuda_propagate_photons", ctypes.c_int, [_VP, _VP, _VP, _VP, _VP, _VP, _VP, _I32, _I32, _I32,
                                                 _VP, ctypes.POINTER(RunOpts), _VP]),
    ("pp_cherenkov_ang_dist", _D, [_D, _D]),
    ("pp_cherenkov_ang_dist_int_exact", _D, [_D, _D, _D]),
    ("pp_cherenkov_ang_dist_int", _D, [_D]),
    ("pp_dir_reweight", ctypes.c_int, [_VP, _D, _VP, _VP, _I64]),
    ("pp_cascade_cos_theta", _D, [_D, _D]),
    ("pp_propagate_fit", ctypes.c_int, [_VP, _VP, _I64, ctypes.POINTER(RunOpts), _VP, _I32, _I64,
                                        ctypes.POINTER(_I64), _VP, _VP, _VP, _VP]),
    ("pp_fit_hits_device", ctypes.c_int, [_VP, _VP, _I64, _I32, _VP, _I64, _VP, _VP, _I32, _VP, _VP, _VP]),
    ("pp_fit_photon_dist_device", ctypes.c_int, [_VP, _I64, _VP, _VP, _VP, _VP, _VP, _VP, _I32, _I64, _VP, _VP,
                                                 _VP]),
    ("pp_medium_density", _D, [ctypes.POINTER(MediumDesc), _I32]),
    ("pp_longitudinal_profile", _D, [ctypes.POINTER(MediumDesc), _I32, _I32, _D, _D]),
    ("pp_cherenkov_track_length", _D, [_I32, _D]),
    ("pp_cherenkov_track_length_dev", _D, [_I32, _D]),
    ("pp_frank_tamm_norm", _D, [ctypes.POINTER(MediumDesc), _D, _D]),
    ("pp_fractional_contrib_long", ctypes.c_int, [ctypes.POINTER(MediumDesc), _I32, _I32, _D, _VP, _I64, _VP]),
    ("pp_particles_to_sources_device", ctypes.c_int, [_VP, _VP, _I64, _D, _D, _D, _I32, _D, _D, _I32, _VP, _I64,
                                                      ctypes.POINTER(_I64), _VP]),
    ("pp_cross_pairs_device", ctypes.c_int, [_VP, _VP, _I64, _VP, _I64, ctypes.c_uint64, _VP, _VP]),
    ("pp_event_llh_device", ctypes.c_int, [_VP, _I32, _I64, _I64, _I64, _VP, _VP, _VP, _VP, _VP, _VP]),
    ("pp_server_create", ctypes.c_int, [_VP, ctypes.POINTER(ServerConfig), ctypes.POINTER(_VP)]),
    ("pp_server_destroy", None, [_VP]),
    ("pp_server_submit", ctypes.c_int, [_VP, _VP, _I32, ctypes.POINTER(ctypes.c_uint64)]),
    ("pp_server_wait", ctypes.c_int, [_VP, ctypes.c_uint64, _D]),
    ("pp_server_result", ctypes.c_int, [_VP, ctypes.c_uint64, _VP, _I64, ctypes.POINTER(_I64), _VP, _VP,
                                        ctypes.POINTER(_D)]),
    ("pp_server_get_counters", ctypes.c_int, [_VP, ctypes.POINTER(ServerCounters)]),
    ("pp_mlp_create", ctypes.c_int, [ctypes.c_int, ctypes.c_uint64, ctypes.POINTER(_VP)]),
    ("pp_mlp_destroy", None, [_VP]),
    ("pp_mlp_last_error", ctypes.c_char_p, [_VP]),
    ("pp_mlp_num_params", ctypes.c_int32, []),
    ("pp_mlp_get_params", ctypes.c_int, [_VP, _VP]),
    ("pp_mlp_set_params", ctypes.c_int, [_VP, _VP]),
    ("pp_mlp_set_normalization", ctypes.c_int, [_VP, _VP, _VP, _VP, _VP]),
    ("pp_mlp_get_normalization", ctypes.c_int, [_VP, _VP]),
    ("pp_mlp_forward", ctypes.c_int, [_VP, _VP, _VP, _I64, _I32, _VP]),
    ("pp_mlp_train_step", ctypes.c_int, [_VP, _VP, _VP, _VP, _I64, ctypes.c_float, ctypes.POINTER(ctypes.c_float),
                                         _VP]),
    ("pp_mlp_gemm_selftest", ctypes.c_int, [ctypes.c_int, _VP, _VP, _VP]),
    ("pp_gamma_mixture_fit", ctypes.c_int, [_VP, _I64, _I32, ctypes.c_float, ctypes.c_float, _VP, _VP, _I32, _VP]),
    ("pp_autotune", ctypes.c_int, [_VP, _VP, _I64, ctypes.POINTER(RunOpts), ctypes.c_char_p,
                                   ctypes.POINTER(RunOpts), ctypes.POINTER(_D)]),
    ("pp_device_eval", ctypes.c_int, [_VP, _I32, _VP, _VP, _I64]),
    ("pp_measure_peaks", ctypes.c_int, [ctypes.c_int, ctypes.POINTER(_D), ctypes.POINTER(_D),
                                        ctypes.POINTER(_D)]),
    ("pp_measure_step_rate", ctypes.c_int, [ctypes.c_int, ctypes.POINTER(_D)]),
]

EXPORTED = [s[0] for s in _SIGS]

PARTICLE_DTYPE = np.dtype([("pos", "<f4", 3), ("time", "<f4"), ("dir", "<f4", 3), ("energy", "<f4"),
                           ("type", "<i4"), ("reserved", "<i4", 3)])
assert PARTICLE_DTYPE.itemsize == 48
LY_REFERENCE, LY_METRES = 0, 1
LLH_PARAMS = 6
LLH_REFERENCE, LLH_SHIFTED = 0, 1

FIT_MOMENTS = 4
FIT_OUT = 3
MAX_FIT_ANGLES = 4096


def load():
    """Loads the library (building it first if sources are newer)."""
    global _lib
    if _lib is None:
        if _build.needs_build():
            _build.build()
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"libphotonprop_b200.so is missing at {LIB_PATH}; build it with "
                               "__graft_entry__.build()")
        L = ctypes.CDLL(LIB_PATH)
        for name, res, args in _SIGS:
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        if L.pp_abi_version() != 1:
            raise RuntimeError("ABI version mismatch")
        _lib = L
    return _lib


def check(status, ctx=None):
    if status != PP_OK:
        L = load()
        msg = L.pp_last_error(ctx)
        raise PPError(status, msg.decode() if msg else "")


def ptr(a):
    """Data pointer of a numpy array or torch tensor (or None)."""
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        return a.ctypes.data
    return a.data_ptr()

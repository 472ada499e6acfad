"""ctypes front end of the FP64 CPU oracle (oracle/pp_oracle.c).

TEST INFRASTRUCTURE ONLY: used by ``tests/``, ``__graft_entry__.smoke()`` and
the CPU-baseline leg of ``bench.py`` as the checker.  The product never
imports it.  Build recipe: ``oracle/Makefile`` (gcc + OpenMP).
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

from . import tables as tb

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle_pp.so")

MAX_KNOTS, MAX_ABS, MAX_PMT = 64, 32, 256
N_STATS = 8
MODE_COMPAT, MODE_PHYSICAL = 0, 1
OPT_PMT_WEIGHT, OPT_NORMALIZE = 1, 2

PAIR_DTYPE = np.dtype([
    ("pos", "<f8", 3), ("t0", "<f8"), ("dir", "<f8", 3), ("track_len", "<f8"),
    ("target", "<f8", 3), ("radius", "<f8"), ("n_photons", "<i8"), ("seed", "<u8"),
    ("emitter", "<i4"), ("pad", "<i4")])

HIT_DTYPE = np.dtype([
    ("pos", "<f8", 3), ("time", "<f8"), ("dir0", "<f8", 3), ("weight", "<f8"),
    ("dir", "<f8", 3), ("wavelength", "<f8"), ("dist", "<f8"), ("pair", "<i8"),
    ("photon", "<i8"), ("step", "<i4"), ("pad", "<i4")])


class Tables(ctypes.Structure):
    _fields_ = [
        ("a01", ctypes.c_double), ("a2", ctypes.c_double), ("a3", ctypes.c_double),
        ("a4", ctypes.c_double), ("c_small", ctypes.c_double), ("c_large", ctypes.c_double),
        ("n_knots", ctypes.c_int32), ("n_abs", ctypes.c_int32), ("n_pmt", ctypes.c_int32),
        ("pad", ctypes.c_int32),
        ("knots", ctypes.c_double * MAX_KNOTS),
        ("abs_wl", ctypes.c_double * MAX_ABS), ("abs_len", ctypes.c_double * MAX_ABS),
        ("pmt_wl", ctypes.c_double * MAX_PMT), ("pmt_acc", ctypes.c_double * MAX_PMT),
        ("casc_fwd", ctypes.c_void_p), ("casc_inv", ctypes.c_void_p),
        ("casc_vmin", ctypes.c_double), ("casc_dv", ctypes.c_double), ("casc_gmin", ctypes.c_double),
        ("casc_dg", ctypes.c_double), ("casc_nf", ctypes.c_int32), ("casc_ni", ctypes.c_int32)]


class Opts(ctypes.Structure):
    _fields_ = [
        ("mode", ctypes.c_int32), ("max_steps", ctypes.c_int32), ("g", ctypes.c_double),
        ("t_max", ctypes.c_double), ("hist_t0", ctypes.c_double),
        ("hist_bin_width", ctypes.c_double), ("hist_bins", ctypes.c_int32),
        ("flags", ctypes.c_uint32)]


_lib = None
last_threads_used = 0  # OpenMP team size of the last propagate() call


def build(force=False):
    if force or not os.path.exists(LIB_PATH) or (
            os.path.getmtime(LIB_PATH) < max(os.path.getmtime(os.path.join(HERE, f))
                                             for f in ("pp_oracle.c", "pp_oracle.h"))):
        subprocess.run(["make", "-s", "-C", HERE, "ORACLE_CC=gcc"], check=True)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(LIB_PATH)
        dp = ctypes.POINTER(ctypes.c_double)
        u32p = ctypes.POINTER(ctypes.c_uint32)
        L.orc_philox4x32_10.argtypes = [u32p, u32p, u32p]
        L.orc_philox2x32_10.argtypes = [u32p, ctypes.c_uint32, u32p]
        L.orc_step_uniforms.argtypes = [u32p, ctypes.POINTER(ctypes.c_double)]
        L.orc_scatter_turn.argtypes = [dp, dp, dp]
        L.orc_uniform.argtypes = [ctypes.c_uint32]
        L.orc_uniform.restype = ctypes.c_double
        L.orc_hg_costheta.argtypes = [ctypes.c_double, ctypes.c_double]
        L.orc_hg_costheta.restype = ctypes.c_double
        L.orc_rotate_to_axis.argtypes = [dp, dp, dp]
        L.orc_update_position.argtypes = [dp, dp, ctypes.c_double, dp]
        L.orc_interp_sorted.argtypes = [ctypes.c_double, dp, dp, ctypes.c_int]
        L.orc_interp_sorted.restype = ctypes.c_double
        L.orc_interp_equidistant.argtypes = [ctypes.c_double, dp, ctypes.c_int,
                                             ctypes.c_double, ctypes.c_double]
        L.orc_interp_equidistant.restype = ctypes.c_double
        for f in ("orc_refractive_index", "orc_group_index", "orc_scattering_length"):
            getattr(L, f).argtypes = [ctypes.POINTER(Tables), ctypes.c_double]
            getattr(L, f).restype = ctypes.c_double
        L.orc_propagate.argtypes = [
            ctypes.POINTER(Tables), ctypes.c_void_p, ctypes.c_int64, ctypes.POINTER(Opts),
            ctypes.c_int64, ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p,
            ctypes.c_int, ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_int)]
        L.orc_propagate.restype = ctypes.c_int64
        L.orc_simulate_one.argtypes = [ctypes.POINTER(Tables), ctypes.c_void_p, ctypes.c_int64,
                                       ctypes.c_int64, ctypes.POINTER(Opts), ctypes.c_void_p]
        L.orc_simulate_one.restype = ctypes.c_int
        _lib = L
    return _lib


def _dptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def philox4x32_10(ctr, key):
    c = (ctypes.c_uint32 * 4)(*ctr)
    k = (ctypes.c_uint32 * 2)(*key)
    o = (ctypes.c_uint32 * 4)()
    lib().orc_philox4x32_10(c, k, o)
    return list(o)


def philox2x32_10(ctr, key):
    c = (ctypes.c_uint32 * 2)(*ctr)
    o = (ctypes.c_uint32 * 2)()
    lib().orc_philox2x32_10(c, int(key) & 0xFFFFFFFF, o)
    return list(o)


def step_uniforms(w):
    """The three 21-bit uniforms of a step from its Philox2x32 block (w0, w1)."""
    c = (ctypes.c_uint32 * 2)(*w)
    u = (ctypes.c_double * 3)()
    lib().orc_step_uniforms(c, u)
    return list(u)


def scatter_turn(old, new):
    """Physical-mode scattering turn of direction `old` by the local vector `new`."""
    o = np.ascontiguousarray(old, dtype=np.float64)
    n = np.ascontiguousarray(new, dtype=np.float64)
    out = np.zeros(3)
    lib().orc_scatter_turn(_dptr(o), _dptr(n), _dptr(out))
    return out


def uniform(w):
    return lib().orc_uniform(int(w) & 0xFFFFFFFF)


def hg_costheta(g, u):
    return lib().orc_hg_costheta(float(g), float(u))


def rotate_to_axis(old, new):
    o = np.ascontiguousarray(old, dtype=np.float64)
    n = np.ascontiguousarray(new, dtype=np.float64)
    r = np.zeros(3)
    lib().orc_rotate_to_axis(_dptr(o), _dptr(n), _dptr(r))
    return r


def update_position(pos, d, step):
    p = np.ascontiguousarray(pos, dtype=np.float64)
    dd = np.ascontiguousarray(d, dtype=np.float64)
    r = np.zeros(3)
    lib().orc_update_position(_dptr(p), _dptr(dd), float(step), _dptr(r))
    return r


def interp_sorted(x, xs, ys):
    xs = np.ascontiguousarray(xs, dtype=np.float64)
    ys = np.ascontiguousarray(ys, dtype=np.float64)
    return lib().orc_interp_sorted(float(x), _dptr(xs), _dptr(ys), len(xs))


def interp_equidistant(x, knots, lo, hi):
    k = np.ascontiguousarray(knots, dtype=np.float64)
    return lib().orc_interp_equidistant(float(x), _dptr(k), len(k), float(lo), float(hi))


def make_tables(medium: tb.Water, knots, pmt=None, abs_table=None) -> Tables:
    t = Tables()
    a01, a2, a3, a4 = tb._fry_coeffs(medium)
    t.a01, t.a2, t.a3, t.a4 = a01, a2, a3, a4
    t.c_small, t.c_large = medium.vol_conc_small_part, medium.vol_conc_large_part
    knots = np.asarray(knots, dtype=np.float64)
    t.n_knots = len(knots)
    t.knots[:len(knots)] = list(knots)
    aw, al = abs_table if abs_table is not None else (tb.ABS_WL, tb.ABS_LEN)
    t.n_abs = len(aw)
    t.abs_wl[:len(aw)] = list(aw)
    t.abs_len[:len(al)] = list(al)
    if pmt is None:
        pmt = (np.array([100.0, 1000.0]), np.array([1.0, 1.0]))
    t.n_pmt = len(pmt[0])
    t.pmt_wl[:len(pmt[0])] = list(pmt[0])
    t.pmt_acc[:len(pmt[1])] = list(pmt[1])
    from . import fits
    fwd, inv, vmin, dv, gmin, dg = fits.cascade_tables()
    t._casc = (fwd, inv)  # keeps the arrays alive with the struct
    t.casc_fwd, t.casc_inv = fwd.ctypes.data, inv.ctypes.data
    t.casc_vmin, t.casc_dv, t.casc_gmin, t.casc_dg = vmin, dv, gmin, dg
    t.casc_nf, t.casc_ni = len(fwd) - 1, len(inv) - 1
    return t


def make_opts(mode=MODE_PHYSICAL, max_steps=None, g=0.95, t_max=500.0, hist_t0=0.0,
              hist_bin_width=1.0, hist_bins=500, flags=0) -> Opts:
    o = Opts()
    o.mode = mode
    o.max_steps = max_steps if max_steps is not None else (10 if mode == MODE_COMPAT else 1000)
    o.g, o.t_max, o.hist_t0, o.hist_bin_width = g, t_max, hist_t0, hist_bin_width
    o.hist_bins, o.flags = hist_bins, flags
    return o


def pairs_array(n):
    return np.zeros(n, dtype=PAIR_DTYPE)


def propagate(tables: Tables, pairs, opts: Opts, photon_limit=-1, n_threads=0,
              hit_cap=None):
    """Runs the oracle; returns (hits, stats, hist, steps, total_hits)."""
    pairs = np.ascontiguousarray(pairs, dtype=PAIR_DTYPE)
    n = len(pairs)
    if hit_cap is None:
        hit_cap = 1 << 20
    hits = np.zeros(hit_cap, dtype=HIT_DTYPE)
    stats = np.zeros((n, N_STATS))
    hist = np.zeros((n, max(opts.hist_bins, 1)))
    steps = ctypes.c_int64(0)
    used = ctypes.c_int(0)
    total = lib().orc_propagate(
        ctypes.byref(tables), pairs.ctypes.data, n, ctypes.byref(opts), int(photon_limit),
        hits.ctypes.data, hit_cap, stats.ctypes.data, hist.ctypes.data, int(n_threads),
        ctypes.byref(steps), ctypes.byref(used))
    global last_threads_used
    last_threads_used = used.value
    return hits[:min(total, hit_cap)], stats, hist[:, :opts.hist_bins], steps.value, total


def simulate_one(tables: Tables, pair, pair_idx, photon, opts: Opts):
    """Replays one photon; returns its hit record or None."""
    p = np.ascontiguousarray(np.asarray(pair, dtype=PAIR_DTYPE).reshape(1))
    h = np.zeros(1, dtype=HIT_DTYPE)
    ok = lib().orc_simulate_one(ctypes.byref(tables), p.ctypes.data, int(pair_idx), int(photon),
                                ctypes.byref(opts), h.ctypes.data)
    return h[0] if ok else None

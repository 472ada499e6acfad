"""Continuous-batching serving loop (pp_server_* of the C ABI) and the
request workloads used to measure it.

Server wraps one native scheduler: submit() queues a request (a list of
pairs) and returns at once; result() waits for it.  requests() draws the
serving workload (Poisson arrivals, 1-64 pairs per request drawn as the mixed
batch with photon counts log-uniform in [1e4, 1e6]); run_open_loop() replays
it against a Server and run_plain_loop() against the one-launch-per-request
loop (pp_propagate called per request, in arrival order, by one worker).
"""
from __future__ import annotations

import contextlib
import ctypes
import gc
import threading
import time
from dataclasses import dataclass

import numpy as np

from . import _lib
from .batches import mixed_batch
from .propagation import Propagator, RunOptions


@dataclass
class RequestResult:
    hits: np.ndarray   # HIT32_DTYPE, pair = index within the request
    stats: np.ndarray  # [n_pairs, 8]
    hist: np.ndarray   # [n_pairs, bins]
    latency_s: float
    overflow: bool


class Server:
    def __init__(self, propagator: Propagator, opts: RunOptions, max_inflight=2, max_pairs_per_batch=4096,
                 hbm_budget_bytes=40 << 30, hit_safety=4.0, max_queued=100000):
        self._L = _lib.load()
        self.prop = propagator
        self.opts = opts
        cfg = _lib.ServerConfig()
        cfg.max_inflight = max_inflight
        cfg.max_pairs_per_batch = max_pairs_per_batch
        cfg.hbm_budget_bytes = hbm_budget_bytes
        cfg.bytes_per_hit = 32
        cfg.hit_safety = hit_safety
        cfg.max_queued = max_queued
        cfg.opts = opts.to_c()
        h = ctypes.c_void_p()
        _lib.check(self._L.pp_server_create(propagator.handle, ctypes.byref(cfg), ctypes.byref(h)))
        self._h = h
        self.bins = cfg.opts.hist_bins
        self._npairs = {}
        self._hitbuf = None  # reused by result(): one allocation, not one per request
        self._hitbuf_lock = threading.Lock()  # result() may be called from several threads

    def close(self):
        if getattr(self, "_h", None):
            self._L.pp_server_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def submit(self, pairs) -> int:
        pairs = np.ascontiguousarray(pairs, dtype=_lib.PAIR_DTYPE)
        rid = ctypes.c_uint64()
        _lib.check(self._L.pp_server_submit(self._h, pairs.ctypes.data, len(pairs), ctypes.byref(rid)))
        self._npairs[rid.value] = (len(pairs), 0)
        return rid.value

    def wait(self, rid: int, timeout_s: float = 60.0):
        _lib.check(self._L.pp_server_wait(self._h, rid, timeout_s))

    def result(self, rid: int, timeout_s: float = 60.0, hit_capacity: int = 1 << 20) -> RequestResult:
        self.wait(rid, timeout_s)
        n, _ = self._npairs.pop(rid)
        stats = np.zeros((n, _lib.N_STATS))
        hist = np.zeros((n, max(self.bins, 1)))
        nh = ctypes.c_int64()
        lat = ctypes.c_double()
        with self._hitbuf_lock:
            if self._hitbuf is None or len(self._hitbuf) < hit_capacity:
                self._hitbuf = np.empty(hit_capacity, dtype=_lib.HIT32_DTYPE)
            hits = self._hitbuf
            st = self._L.pp_server_result(self._h, rid, hits.ctypes.data, hit_capacity, ctypes.byref(nh),
                                          stats.ctypes.data, hist.ctypes.data, ctypes.byref(lat))
            if st not in (_lib.PP_OK, _lib.PP_ERR_OVERFLOW):
                _lib.check(st)
            hits = hits[:min(nh.value, hit_capacity)].copy()
        return RequestResult(hits, stats, hist[:, :self.bins], lat.value, st == _lib.PP_ERR_OVERFLOW)

    def counters(self) -> dict:
        c = _lib.ServerCounters()
        _lib.check(self._L.pp_server_get_counters(self._h, ctypes.byref(c)))
        return {f: getattr(c, f) for f, _ in c._fields_}


def requests(rate_hz=200.0, duration_s=60.0, seed=0, min_pairs=1, max_pairs=64, n_min=1e4, n_max=1e6):
    """Poisson arrival times and per-request pair arrays of the serving workload."""
    rng = np.random.Generator(np.random.PCG64(seed))
    t, arrivals = 0.0, []
    while True:
        t += rng.exponential(1.0 / rate_hz)
        if t >= duration_s:
            break
        arrivals.append(t)
    sizes = rng.integers(min_pairs, max_pairs + 1, size=len(arrivals))
    pool = mixed_batch(int(sizes.sum()), seed=seed + 1, n_min=n_min, n_max=n_max)
    reqs, off = [], 0
    for n in sizes:
        reqs.append(pool[off:off + n].copy())
        off += n
    return np.array(arrivals), reqs


def _percentiles(lat):
    a = np.sort(np.asarray(lat))
    return {"p50_ms": float(np.percentile(a, 50) * 1e3), "p99_ms": float(np.percentile(a, 99) * 1e3),
            "p99.9_ms": float(np.percentile(a, 99.9) * 1e3), "max_ms": float(a[-1] * 1e3)}


@contextlib.contextmanager
def _gc_paused():
    """Python's cyclic garbage collector paused for a timed stream: a full
    collection walks every result kept so far and can hold the interpreter
    lock for tens of milliseconds, which would show up as submission delay."""
    was = gc.isenabled()
    gc.collect()
    gc.disable()
    try:
        yield
    finally:
        if was:
            gc.enable()


def run_open_loop(server: Server, arrivals, reqs, timeout_s=120.0):
    """Submits each request at its arrival time (open loop) from this thread and
    collects results on a second thread.  Latency = completion - scheduled
    arrival: the server's submit-to-completion time plus any delay of the
    submission behind its scheduled arrival."""
    ids = [None] * len(reqs)
    results = [None] * len(reqs)
    late = [0.0] * len(reqs)
    submitted = threading.Semaphore(0)

    def collect():
        for i in range(len(reqs)):
            submitted.acquire()
            results[i] = server.result(ids[i], timeout_s)

    th = threading.Thread(target=collect)
    with _gc_paused():
        th.start()
        t0 = time.perf_counter()
        for i, (t, r) in enumerate(zip(arrivals, reqs)):
            dt = t0 + t - time.perf_counter()
            if dt > 0:
                time.sleep(dt)
            late[i] = max(0.0, time.perf_counter() - (t0 + t))
            ids[i] = server.submit(r)
            submitted.release()
        th.join()
        wall = time.perf_counter() - t0
    photons = float(sum(int(r["n_photons"].sum()) for r in reqs))
    lat = [x.latency_s + d for x, d in zip(results, late)]
    out = {"requests": len(reqs), "photons": photons, "wall_s": wall, "photons_per_s": photons / wall,
           "overflow_requests": int(sum(x.overflow for x in results)),
           "max_submit_delay_ms": float(max(late) * 1e3) if late else 0.0}
    out.update(_percentiles(lat))
    return out, results


def run_plain_loop(prop: Propagator, opts: RunOptions, arrivals, reqs, hit_capacity=1 << 20):
    """One pp_propagate call per request in arrival order on one worker;
    latency = completion - arrival."""
    o = RunOptions(**{**opts.__dict__})
    o.write_hits = True
    lat = []
    with _gc_paused():
        t0 = time.perf_counter()
        for t, r in zip(arrivals, reqs):
            dt = t0 + t - time.perf_counter()
            if dt > 0:
                time.sleep(dt)
            prop.propagate(r, o, hit_capacity=hit_capacity)
            lat.append(time.perf_counter() - (t0 + t))
        wall = time.perf_counter() - t0
    photons = float(sum(int(r["n_photons"].sum()) for r in reqs))
    out = {"requests": len(reqs), "photons": photons, "wall_s": wall, "photons_per_s": photons / wall}
    out.update(_percentiles(lat))
    return out

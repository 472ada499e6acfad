#!/usr/bin/env python
"""Benchmark: propagated photons/s of the batched persistent kernel on the
4096-pair mixed batch, next to the plain one-pair-per-launch path, the
end-to-end C-ABI call with host buffers and the CPU baseline.

One step = one propagation of a 4096-pair batch (photon counts log-uniform
in [1e4, 1e7], 50/50 isotropic point / 1 m Cherenkov-cone emitters with
random directions, sphere r = 0.21 m at a uniform distance in [2, 150] m in a
random direction; seawater 35 permille / 2 degC, Frank-Tamm spectrum
300-800 nm, HG g = 0.95, group-velocity time, PMT weighting, FP64 per-pair
statistics and 1000 x 1 ns histograms).  Every step uses a fresh batch
(different seeds).  Under torchrun each rank propagates its own batch (weak
scaling, no collective on the data path).

  python bench.py [--gpus N --steps K --warmup W] [--impl reference]
"""
import argparse
import datetime
import json
import os
import statistics
import subprocess
import sys
import threading
import time

REPO = os.path.dirname(os.path.abspath(__file__))
PKG_ROOT = os.path.join(REPO, "photonprop.jl_b200")
for _p in (REPO, PKG_ROOT):
    if _p not in sys.path:
        sys.path.insert(0, _p)

import numpy as np  # noqa: E402

METRIC = "propagated photons/s (batched vs plain, 1 B200); p50/p99 solve latency"
UNIT = "photons/s"
WORKLOAD = ("4096-pair mixed batch: photons/pair log-uniform [1e4,1e7], 50/50 isotropic point / 1 m "
            "Cherenkov-cone emitters (random directions), sphere r=0.21 m at U[2,150] m in a random "
            "direction; seawater 35 permille 2 degC, Frank-Tamm 300-800 nm, HG g=0.95, physical mode, "
            "PMT weight, FP64 per-pair stats + 1000 x 1 ns histograms")
RUN_KW = dict(mode="physical", g=0.95, t_max=1000.0, hist_t0=0.0, hist_bin_width=1.0, hist_bins=1000,
              pmt_weight=True)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--pairs", type=int, default=4096)
    ap.add_argument("--seed", type=int, default=2024)
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--no-tune", action="store_true")
    ap.add_argument("--serving-seconds", type=float, default=60.0,
                    help="length of the serving sample in the default run (0 = skip; one GPU only)")
    ap.add_argument("--serving-rate", type=float, default=200.0, help="request arrival rate, Hz")
    ap.add_argument("--overload-rate", type=float, default=2000.0,
                    help="arrival rate of the second, overload serving sample, Hz")
    ap.add_argument("--overload-seconds", type=float, default=10.0,
                    help="length of the overload serving sample (0 = skip)")
    ap.add_argument("--workload", choices=["batch", "serving", "surrogate", "surrogate-infer", "cone-grid", "point",
                                           "fits", "event", "llh", "large-pairs"], default="batch")
    ap.add_argument("--fit-photons", type=int, default=100_000_000, help="fits workload: photons per distance")
    ap.add_argument("--fit-distances", type=int, default=250)
    ap.add_argument("--fit-angles", type=int, default=250)
    ap.add_argument("--train-pairs", type=int, default=200_000)
    ap.add_argument("--test-pairs", type=int, default=20_000)
    ap.add_argument("--epochs", type=int, default=400)
    ap.add_argument("--train-distance", choices=["uniform", "loguniform"], default="loguniform",
                    help="distance law of the surrogate's training pairs (held-out pairs: uniform)")
    ap.add_argument("--full-weight-hits", type=float, default=1000.0)
    ap.add_argument("--max-photons", type=int, default=0,
                    help="cap photons per pair (small profiling cases; 0 = no cap)")
    ap.add_argument("--cascade-variant", action="store_true",
                    help="batch workload: run the kernel variant that samples the cascade profile "
                         "(PP_OPT_CASCADE) on the same pairs")
    return ap.parse_args()


def measured_hbm_gbs():
    """The pool's measured copy bandwidth (MEASURED_PEAKS.json), else the
    earlier measurement on this pool."""
    try:
        with open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"])
    except (OSError, KeyError, ValueError):
        return 6650.0


# ---------------------------------------------------------------------------
class ClockSampler:
    """nvidia-smi clocks and throttle reasons, sampled every 200 ms."""

    FIELDS = ["uuid", "clocks.sm", "clocks.max.sm", "power.draw", "clocks_event_reasons.active",
              "clocks_event_reasons.hw_slowdown", "clocks_event_reasons.hw_thermal_slowdown",
              "clocks_event_reasons.sw_thermal_slowdown", "clocks_event_reasons.sw_power_cap"]

    def __init__(self, uuid=None):
        self.uuid = uuid
        self.rows = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "--query-gpu=" + ",".join(self.FIELDS), "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) == len(self.FIELDS):
                self.rows.append(parts)

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        rows = self.rows
        if self.uuid:
            mine = [r for r in rows if self.uuid in r[0]]
            rows = mine or rows
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}

        def num(x):
            try:
                return float(x)
            except ValueError:
                return None
        sm = [num(r[1]) for r in rows if num(r[1]) is not None]
        mx = [num(r[2]) for r in rows if num(r[2]) is not None]
        pw = [num(r[3]) for r in rows if num(r[3]) is not None]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({n for r in rows for n, v in zip(names, r[5:9]) if v.strip().lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "power_w_max": max(pw) if pw else None, "samples": len(rows), "reasons": reasons}


# ---------------------------------------------------------------------------
class CpuArm:
    """The reference's algorithm on the host cores: the FP64 C restatement of
    cuda_propagate_photons! (src/photon_prop_cuda.jl:262-386) and of
    propagate_distance's host finish (:588-644) in oracle/, OpenMP over one
    flat (pair, photon-chunk) index space on every host thread.  The batch is
    built by oracle/batches.py (the same numbers as the product's generator),
    so a process that times it never loads the product library.  The sample is
    the first ceil(f N_i) photons of every pair, f chosen for a given length of
    work, so its photon mix (emitters, distances, photons per pair) follows the
    batch's."""

    def __init__(self, seed, n_pairs, run_kw, max_photons=0):
        from oracle import batches as ob
        from oracle import oracle as O
        from oracle import tables as tb
        self.ob, self.O = ob, O
        m = tb.cascadia(35.0, 2.0)
        knots = tb.cherenkov_spectrum_knots((300.0, 800.0), 20, m).astype(np.float32).astype(np.float64)
        self.T = O.make_tables(m, knots, pmt=ob.pmt_table())
        self.n_pairs = n_pairs
        self.batch = ob.mixed_batch(n_pairs, seed=seed)
        if max_photons > 0:  # the GPU arm's --max-photons cap
            self.batch["n_photons"] = np.minimum(self.batch["n_photons"], max_photons)
        self.oo = O.make_opts(mode=O.MODE_PHYSICAL, g=float(np.float32(run_kw["g"])), t_max=run_kw["t_max"],
                              hist_t0=run_kw["hist_t0"], hist_bin_width=run_kw["hist_bin_width"],
                              hist_bins=run_kw["hist_bins"], flags=O.OPT_PMT_WEIGHT)
        self.cores = os.cpu_count() or 1
        self.batch_photons = int(self.batch["n_photons"].sum())
        self.frac = min(1.0, 2e5 / self.batch_photons)
        self.sample = self.ob.sampled(self.batch, self.frac)

    def run(self):
        """One pass over the sample: (photons, seconds, threads that ran)."""
        t0 = time.perf_counter()
        self.O.propagate(self.T, self.sample, self.oo, n_threads=self.cores)
        dt = time.perf_counter() - t0
        return int(self.sample["n_photons"].sum()), dt, self.O.last_threads_used

    def calibrate(self, seconds):
        """Sizes the sample for about `seconds` of work per pass."""
        _, dt, _ = self.run()
        self.frac = min(1.0, self.frac * seconds / max(dt, 1e-3))
        self.sample = self.ob.sampled(self.batch, self.frac)

    def describe(self, photons, dt, used):
        return {"value": photons / dt, "unit": UNIT, "cores": used, "kind": "port", "seconds": dt,
                "photons": photons, "batch_photons": self.batch_photons,
                "sample": f"first ceil({self.frac:.3e} N_i) photons of each of the {self.n_pairs} pairs of the "
                          f"batch ({photons:.3e} photons, {dt:.1f} s), FP64 oracle, OpenMP over (pair, photon) "
                          f"chunks, {used} threads ran (host has {self.cores})"}


def cpu_baseline(seed, n_pairs, target_seconds, run_kw, max_photons=0):
    """One calibrated CPU pass of about target_seconds (see CpuArm)."""
    arm = CpuArm(seed, n_pairs, run_kw, max_photons)
    arm.calibrate(target_seconds)
    return arm.describe(*arm.run())


def bench_config(n_pairs, seed, photons, world):
    """The `config` object both arms print (the same workload)."""
    return {"workload": WORKLOAD, "pairs": n_pairs, "batch_seed": seed, "photons_per_step_per_gpu": photons,
            "mode": "physical", "histogram": "1000 x 1 ns FP64 per pair",
            "l2": "inputs and outputs of a step exceed L2 (~5.9e9 photons, 32.8 MB histograms); the GPU arm "
                  "also writes 256 MiB between timed steps",
            "parallelism": f"{world} independent ranks (weak scaling, no collective)"}


def run_serving(prop, seconds, seed=0, rate_hz=200.0):
    """Open-loop Poisson stream (rate_hz, 1-64 pairs per request, 1e4-1e6
    photons per pair) through the continuous-batching server and through the
    one-launch-per-request loop on the same arrivals."""
    from photonprop_b200 import serving
    arrivals, reqs = serving.requests(rate_hz=rate_hz, duration_s=seconds, seed=seed)
    opts = serving.RunOptions(mode="physical", g=0.95, t_max=1000.0, hist_bins=1000)
    with serving.Server(prop, opts) as srv:
        w_arr, w_req = serving.requests(rate_hz=rate_hz, duration_s=min(1.0, seconds), seed=seed + 99)
        serving.run_open_loop(srv, w_arr, w_req)  # warm-up
        out, _ = serving.run_open_loop(srv, arrivals, reqs)
        out["batches"] = srv.counters()["batches"]
    plain = serving.run_plain_loop(prop, opts, arrivals, reqs)
    return {"rate_hz": rate_hz, "seconds": seconds, "continuous_batching": out, "plain_loop": plain,
            "what": "request latency = completion - arrival (host clock); photons/s over the stream"}


def run_serving_workload(args):
    """--workload serving: the full serving configuration on one GPU."""
    import torch
    import photonprop_b200 as pp
    torch.cuda.set_device(0)
    medium = pp.make_seawater(35.0, 2.0)
    spec = pp.CherenkovSpectrum((300.0, 800.0), 20, medium)
    with pp.Propagator(medium, spec, pp.p_one_pmt_acc, device=0) as prop:
        r = run_serving(prop, args.serving_seconds, seed=args.seed, rate_hz=args.serving_rate)
    cb = r["continuous_batching"]
    line = {"metric": "serving photons/s; p50/p99/p99.9 request latency", "value": cb["photons_per_s"],
            "unit": UNIT, "n_gpus": 1, "latency_ms": {k: cb[k] for k in ("p50_ms", "p99_ms", "p99.9_ms")},
            "higher_is_better": True, "data": "synthetic",
            "config": {"workload": f"Poisson {r['rate_hz']} req/s for {r['seconds']} s, 1-64 pairs/request, "
                                   "photons/pair log-uniform [1e4,1e6], mixed emitters, 40 GB HBM admission "
                                   "budget at 32 B per expected hit"},
            "serving": r}
    print(json.dumps(line), flush=True)


def surrogate_inference_rate(device, n=1_000_000, net=None, reps=10):
    """Device queries/s of the surrogate network's tcgen05 inference kernel on
    n queries per batch (features drawn over the trained range)."""
    import torch
    from photonprop_b200 import surrogate as sg
    own = net is None
    if own:
        net = sg.MLP(device, seed=1)
        net.set_normalization([1.2, 0.0, 5.5, 0.5], [0.5, 0.6, 0.9, 0.5], [0, 0, 0, 0, 0], [1, 1, 1, 1, 1])
    rng = np.random.default_rng(0)
    x = np.stack([rng.uniform(np.log10(2), np.log10(150), n), rng.uniform(-1, 1, n), rng.uniform(4, 7, n),
                  rng.integers(0, 2, n)], axis=1).astype(np.float32)
    dev = torch.device("cuda", device)
    d_x = torch.from_numpy(x).to(dev)
    d_o = torch.empty((5, n), dtype=torch.float32, device=dev)
    s = torch.cuda.Stream(device=dev)
    for _ in range(3):
        net.forward(d_x, d_o, n, physical=True, stream=s)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(s)
    for _ in range(reps):
        net.forward(d_x, d_o, n, physical=True, stream=s)
    e1.record(s)
    s.synchronize()
    t = e0.elapsed_time(e1) / 1e3 / reps
    flops = 2.0 * (4 * 128 + 2 * 128 * 128 + 128 * 5) * n
    if own:
        net.close()
    return {"queries": n, "seconds_per_batch": t, "queries_per_s": n / t, "tflops": flops / t / 1e12}


def arrival_time_shape(test, g, pred, hi, opts):
    """How well the predicted arrival-time mixture matches the MC's residual
    time distribution on the selected held-out pairs: the Kolmogorov distance
    between the mixture's CDF and the 1e7-photon MC histogram's CDF, beside
    that of the pair's own EM fit (what a 2-Gamma mixture can do) and of the
    1e6-photon MC histogram (the noise floor), and the error of the mean."""
    from scipy import stats
    t0, bw, bins = opts.hist_t0, opts.hist_bin_width, opts.hist_bins
    edges = t0 + bw * np.arange(1, bins + 1)

    def mix_cdf(p, r):
        w, a1, a2, th = p
        return w * stats.gamma.cdf(r, a1, scale=th) + (1 - w) * stats.gamma.cdf(r, a2, scale=th)

    ks_nn, ks_fit, ks_mc, mean_err = [], [], [], []
    fits = test.y[g].astype(np.float64)
    for i, k in enumerate(np.nonzero(g)[0]):
        h_hi = hi.hist[i]
        if h_hi.sum() <= 0:
            continue
        r = edges - test.tshift[k]
        c_hi = np.cumsum(h_hi) / h_hi.sum()
        c_lo = np.cumsum(test.hist[k]) / max(test.hist[k].sum(), 1e-300)
        w_fit = 1 / (1 + np.exp(-fits[i, 1]))
        ks_nn.append(np.max(np.abs(mix_cdf(pred[k, 1:5], r) - c_hi)))
        ks_fit.append(np.max(np.abs(mix_cdf((w_fit, *np.exp(fits[i, 2:5])), r) - c_hi)))
        ks_mc.append(np.max(np.abs(c_lo - c_hi)))
        centres = edges - 0.5 * bw - test.tshift[k]
        m_hi = float(np.sum(h_hi * centres) / h_hi.sum())
        w, a1, a2, th = pred[k, 1:5]
        m_nn = th * (w * a1 + (1 - w) * a2)
        mean_err.append(abs(m_nn - m_hi) / max(abs(m_hi), 1e-9))
    return {"pairs": len(ks_nn), "median_ks_surrogate": float(np.median(ks_nn)),
            "median_ks_em_fit": float(np.median(ks_fit)), "median_ks_mc_1e6": float(np.median(ks_mc)),
            "median_rel_err_mean_residual": float(np.median(mean_err)),
            "what": "Kolmogorov distance to the 1e7-photon MC residual-time CDF"}


def run_surrogate_workload(args):
    """--workload surrogate: MC training set (mixed-batch geometry, 1e6 photons
    per pair), training by the library's kernels, held-out accuracy against MC,
    query rate against the MC kernel."""
    import torch
    import photonprop_b200 as pp
    from photonprop_b200 import surrogate as sg
    torch.cuda.set_device(0)
    medium = pp.make_seawater(35.0, 2.0)
    spec = pp.CherenkovSpectrum((300.0, 800.0), 20, medium)
    opts = pp.RunOptions(mode="physical", g=0.95, t_max=1000.0, hist_bins=1000)
    out = {}
    with pp.Propagator(medium, spec, pp.p_one_pmt_acc, device=0) as prop:
        t0 = time.perf_counter()
        train = sg.mc_dataset(prop, sg.training_pairs(args.train_pairs, 1_000_000, seed=args.seed,
                                                      distance_law=args.train_distance), opts,
                              full_weight_hits=args.full_weight_hits)
        test_pairs = sg.training_pairs(args.test_pairs, 1_000_000, seed=args.seed + 1)
        test = sg.mc_dataset(prop, test_pairs, opts, return_hist=True)
        t_data = time.perf_counter() - t0
        s = sg.Surrogate(prop, opts, seed=args.seed)
        t0 = time.perf_counter()
        losses = s.fit(train, epochs=args.epochs, batch=4096, lr=2e-3)
        t_train = time.perf_counter() - t0
        pred = s.predict_features(test.x, physical=True)
        raw = s.predict_features(test.x, physical=False)
        acc = {}
        for cut in (100, 1000, 10000):
            g = test.hits >= cut
            if g.sum():
                rel = np.abs(pred[g, 0] - test.mu[g]) / test.mu[g]
                acc[f"hits>={cut}"] = {"pairs": int(g.sum()), "median_rel_err": float(np.median(rel)),
                                       "frac_within_5pct": float(np.mean(rel < 0.05)),
                                       "sum_ratio": float(pred[g, 0].sum() / test.mu[g].sum())}
        # the same held-out pairs with >= 1000 hits again at 1e7 photons (other seeds): a
        # truth with 10x the statistics, and the 1e6-photon MC judged against it as the noise floor
        g = test.hits >= 1000
        hp = np.ascontiguousarray(test_pairs[g]).copy()
        hp["n_photons"] = 10_000_000
        hp["seed"] = [pp.propagation.pair_seed(args.seed + 77, i) for i in range(len(hp))]
        hi = sg.mc_dataset(prop, hp, opts, min_hits_mu=0, min_hits_fit=0, return_hist=True)
        truth = hi.mu / 10.0
        rel_nn = np.abs(pred[g, 0] - truth) / truth
        rel_mc = np.abs(test.mu[g] - truth) / truth
        acc["hits>=1000, 1e7-photon truth"] = {
            "pairs": int(g.sum()), "median_rel_err": float(np.median(rel_nn)),
            "frac_within_5pct": float(np.mean(rel_nn < 0.05)), "sum_ratio": float(pred[g, 0].sum() / truth.sum()),
            "mc_1e6_median_rel_err": float(np.median(rel_mc)), "mc_1e6_frac_within_5pct": float(np.mean(rel_mc < 0.05))}
        acc["arrival_time_shape, hits>=1000"] = arrival_time_shape(test, g, pred, hi, opts)
        r2 = {}
        for j, name in enumerate(["ln_mu_over_N", "logit_w", "ln_a1", "ln_a2", "ln_theta"]):
            m = test.mask[:, j] > 0
            if m.sum() > 2:
                r2[name] = float(1 - np.mean((raw[m, j] - test.y[m, j]) ** 2) / np.var(test.y[m, j]))
        inf = surrogate_inference_rate(0, 1_000_000, net=s.net)
        # MC rate on the same kind of query (1e6 photons per pair)
        mc_pairs = np.ascontiguousarray(test_pairs[:4096])
        dev = torch.device("cuda", 0)
        d_pairs = torch.from_numpy(mc_pairs.view(np.uint8).copy()).to(dev)
        d_cnt = torch.zeros(4, dtype=torch.int64, device=dev)
        d_st = torch.zeros((len(mc_pairs), 8), dtype=torch.float64, device=dev)
        d_hi = torch.zeros((len(mc_pairs), 1000), dtype=torch.float64, device=dev)
        d_h = torch.zeros(64, dtype=torch.uint8, device=dev)
        o = pp.RunOptions(**{**opts.__dict__})
        o.write_hits = False
        prop.propagate_device(d_pairs, len(mc_pairs), o, d_h, 0, d_cnt, d_st, d_hi)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        prop.propagate_device(d_pairs, len(mc_pairs), o, d_h, 0, d_cnt, d_st, d_hi)
        e1.record()
        torch.cuda.synchronize()
        mc_rate = len(mc_pairs) / (e0.elapsed_time(e1) / 1e3)
        out = {"metric": "surrogate queries/s and hit-count error vs MC", "value": inf["queries_per_s"],
               "unit": "queries/s", "n_gpus": 1, "higher_is_better": True, "data": "synthetic",
               "config": {"workload": f"{args.train_pairs} training ({args.train_distance} distance) + {args.test_pairs} "
                                      "held-out pairs of the mixed-batch geometry, 1e6 photons each; MLP 4-128-128-128-5 GELU, "
                                      f"BF16/FP32-acc, Adam 2e-3 cosine-decayed, batch 4096, {args.epochs} epochs; "
                                      "inference at 1e6 queries per batch"},
               "inference": inf, "mc_queries_per_s": mc_rate, "speedup_vs_mc": inf["queries_per_s"] / mc_rate,
               "held_out_mu": acc, "held_out_r2": r2, "loss_first_last": [losses[0], losses[-1]],
               "seconds": {"mc_dataset": t_data, "training": t_train}}
    print(json.dumps(out), flush=True)


def run_cone_grid(args):
    """--workload cone-grid: a 1 m Cherenkov track along +z, 1e8 photons per
    launch, spheres at {5,10,20,50,100} m x polar {0,45,90,135,180} deg; PMT
    weighting from the 5 nm table; one pair per launch (plain) and all 25 in
    one batched launch."""
    import torch
    import photonprop_b200 as pp
    torch.cuda.set_device(0)
    medium = pp.make_seawater(35.0, 2.0)
    spec = pp.CherenkovSpectrum((300.0, 800.0), 20, medium)
    pairs = pp.batches.cone_grid_pairs(n_photons=100_000_000, seed=args.seed)
    ro = pp.RunOptions(mode="physical", g=0.95, t_max=1000.0, hist_bins=1000)
    with pp.Propagator(medium, spec, pp.p_one_pmt_acc_5nm, device=0) as prop:
        # warm-up at the timed hit capacity, so that no device allocation
        # falls inside the timed pass
        prop.propagate_plain(pairs[:2], ro, hit_capacity=1 << 24)
        t0 = time.perf_counter()
        rp = prop.propagate_plain(pairs, ro, hit_capacity=1 << 24)
        tp = time.perf_counter() - t0
        prop.propagate(pairs, ro, hit_capacity=1 << 24)
        t0 = time.perf_counter()
        rb = prop.propagate(pairs, ro, hit_capacity=1 << 24)
        tb = time.perf_counter() - t0
    photons = float(pairs["n_photons"].sum())
    line = {"metric": "propagated photons/s, one pair per launch (cone grid)", "value": photons / tp,
            "unit": UNIT, "n_gpus": 1, "higher_is_better": True, "data": "synthetic", "dtype": "f32",
            "config": {"workload": "1 m Cherenkov track along +z, 1e8 photons per launch, r=0.21 m spheres at "
                                   "{5,10,20,50,100} m x polar {0,45,90,135,180} deg (25 launches), PMT 5 nm table "
                                   "300-700 nm (peak 0.2708), seawater 35 permille 2 degC, g=0.95"},
            "plain_host_api_photons_per_s": photons / tp, "batched_host_api_photons_per_s": photons / tb,
            "hits_per_pair": rp.stats[:, 0].tolist(), "sum_w_per_pair": rp.stats[:, 1].tolist(),
            "identical_stats": bool(np.allclose(rp.stats, rb.stats, rtol=1e-9))}
    print(json.dumps(line), flush=True)


def run_large_pairs(args):
    """--workload large-pairs: eight pairs of 9e6-1e7 photons (the decade that
    holds 90 % of the benchmark batch's photons), 20-40 m, one launch per
    pair and one batched launch, host API, twice; photons/s of each."""
    import torch
    import photonprop_b200 as pp
    torch.cuda.set_device(0)
    medium = pp.make_seawater(35.0, 2.0)
    spec = pp.CherenkovSpectrum((300.0, 800.0), 20, medium)
    b = pp.batches.mixed_batch(8, seed=77, n_min=9e6, n_max=1e7, d_min=20.0, d_max=40.0)
    ro = pp.RunOptions(**RUN_KW)
    with pp.Propagator(medium, spec, pp.p_one_pmt_acc, device=0) as prop:
        tp = tb = 0.0
        for _ in range(2):
            t0 = time.perf_counter()
            a = prop.propagate_plain(b, ro)
            tp = time.perf_counter() - t0
            t0 = time.perf_counter()
            c = prop.propagate(b, ro)
            tb = time.perf_counter() - t0
    photons = float(b["n_photons"].sum())
    print(json.dumps({"metric": "photons/s on eight 9e6-1e7-photon pairs, plain vs batched (host API)",
                      "unit": UNIT, "plain_photons_per_s": photons / tp, "batched_photons_per_s": photons / tb,
                      "hits_plain": a.n_hits, "hits_batched": c.n_hits, "n_gpus": 1, "data": "synthetic"}),
          flush=True)


def run_point(args):
    """--workload point: the small CPU-runnable case (isotropic point source,
    1e5 photons, sphere at 10 m along +x, 500 x 1 ns histogram, seed 0) on the
    GPU and through the FP64 oracle on all host cores, matched photon by photon."""
    import torch
    import photonprop_b200 as pp
    from oracle import oracle as O
    from oracle import tables as tb
    torch.cuda.set_device(0)
    medium = pp.make_seawater(35.0, 2.0)
    spec = pp.CherenkovSpectrum((300.0, 800.0), 20, medium)
    pair = pp.batches.point_source_pair(100_000, target=(10.0, 0.0, 0.0), seed=0)
    ro = pp.RunOptions(mode="physical", g=0.95, t_max=500.0, hist_bins=500)
    with pp.Propagator(medium, spec, pp.p_one_pmt_acc, device=0) as prop:
        for _ in range(3):
            prop.propagate(pair, ro)
        t0 = time.perf_counter()
        r = prop.propagate(pair, ro)
        tg = time.perf_counter() - t0
        knots = prop.knots().astype(np.float64)
    T = O.make_tables(tb.cascadia(35.0, 2.0), knots, pmt=(pp.p_one_pmt_acc.wavelengths, pp.p_one_pmt_acc.acceptance))
    op = O.pairs_array(1)
    for f in ("pos", "t0", "dir", "track_len", "target", "radius", "n_photons", "seed", "emitter"):
        op[f] = pair[f]
    c = ro.to_c()
    oo = O.make_opts(mode=c.mode, max_steps=c.max_steps, g=float(np.float32(c.g)), t_max=c.t_max,
                     hist_bins=c.hist_bins, flags=c.flags & 3)
    t0 = time.perf_counter()
    h, s, hist, steps, total = O.propagate(T, op, oo, n_threads=os.cpu_count() or 1)
    tc = time.perf_counter() - t0
    gk = {int(x["photon"]): x for x in r.hits}
    ok = {int(x["photon"]): x for x in h}
    both = sorted(set(gk) & set(ok))
    dt = max((abs(float(gk[k]["time"]) - ok[k]["time"]) for k in both), default=0.0)
    line = {"metric": "isotropic point source, 1e5 photons: hits, histogram, GPU vs FP64 oracle",
            "value": 1e5 / tg, "unit": UNIT, "n_gpus": 1, "data": "synthetic",
            "gpu_e2e_seconds": tg, "cpu_oracle_seconds": tc, "cpu_cores": os.cpu_count(),
            "hits_gpu": r.n_hits, "hits_oracle": int(total), "matched": len(both), "max_abs_dt_ns": dt,
            "sum_w_gpu": float(r.stats[0, 1]), "sum_w_oracle": float(s[0, 1]),
            "hist_nonzero_bins": int(np.count_nonzero(r.hist[0]))}
    print(json.dumps(line), flush=True)


def run_fits(args):
    """--workload fits: make_photon_fits(1e8 photons, 250 distances, 250
    angles, 300 m) as example_full.jl:136 calls it: compat mode, Cascadia
    medium, PMT weight.  e2e = the public call (pairs built on the host, one
    batched launch, reweighting and Gamma fits on the device, the fit table
    back on the host).  The device breakdown times the propagation and the
    fit stage with CUDA events; the CPU baseline is the FP64 oracle's
    propagation of the first L photons of every distance plus its fits."""
    import torch
    import photonprop_b200 as pp
    from photonprop_b200 import modelling as md
    torch.cuda.set_device(0)
    n_ph, n_d, n_a, maxd = args.fit_photons, args.fit_distances, args.fit_angles, 300.0
    m = pp.make_cascadia_medium_properties()
    spec = pp.CherenkovSpectrum((300.0, 800.0), 20, m)
    ro = pp.RunOptions(mode="compat", pmt_weight=True, hist_bins=0)
    pairs, distances, angles = md.fit_pairs(n_ph, n_d, n_a, maxd, seed=args.seed)
    with pp.Propagator(m, spec, pp.p_one_pmt_acc, device=0) as prop:
        warm = md.propagate_fit(prop, pairs, angles, ro)  # allocates the buffers
        cap = int(warm.n_hits * 1.05) + 4096  # the device breakdown keeps every hit
        e2e = []
        for _ in range(2):
            t0 = time.perf_counter()
            df = md.make_photon_fits(n_ph, n_d, n_a, maxd, propagator=prop, seed=args.seed)
            e2e.append(time.perf_counter() - t0)
        # device breakdown
        dev = torch.device("cuda", 0)
        d_pairs = torch.from_numpy(pairs.view(np.uint8).copy()).to(dev)
        d_hits = torch.empty(cap * 64, dtype=torch.uint8, device=dev)
        d_cnt = torch.zeros(4, dtype=torch.int64, device=dev)
        d_stats = torch.zeros((n_d, 8), dtype=torch.float64, device=dev)
        d_m = torch.zeros((n_d, n_a, 4), dtype=torch.float64, device=dev)
        d_f = torch.zeros((n_d, n_a, 3), dtype=torch.float64, device=dev)
        L = pp._lib.load()
        stream = torch.cuda.current_stream(dev)
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
        t_prop, t_fit = [], []
        for _ in range(4):
            ev[0].record(stream)
            prop.propagate_device(d_pairs, n_d, ro, d_hits, cap, d_cnt, d_stats, None, stream=stream)
            ev[1].record(stream)
            pp._lib.check(L.pp_fit_hits_device(prop.handle, d_pairs.data_ptr(), n_d, pp._lib.MODE_COMPAT,
                                               d_hits.data_ptr(), cap, d_cnt.data_ptr(), angles.ctypes.data, n_a,
                                               d_m.data_ptr(), d_f.data_ptr(), stream.cuda_stream), prop.handle)
            ev[2].record(stream)
            torch.cuda.synchronize()
            t_prop.append(ev[0].elapsed_time(ev[1]) / 1e3)
            t_fit.append(ev[1].elapsed_time(ev[2]) / 1e3)
        hits = int(d_cnt[0].item())
        knots = prop.knots().astype(np.float64)
    photons = float(n_ph) * n_d
    tp, tf = float(np.median(t_prop[1:])), float(np.median(t_fit[1:]))
    line = {"metric": "make_photon_fits photons/s (propagation + reweighting + Gamma fits)",
            "value": photons / min(e2e), "unit": UNIT, "n_gpus": 1, "higher_is_better": True, "data": "synthetic",
            "dtype": "f32 (FP64 moments and fits)",
            "config": {"workload": f"make_photon_fits({n_ph:.0e}, {n_d}, {n_a}, {maxd:.0f} m): isotropic source, "
                                   "0.21 m sphere at Sobol distances, Sobol observation angles, compat mode, "
                                   "Cascadia medium, PMT weight"},
            "e2e_seconds": min(e2e), "hits": hits,
            "device": {"propagation_s": tp, "fit_stage_s": tf, "propagation_photons_per_s": photons / tp,
                       "fit_hit_angle_evals_per_s": hits * n_a / tf},
            "fit_table_rows": len(df), "finite_fits": int(np.isfinite(df["fit_alpha"]).sum())}
    if not args.no_cpu_baseline:
        line["cpu_baseline"] = fits_cpu_baseline(pairs, angles, knots, args.cpu_seconds)
    print(json.dumps(line), flush=True)


def fits_cpu_baseline(pairs, angles, knots, target_seconds):
    """FP64 oracle: propagation of the first L photons of every distance
    (all host threads) and the reweighting + Gamma fits of its hits."""
    from oracle import fits as F
    from oracle import oracle as O
    from oracle import tables as tb
    import photonprop_b200 as pp
    m = tb.cascadia()
    T = O.make_tables(m, knots, pmt=(pp.p_one_pmt_acc.wavelengths, pp.p_one_pmt_acc.acceptance))
    op = O.pairs_array(len(pairs))
    for f in ("pos", "t0", "dir", "track_len", "target", "radius", "n_photons", "seed", "emitter"):
        op[f] = pairs[f]
    oo = O.make_opts(mode=O.MODE_COMPAT, g=0.99, hist_bins=0, flags=O.OPT_PMT_WEIGHT)
    cores = os.cpu_count() or 1

    def run(lim):
        t0 = time.perf_counter()
        h, s, _, _, total = O.propagate(T, op, oo, photon_limit=lim, n_threads=cores, hit_cap=1 << 22)
        n800 = tb.refractive_index(800.0, m)
        tab = F.int_table()
        for p in range(len(pairs)):
            hp = h[h["pair"] == p]
            if len(hp) == 0:
                continue
            d = float(np.linalg.norm(pairs["target"][p].astype(np.float64)))
            tres = hp["time"] - (d - 0.21) * n800 / 0.299792458
            theta = np.arccos(np.clip(hp["dir0"][:, 2], -1, 1))
            n = tb.refractive_index(hp["wavelength"], m)
            for a in angles:
                mo = F.moments(tres, F.get_dir_reweight(theta, a, n, tab) * hp["weight"])
                F.gamma_fit_moments(mo[1], mo[2], mo[3])
        return time.perf_counter() - t0

    lim = 2000
    dt = max(run(lim), 1e-3)
    lim = int(max(2000, min(int(pairs["n_photons"][0]), lim * target_seconds / dt)))
    dt = run(lim)
    photons = lim * len(pairs)
    return {"value": photons / dt, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": f"first {lim} photons of each of the {len(pairs)} distances ({photons:.3e} photons, {dt:.1f} s), "
                      f"FP64 oracle propagation (OpenMP {cores} threads) + numpy reweighting/fits over "
                      f"{len(angles)} angles"}


def run_event(args):
    """--workload event: one 100 GeV electron cascade at the origin along +z
    -> point sources with the cascade angular profile every 0.1 m over 20 m
    (light-yield kernel, metres mode) -> every source with every module of a 5 x 5 string
    detector (20 m string spacing, 20 modules 5 m apart, r = 0.21 m) ->
    batched propagation (physical mode).  Everything stays on the device;
    each stage is timed with CUDA events."""
    import ctypes
    import torch
    import photonprop_b200 as pp
    from photonprop_b200 import lightyield as ly
    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    medium = pp.make_seawater(35.0, 2.0)
    spec = pp.CherenkovSpectrum((300.0, 800.0), 20, medium)
    parts = ly.particles_array([ly.Particle((0.0, 0.0, 0.0), (0.0, 0.0, 1.0), 0.0, 100.0, ly.ParticleType.EMinus)])
    xs = np.arange(-40.0, 40.1, 20.0)
    mods = np.array([[x, y, z, 0.21] for x in xs for y in xs for z in np.arange(-40.0, 55.1, 5.0)],
                    dtype=np.float32)
    ro = pp.RunOptions(mode="physical", g=0.95, t_max=1000.0, hist_bins=1000, cascade=True)
    L = pp._lib.load()
    with pp.Propagator(medium, spec, pp.p_one_pmt_acc, device=0) as prop:
        n_src_cap = 400
        d_parts = torch.from_numpy(parts.view(np.uint8).copy()).to(dev)
        d_src = torch.zeros(n_src_cap * 80, dtype=torch.uint8, device=dev)
        d_mods = torch.from_numpy(mods.copy()).to(dev)
        ng = ctypes.c_int64(0)
        s = torch.cuda.current_stream(dev)
        # sizes first (one untimed pass)
        pp._lib.check(L.pp_particles_to_sources_device(prop.handle, d_parts.data_ptr(), 1, 0.0, 20.0, 0.1,
                                                       pp._lib.LY_METRES, 300.0, 800.0,
                                                       pp._lib.EMITTER_CASCADE, d_src.data_ptr(), n_src_cap,
                                                       ctypes.byref(ng), s.cuda_stream), prop.handle)
        n_src = int(ng.value) - 1
        n_pairs = n_src * len(mods)
        d_pairs = torch.zeros(n_pairs * 80, dtype=torch.uint8, device=dev)
        cap = 1 << 22
        d_hits = torch.empty(cap * 64, dtype=torch.uint8, device=dev)
        d_cnt = torch.zeros(4, dtype=torch.int64, device=dev)
        d_stats = torch.zeros((n_pairs, 8), dtype=torch.float64, device=dev)
        d_hist = torch.zeros((n_pairs, 1000), dtype=torch.float64, device=dev)
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
        times = []
        for it in range(4):
            ev[0].record(s)
            pp._lib.check(L.pp_particles_to_sources_device(prop.handle, d_parts.data_ptr(), 1, 0.0, 20.0, 0.1,
                                                           pp._lib.LY_METRES, 300.0, 800.0,
                                                           pp._lib.EMITTER_CASCADE, d_src.data_ptr(),
                                                           n_src_cap, ctypes.byref(ng), s.cuda_stream), prop.handle)
            ev[1].record(s)
            pp._lib.check(L.pp_cross_pairs_device(prop.handle, d_src.data_ptr(), n_src, d_mods.data_ptr(), len(mods),
                                                  it, d_pairs.data_ptr(), s.cuda_stream), prop.handle)
            ev[2].record(s)
            prop.propagate_device(d_pairs, n_pairs, ro, d_hits, cap, d_cnt, d_stats, d_hist, stream=s)
            ev[3].record(s)
            torch.cuda.synchronize()
            times.append([ev[0].elapsed_time(ev[1]), ev[1].elapsed_time(ev[2]), ev[2].elapsed_time(ev[3])])
        src = d_src[: n_src * 80].cpu().numpy().view(pp._lib.PAIR_DTYPE)
        photons = float(src["n_photons"].sum()) * len(mods)
        hits = int(d_cnt[0].item())
    t = np.median(np.array(times[1:]), axis=0)
    line = {"metric": "event-driven batch: cascade -> sources -> pairs -> propagation, photons/s", "unit": UNIT,
            "value": photons / (t.sum() / 1e3), "n_gpus": 1, "data": "synthetic", "higher_is_better": True,
            "config": {"workload": "100 GeV e- cascade along +z, cascade-profile point sources every 0.1 m over 20 m, "
                                   f"{len(mods)} modules (5 x 5 strings, 20 m spacing, 20 modules 5 m apart), "
                                   "physical mode, 1000 x 1 ns histograms"},
            "sources": n_src, "pairs": n_pairs, "photons": photons, "hits": hits,
            "device_ms": {"particle_to_sources": float(t[0]), "cross_pairs": float(t[1]),
                          "propagation": float(t[2])}}
    print(json.dumps(line), flush=True)


def run_llh(args):
    """--workload llh: the event of --workload event (100 GeV e-, 200
    cascade-profile sources x 500 modules) observed once by the MC kernel (each weighted hit
    kept with probability = its weight), per-(source, module) hypothesis
    parameters from an independent MC run (expected photons + Gamma-mixture
    fit of each pair), then the extended likelihood of 64 energy hypotheses
    per launch on the device.  Reported: hypotheses/s of the likelihood
    kernel, the surrogate's cost of producing one hypothesis's parameters
    (1e5 queries), and the MC kernel's time for one hypothesis."""
    import torch
    import photonprop_b200 as pp
    from photonprop_b200 import event as ev
    from photonprop_b200 import lightyield as ly
    from photonprop_b200 import surrogate as sg
    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    medium = pp.make_seawater(35.0, 2.0)
    spec = pp.CherenkovSpectrum((300.0, 800.0), 20, medium)
    xs = np.arange(-40.0, 40.1, 20.0)
    mods = np.array([[x, y, z, 0.21] for x in xs for y in xs for z in np.arange(-40.0, 55.1, 5.0)],
                    dtype=np.float32)
    part = ly.Particle((0.0, 0.0, 0.0), (0.0, 0.0, 1.0), 0.0, 100.0, ly.ParticleType.EMinus)
    ro = pp.RunOptions(mode="physical", g=0.95, t_max=1000.0, hist_bins=1000)
    with pp.Propagator(medium, spec, pp.p_one_pmt_acc, device=0) as prop:
        src, _ = ly.particles_to_sources(prop, [part], (0.0, 20.0), 0.1, mode="metres", emitter="cascade")
        S, M = len(src), len(mods)
        obs_pairs = ly.cross_pairs(prop, src, mods, seed=11)
        t0 = time.perf_counter()
        res = prop.propagate(obs_pairs, pp.RunOptions(mode="physical", g=0.95, t_max=1000.0, hist_bins=0),
                             hit_capacity=1 << 22)
        t_mc = time.perf_counter() - t0
        keep = np.random.default_rng(0).uniform(size=len(res.hits)) < res.hits["weight"]
        res.hits = res.hits[keep]
        times = ev.mc_hit_times(res, S, M)
        hyp_pairs = ly.cross_pairs(prop, src, mods, seed=12)
        ds = sg.mc_dataset(prop, hyp_pairs, ro, min_hits_mu=0, min_hits_fit=0)
        y = ds.y.astype(np.float64)
        prm = np.stack([ds.mu, 1 / (1 + np.exp(-y[:, 1])), np.exp(y[:, 2]), np.exp(y[:, 3]), np.exp(y[:, 4]),
                        sg.time_shift(hyp_pairs, medium) + hyp_pairs["t0"]], axis=1)
        prm = np.nan_to_num(prm.reshape(S, M, 6).transpose(1, 0, 2), nan=1.0)
        H = 64
        scales = np.geomspace(0.5, 2.0, H)
        hyp = np.repeat(prm[None], H, axis=0)
        hyp[..., 0] *= scales[:, None, None]
        counts = np.array([len(t) for t in times], dtype=np.int64)
        offs = np.concatenate([[0], np.cumsum(counts)])
        d_p = torch.from_numpy(np.ascontiguousarray(hyp)).to(dev)
        d_o = torch.from_numpy(offs).to(dev)
        d_t = torch.from_numpy(np.concatenate(times)).to(dev)
        d_l = torch.zeros((H, M), dtype=torch.float64, device=dev)
        L = pp._lib.load()
        st = torch.cuda.current_stream(dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        tl = []
        for _ in range(4):
            e0.record(st)
            pp._lib.check(L.pp_event_llh_device(prop.handle, pp._lib.LLH_SHIFTED, H, S, M, d_p.data_ptr(), None,
                                                d_o.data_ptr(), d_t.data_ptr(), d_l.data_ptr(), st.cuda_stream),
                          prop.handle)
            e1.record(st)
            torch.cuda.synchronize()
            tl.append(e0.elapsed_time(e1) / 1e3)
        per_mod = d_l.cpu().numpy()
        finite = np.all(np.isfinite(per_mod), axis=0)  # a hit no source can produce gives ln f = -inf
        llh = per_mod[:, finite].sum(axis=1)
        inf = surrogate_inference_rate(0, S * M)
    t_llh = float(np.median(tl[1:]))
    per_hyp = t_llh / H + S * M / inf["queries_per_s"]
    line = {"metric": "event likelihood hypotheses/s (surrogate parameters + FP64 likelihood kernel)",
            "value": 1.0 / per_hyp, "unit": "hypotheses/s", "n_gpus": 1, "higher_is_better": True,
            "data": "synthetic",
            "config": {"workload": f"100 GeV e- cascade, {S} cascade-profile sources x {M} modules, {int(counts.sum())} "
                                   f"observed hits, {H} energy hypotheses per launch (x0.5 .. x2)"},
            "llh_kernel_s_per_launch": t_llh, "llh_hypotheses_per_s": H / t_llh,
            "surrogate_queries_per_hypothesis": S * M, "surrogate_queries_per_s": inf["queries_per_s"],
            "mc_seconds_per_hypothesis": t_mc, "speedup_vs_mc": t_mc / per_hyp,
            "best_scale": float(scales[int(np.argmax(llh))]),
            "modules_with_an_impossible_hit": int((~finite).sum())}
    print(json.dumps(line), flush=True)


def run_reference(args):
    """--impl reference: the reference's algorithm (its FP64 C restatement,
    oracle/) on all host cores, on a bounded sample of the first timed batch of
    the GPU arm; rank 0 alone runs it.  Nothing here imports the product."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    steps, warm = args.steps, args.warmup
    seed = args.seed + warm  # the GPU arm's first timed batch (rank 0)
    arm = CpuArm(seed, args.pairs, RUN_KW, args.max_photons)
    per_step = max(1.0, min(args.cpu_seconds, 90.0 / max(steps + warm, 1)))
    arm.calibrate(per_step)
    photons = []
    times = []
    threads = []
    for i in range(warm + steps):
        ph, dt, used = arm.run()
        if i >= warm:
            photons.append(ph)
            times.append(dt)
            threads.append(used)
    t = sum(times)
    v = sum(photons) / t
    base = arm.describe(photons[-1], statistics.median(times), min(threads))
    base["value"] = v
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
            "steps": steps, "warmup": warm, "ms_per_step": t * 1e3 / steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": bench_config(args.pairs, seed, arm.batch_photons, args.gpus),
            "cpu_baseline": base, "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0,
                                          "d2h_bytes_per_step": 0},
            "step": "one pass over the sample (the first ceil(f N_i) photons of every pair of the batch)",
            "note": "the reference's propagation exists only as a CUDA.jl kernel (Julia is not installed); "
                    "this arm times its FP64 C restatement on the host cores, without the product library"}
    print(json.dumps(line), flush=True)


def plain_by_pair_size(prop, ro, b, d_batch, d_pair_views, h_pairs, d_hits, cap, d_cnt, d_st1, d_hi1, d_stats,
                       d_hist, s, flush):
    """Where the one-pair-per-launch path loses against the batched kernel:
    per-pair device time of the plain path (its memsets, counter reset,
    kernel and finalisation, launched back to back as in the plain pass) and
    the batched kernel on each photon-count decade of the same batch alone,
    photons/s per decade, plus the plain path's fixed cost per pair (the
    median time of the pairs below 2e4 photons)."""
    import torch
    n = np.asarray(b["n_photons"], dtype=np.int64)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(len(b))]
    with torch.cuda.stream(s):
        flush.fill_(3)
    for i in range(len(b)):
        ev[i][0].record(s)
        prop.propagate_plain_device(d_pair_views[i], h_pairs[i], i, ro, d_hits, cap, d_cnt, d_st1, d_hi1, stream=s)
        ev[i][1].record(s)
    s.synchronize()
    t = np.array([a.elapsed_time(e) / 1e3 for a, e in ev])
    out = {"what": "plain: per-pair device time (memsets, reset, kernel, finalisation) summed per decade; batched: "
                   "the decade's pairs as one batched launch",
           "plain_fixed_cost_us_per_pair": float(np.median(t[n < 20000]) * 1e6) if np.any(n < 20000) else None,
           "decades": []}
    for lo, hi in ((1e4, 1e5), (1e5, 1e6), (1e6, 1e7 + 1)):
        sel = np.nonzero((n >= lo) & (n < hi))[0]
        if len(sel) == 0:
            continue
        ph = float(n[sel].sum())
        sub = np.ascontiguousarray(b[sel])
        d_sub = torch.from_numpy(sub.view(np.uint8).copy()).to(d_batch.device)
        for _ in range(2):
            prop.propagate_device(d_sub, len(sel), ro, d_hits, cap, d_cnt, d_stats, d_hist, stream=s)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(s):
            flush.fill_(5)
        e0.record(s)
        prop.propagate_device(d_sub, len(sel), ro, d_hits, cap, d_cnt, d_stats, d_hist, stream=s)
        e1.record(s)
        s.synchronize()
        tb = e0.elapsed_time(e1) / 1e3
        tp = float(t[sel].sum())
        out["decades"].append({"photons": [lo, min(hi, 1e7)], "pairs": int(len(sel)), "photon_share": ph / n.sum(),
                               "plain_photons_per_s": ph / tp, "batched_photons_per_s": ph / tb,
                               "batched_over_plain": tp / tb, "plain_time_share": tp / t.sum()})
    return out


# ---------------------------------------------------------------------------
def run_ours(args):
    import torch
    import torch.distributed as dist

    import photonprop_b200 as pp
    from photonprop_b200 import roofline

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=dev)

    def barrier():
        if world > 1:
            dist.barrier()

    def reduce(x, op):
        if world == 1:
            return x
        t = torch.tensor([float(x)], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=op)
        return float(t.item())

    SUM = dist.ReduceOp.SUM if world > 1 else None
    MAX = dist.ReduceOp.MAX if world > 1 else None

    peaks = pp.measure_peaks(local)
    sol_steps = pp.measure_step_rate(local)
    medium = pp.make_seawater(35.0, 2.0)
    spec = pp.CherenkovSpectrum((300.0, 800.0), 20, medium)
    prop = pp.Propagator(medium, spec, pp.p_one_pmt_acc, device=local)
    ro = pp.RunOptions(**RUN_KW, cascade=args.cascade_variant)
    W, K = args.warmup, args.steps
    batches = [pp.batches.mixed_batch(args.pairs, seed=args.seed + 7919 * rank + i) for i in range(W + K)]
    if args.max_photons > 0:
        for b in batches:
            b["n_photons"] = np.minimum(b["n_photons"], args.max_photons)
    n_pairs = args.pairs
    bins = RUN_KW["hist_bins"]

    tune = None
    if not args.no_tune:
        sample = batches[0][:512].copy()
        sample["n_photons"] = np.minimum(sample["n_photons"], 2_000_000)
        tune = prop.autotune(sample, ro)
        ro.block_size, ro.blocks_per_sm, ro.chunk_photons = (tune["block_size"], tune["blocks_per_sm"],
                                                             tune["chunk_photons"])

    cap = 1 << 22
    d_pairs = [torch.from_numpy(b.view(np.uint8).copy()).to(dev) for b in batches]
    d_hits = torch.empty(cap * 64, dtype=torch.uint8, device=dev)
    d_cnt = torch.zeros(4, dtype=torch.int64, device=dev)
    d_stats = torch.zeros((n_pairs, 8), dtype=torch.float64, device=dev)
    d_hist = torch.zeros((n_pairs, bins), dtype=torch.float64, device=dev)
    cnt_log = torch.zeros((K, 4), dtype=torch.int64, device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)  # > 126 MB L2
    s = torch.cuda.Stream(device=dev)

    for i in range(W):
        prop.propagate_device(d_pairs[i], n_pairs, ro, d_hits, cap, d_cnt, d_stats, d_hist, stream=s)
    s.synchronize()
    barrier()

    uuid = None
    try:
        uuid = str(torch.cuda.get_device_properties(local).uuid)
    except Exception:
        pass
    sampler = ClockSampler(uuid)
    sampler.start()
    time.sleep(0.3)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(K)]
    launches0 = pp.launch_count()
    torch.cuda.synchronize()
    barrier()
    t_wall = time.perf_counter()
    for k in range(K):
        with torch.cuda.stream(s):
            flush.fill_(k & 0xFF)
        ev[k][0].record(s)
        prop.propagate_device(d_pairs[W + k], n_pairs, ro, d_hits, cap, d_cnt, d_stats, d_hist, stream=s)
        ev[k][1].record(s)
        with torch.cuda.stream(s):
            cnt_log[k].copy_(d_cnt)
    s.synchronize()
    torch.cuda.synchronize()
    barrier()
    wall = time.perf_counter() - t_wall
    launches = pp.launch_count() - launches0
    clocks = sampler.stop()

    step_ms = [a.elapsed_time(b) for a, b in ev]
    cnt = cnt_log.cpu().numpy()
    photons_local = [int(batches[W + k]["n_photons"].sum()) for k in range(K)]
    t_local = sum(step_ms) / 1e3
    t_max = reduce(t_local, MAX)
    photons_all = reduce(sum(photons_local), SUM)
    value = photons_all / t_max
    # roofline of the batched launch sequence (the batched kernel is >99.9 % of it)
    iso = [int(batches[W + k]["n_photons"][batches[W + k]["emitter"] == 0].sum()) for k in range(K)]
    cone = [photons_local[k] - iso[k] for k in range(K)]
    steps_total = int(cnt[:, 1].sum())
    mufu, fp32, iops = roofline.op_counts(steps_total, sum(iso), sum(cone), algorithmic=True)
    mufu_i, fp32_i, _ = roofline.op_counts(steps_total, sum(iso), sum(cone), algorithmic=False)
    a_mufu, a_fp32, a_int = mufu / t_local, fp32 / t_local, iops / t_local
    f_mufu, f_fp32 = a_mufu / peaks["mufu_ops"], a_fp32 / peaks["fp32_ops"]
    hits_local = int(cnt[:, 0].sum())
    # algorithmic HBM bytes over the K steps: pairs in, hits out, histograms and statistics zeroed and written,
    # chunk offsets written and read
    alg_bytes = K * (n_pairs * 80 + 2 * n_pairs * (bins + 8) * 8 + 2 * (n_pairs + 1) * 8) + hits_local * 64

    # plain: one launch per pair on the same batch, kernels only (no host sync
    # between pairs) and through the host-buffer API (sync + copy-back per pair)
    plain = None
    if not args.no_plain:
        b = batches[W]
        h_pairs = [b[i:i + 1].copy() for i in range(n_pairs)]
        d_pair_views = [d_pairs[W][i * 80:(i + 1) * 80] for i in range(n_pairs)]
        d_st1 = torch.zeros((1, 8), dtype=torch.float64, device=dev)
        d_hi1 = torch.zeros((1, bins), dtype=torch.float64, device=dev)

        def plain_pass():
            for i in range(n_pairs):
                prop.propagate_plain_device(d_pair_views[i], h_pairs[i], i, ro, d_hits, cap, d_cnt, d_st1, d_hi1,
                                            stream=s)
        plain_pass()  # warm-up
        s.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(s):
            flush.fill_(1)
        e0.record(s)
        plain_pass()
        e1.record(s)
        s.synchronize()
        t_pk = e0.elapsed_time(e1) / 1e3
        hits_np = np.zeros(cap, dtype=pp.HIT_DTYPE)
        st_np = np.zeros((n_pairs, 8))
        hi_np = np.zeros((n_pairs, bins))
        t0 = time.perf_counter()
        prop.propagate_into(b, ro, hits_np, st_np, hi_np, plain=True)
        t_ph = time.perf_counter() - t0
        ph = photons_local[0]
        plain = {"kernel_photons_per_s": reduce(ph, SUM) / reduce(t_pk, MAX),
                 "host_api_photons_per_s": reduce(ph, SUM) / reduce(t_ph, MAX),
                 "launches_per_pass": 3 * n_pairs}
        plain["batched_over_plain_kernel"] = value / plain["kernel_photons_per_s"]
        plain["batched_over_plain_host_api"] = value / plain["host_api_photons_per_s"]
        plain["by_pair_size"] = plain_by_pair_size(prop, ro, b, d_pairs[W], d_pair_views, h_pairs, d_hits, cap,
                                                   d_cnt, d_st1, d_hi1, d_stats, d_hist, s, flush)
        # the reference's own launch shape: cuda_propagate_photons! as propagate_distance launches
        # it (16 blocks x 1024 threads, per-block hit stacks), one pair per launch, on the first
        # 256 pairs of the same batch
        nref, blocks, threads, stack_len = min(256, n_pairs), 16, 1024, 65536
        arrs = pp.initialize_photon_arrays(stack_len, blocks, device=dev)

        def ref_pass():
            for i in range(nref):
                prop.cuda_propagate_photons(*arrs, stack_len, h_pairs[i], ro, threads, stream=s)
        ref_pass()
        s.synchronize()
        e0.record(s)
        ref_pass()
        e1.record(s)
        s.synchronize()
        t_ref = e0.elapsed_time(e1) / 1e3
        # every thread simulates cld(N, blocks x threads) photons, so a launch simulates that many
        # rounds of 16384 photons unless a block's stack fills first (checked on a sample)
        per = blocks * threads
        sim = -(-np.asarray(b["n_photons"][:nref], dtype=np.int64) // per) * per
        full = True
        for i in range(0, nref, 17):
            with torch.cuda.stream(s):
                arrs[5].zero_()  # the kernel adds to the count, like the reference's atomic_add!
            prop.cuda_propagate_photons(*arrs, stack_len, h_pairs[i], ro, threads, stream=s)
            s.synchronize()
            full = full and int(arrs[5][0].item()) == int(sim[i])
        ph_ref = float(sim.sum())
        plain["reference_launch_shape"] = {
            "photons_per_s": ph_ref / t_ref, "pairs": nref, "photons": ph_ref, "all_photons_simulated": full,
            "what": "pp_cuda_propagate_photons per pair, 16 x 1024 threads as propagate_distance launches "
                    "cuda_propagate_photons! (src/photon_prop_cuda.jl:598-606), synchronous per call as there"}
        plain["batched_over_reference_launch_shape"] = value / (ph_ref / t_ref)

    # e2e: the C-ABI host-buffer call, pinned host memory, copies inside the timing
    pin_pairs = [torch.from_numpy(b.view(np.uint8).copy()).pin_memory().numpy().view(pp.PAIR_DTYPE)
                 for b in batches]
    pin_hits = torch.empty(cap * 64, dtype=torch.uint8).pin_memory().numpy().view(pp.HIT_DTYPE)
    pin_stats = torch.empty(n_pairs * 8, dtype=torch.float64).pin_memory().numpy().reshape(n_pairs, 8)
    pin_hist = torch.empty(n_pairs * bins, dtype=torch.float64).pin_memory().numpy().reshape(n_pairs, bins)
    prop.propagate_into(pin_pairs[0], ro, pin_hits, pin_stats, pin_hist)
    barrier()
    e2e_t = 0.0
    d2h = 0
    for k in range(K):
        t0 = time.perf_counter()
        nh, _ = prop.propagate_into(pin_pairs[W + k], ro, pin_hits, pin_stats, pin_hist)
        e2e_t += time.perf_counter() - t0
        d2h += 32 + min(nh, cap) * 64 + n_pairs * 8 * 8 + n_pairs * bins * 8
    e2e_value = photons_all / reduce(e2e_t, MAX)

    surrogate_inf = surrogate_inference_rate(local)

    # serving: the configured stream (Poisson 200 req/s) and an overload sample where the one-launch-
    # per-request loop saturates; one GPU only (the scaling runs measure the batch)
    serve = None
    if args.serving_seconds > 0 and world == 1:
        serve = {"configured": run_serving(prop, args.serving_seconds, seed=args.seed + rank,
                                           rate_hz=args.serving_rate)}
        if args.overload_seconds > 0:
            serve["overload"] = run_serving(prop, args.overload_seconds, seed=args.seed + 17 + rank,
                                            rate_hz=args.overload_rate)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(args.seed + W, n_pairs, args.cpu_seconds, RUN_KW, args.max_photons)
        from oracle import batches as ob
        ob_batch = ob.mixed_batch(n_pairs, seed=args.seed + W)
        if args.max_photons > 0:
            ob_batch["n_photons"] = np.minimum(ob_batch["n_photons"], args.max_photons)
        cpu["same_batch_as_gpu"] = bool(np.array_equal(ob_batch["n_photons"], batches[W]["n_photons"])
                                        and np.array_equal(ob_batch["seed"], batches[W]["seed"])
                                        and np.array_equal(ob_batch["target"], batches[W]["target"]))

    lat = sorted(step_ms)
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": K, "warmup": W,
        "ms_per_step": reduce(t_local, MAX) * 1e3 / K, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": bench_config(n_pairs, args.seed + 7919 * rank + W, photons_local[0], world),
        "launch": {"block": ro.block_size, "blocks_per_sm": ro.blocks_per_sm, "chunk_photons": ro.chunk_photons,
                   "autotuned": tune is not None,
                   "kernel_variant": "cascade emitter" if args.cascade_variant else "basic emitters"},
        "timing": "CUDA events per step on the launch stream, summed; max over ranks; L2 flushed between steps "
                  "(256 MiB write outside the per-step events)",
        "latency_ms": {"p50": statistics.median(lat), "p99": lat[min(len(lat) - 1, int(0.99 * len(lat)))],
                       "what": "device time of one 4096-pair batch solve"},
        "roofline": {"bound": "mufu", "achieved": a_mufu / 1e9, "peak": peaks["mufu_ops"] / 1e9,
                     "unit": "Gop/s", "frac": f_mufu,
                     "traffic": roofline.NCU_DRAM_BYTES_PER_LAUNCH,
                     "traffic_note": "dram__bytes_read.sum + dram__bytes_write.sum of a full-size launch of this "
                                     "workload (ncu, one pass, mean of two timed launches after an L2 flush); the "
                                     "histograms and hits accumulate in L2 and reach DRAM after the launch",
                     "issue_active_ncu": roofline.NCU_ISSUE_ACTIVE,
                     "lanes_active_ncu": roofline.NCU_LANES_ACTIVE,
                     "note": "issue-bound: ncu shows {:.0%} of issue slots busy (ALU pipe {:.0%}, FMA {:.0%}, XU {:.0%})".format(
                         roofline.NCU_ISSUE_ACTIVE, roofline.NCU_PIPES["alu"], roofline.NCU_PIPES["fma"],
                         roofline.NCU_PIPES["xu"]),
                     "peak_source": "measured live: ex2.approx dependent chains over every SM (pp_measure_peaks)",
                     "counts": "achieved = algorithmic MUFU operations (the reference's arithmetic: 7 per photon "
                               "step, 10 per isotropic / 14 per cone photon start) per second; 'issued' = this "
                               "kernel's own count (7 MUFU and 46 FP32 per step, ncu opcode counts)",
                     "issued": {"mufu_achieved": mufu_i / t_local / 1e9,
                                "mufu_frac": mufu_i / t_local / peaks["mufu_ops"],
                                "fp32_frac": fp32_i / t_local / peaks["fp32_ops"]},
                     "fp32": {"achieved": a_fp32 / 1e9, "peak": peaks["fp32_ops"] / 1e9, "frac": f_fp32},
                     "philox": {"achieved_blocks_per_s": a_int, "peak_blocks_per_s": peaks["philox_blocks"],
                                "frac": a_int / peaks["philox_blocks"]},
                     "photon_steps_per_s": steps_total / t_local,
                     "steps_per_photon": steps_total / max(sum(photons_local), 1),
                     "step_speed_of_light": {
                         "steps_per_s": sol_steps,
                         "what": "bare physical step on every SM (Philox block, ray-sphere, move, turn; no emission, "
                                 "refill, hits or loop bookkeeping), pp_measure_step_rate",
                         "mufu_frac_ceiling": roofline.MUFU_PER_STEP_ALG * sol_steps / peaks["mufu_ops"],
                         "mufu_frac_ceiling_issued": roofline.MUFU_PER_STEP * sol_steps / peaks["mufu_ops"],
                         "batched_steps_frac": steps_total / t_local / sol_steps,
                         "frac_of_ceiling": f_mufu / (roofline.MUFU_PER_STEP_ALG * sol_steps / peaks["mufu_ops"])},
                     "hbm": {"achieved_gbs": alg_bytes / t_local / 1e9, "peak_gbs": measured_hbm_gbs(),
                             "frac": alg_bytes / t_local / 1e9 / measured_hbm_gbs(),
                             "algorithmic_bytes_per_step": alg_bytes / K,
                             "what": "algorithmic HBM bytes of a step: pair records read (80 B each), hit records "
                                     "written (64 B each), the FP64 histograms and statistics written (zeroed, then "
                                     "the accumulated table), the work-queue offsets written and read",
                             "peak_source": "MEASURED_PEAKS.json hbm_gbs (else 6650 GB/s, an earlier measurement "
                                            "on this pool)"}},
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": n_pairs * 80,
                "d2h_bytes_per_step": int(d2h / K)},
        "plain": plain,
        "serving": serve,
        "surrogate_inference": surrogate_inf,
        "cpu_baseline": cpu,
        "clocks": clocks,
        "gpu_launches": launches,
        "wall_s": wall,
        "hits_per_step": hits_local / K,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    prop.close()
    if world > 1:
        dist.destroy_process_group()


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "serving":
        run_serving_workload(args)
    elif args.workload == "surrogate":
        run_surrogate_workload(args)
    elif args.workload == "cone-grid":
        run_cone_grid(args)
    elif args.workload == "point":
        run_point(args)
    elif args.workload == "fits":
        run_fits(args)
    elif args.workload == "event":
        run_event(args)
    elif args.workload == "llh":
        run_llh(args)
    elif args.workload == "large-pairs":
        run_large_pairs(args)
    elif args.workload == "surrogate-infer":
        import torch
        torch.cuda.set_device(0)
        print(json.dumps({"metric": "surrogate inference queries/s (untrained weights)",
                          **surrogate_inference_rate(0, 1_000_000)}), flush=True)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()

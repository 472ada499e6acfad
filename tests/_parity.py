"""Shared checks of the CUDA path against the FP64 oracle (test helpers)."""
import numpy as np

from oracle import oracle as O


def to_oracle_pairs(pairs):
    p = np.asarray(pairs)
    o = O.pairs_array(len(p))
    for f in ("pos", "t0", "dir", "track_len", "target", "radius", "n_photons", "seed", "emitter"):
        o[f] = p[f]
    return o


def to_oracle_opts(ro):
    """oracle Opts from a photonprop RunOptions (through its C struct)."""
    c = ro.to_c()
    return O.make_opts(mode=c.mode, max_steps=c.max_steps, g=float(np.float32(c.g)), t_max=float(c.t_max),
                       hist_t0=float(c.hist_t0), hist_bin_width=float(c.hist_bin_width), hist_bins=c.hist_bins,
                       flags=c.flags & 3)


def match_hits(gpu_hits, orc_hits):
    """Joins hits on (pair, photon).  Returns (gpu_matched, orc_matched,
    n_gpu_only, n_orc_only)."""
    gk = {(int(h["pair"]), int(h["photon"])): i for i, h in enumerate(gpu_hits)}
    ok = {(int(h["pair"]), int(h["photon"])): i for i, h in enumerate(orc_hits)}
    both = sorted(set(gk) & set(ok))
    gi = np.array([gk[k] for k in both], dtype=np.int64)
    oi = np.array([ok[k] for k in both], dtype=np.int64)
    return gpu_hits[gi], orc_hits[oi], len(gk) - len(both), len(ok) - len(both)


def per_photon_errors(g, o):
    """Absolute position / time errors and relative weight error of matched hits."""
    dpos = np.linalg.norm(g["pos"].astype(np.float64) - o["pos"], axis=1)
    dt = np.abs(g["time"].astype(np.float64) - o["time"])
    dw = np.abs(g["weight"].astype(np.float64) - o["weight"]) / np.maximum(o["weight"], 1e-30)
    dwl = np.abs(g["wavelength"].astype(np.float64) - o["wavelength"]) / o["wavelength"]
    dd0 = np.linalg.norm(g["dir0"].astype(np.float64) - o["dir0"], axis=1)
    ddir = np.linalg.norm(g["dir"].astype(np.float64) - o["dir"], axis=1)
    dnorm = np.abs(np.linalg.norm(g["dir"].astype(np.float64), axis=1) - 1.0)
    ddist = np.abs(g["dist"].astype(np.float64) - o["dist"])
    return {"pos": dpos, "time": dt, "weight": dw, "wavelength": dwl, "dir0": dd0, "dir": ddir, "dir_norm": dnorm,
            "dist": ddist}


def summary(err):
    return {k: (float(v.max()) if len(v) else 0.0, float(np.percentile(v, 99)) if len(v) else 0.0)
            for k, v in err.items()}


def chi2_two_sample(a, b, min_count=10):
    """Two-sample chi-square on histograms of counts (Press et al. 14.3),
    merging adjacent bins until each merged bin has min_count entries in
    total.  Returns (chi2, dof, p)."""
    from scipy import stats as st
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    ra, rb = [], []
    ca = cb = 0.0
    for x, y in zip(a, b):
        ca += x
        cb += y
        if ca + cb >= min_count:
            ra.append(ca)
            rb.append(cb)
            ca = cb = 0.0
    if ca + cb > 0 and ra:
        ra[-1] += ca
        rb[-1] += cb
    ra, rb = np.array(ra), np.array(rb)
    na, nb = ra.sum(), rb.sum()
    ka, kb = np.sqrt(nb / na), np.sqrt(na / nb)
    chi2 = float(np.sum((ka * ra - kb * rb) ** 2 / (ra + rb)))
    dof = len(ra) - 1
    return chi2, dof, float(st.chi2.sf(chi2, dof))


def check_matched(g, o, n_gpu_only, n_orc_only, label, flip_frac=0.01, flip_abs=3):
    """Per-photon tolerances of matched hits (GPU FP32 against the FP64 oracle
    on the same Philox numbers):  |d pos| <= 2e-3 m + 2e-5 path,
    |d t| <= 1e-2 ns + 1e-5 t, |d w| <= 1e-3 w + 1e-8, |d lambda| / lambda <= 1e-5,
    arrival direction |d dir| <= 1e-3 with | |dir| - 1 | <= 1e-5 (the
    physical-mode turn is not renormalised: its norm error must stay
    bounded); photons detected on one side only (sphere-rim flips) <=
    flip_frac of the hits + flip_abs."""
    err = per_photon_errors(g, o)
    s = summary(err)
    print(label, "matched", len(g), "gpu-only", n_gpu_only, "oracle-only", n_orc_only, s)
    n = max(len(g), 1)
    assert n_gpu_only + n_orc_only <= flip_frac * n + flip_abs, (label, n_gpu_only, n_orc_only, len(g))
    path = o["dist"]
    assert np.all(err["pos"] <= 2e-3 + 2e-5 * path), (label, s["pos"])
    assert np.all(err["time"] <= 1e-2 + 1e-5 * o["time"]), (label, s["time"])
    # relative 1e-3, plus an absolute floor where the PMT acceptance tends to zero
    assert np.all(np.abs(g["weight"] - o["weight"]) <= 1e-3 * o["weight"] + 1e-8), (label, s["weight"])
    assert np.all(err["wavelength"] <= 1e-5), (label, s["wavelength"])
    assert np.all(err["dir"] <= 1e-3), (label, s["dir"])
    assert np.all(err["dir_norm"] <= 1e-5), (label, s["dir_norm"])
    return s


def _split(gpu_hits, orc_hits):
    gk = {(int(h["pair"]), int(h["photon"])): i for i, h in enumerate(gpu_hits)}
    ok = {(int(h["pair"]), int(h["photon"])): i for i, h in enumerate(orc_hits)}
    both = sorted(set(gk) & set(ok))
    g_only = np.array(sorted(gk[k] for k in set(gk) - set(ok)), dtype=np.int64)
    o_only = np.array(sorted(ok[k] for k in set(ok) - set(gk)), dtype=np.int64)
    gi = np.array([gk[k] for k in both], dtype=np.int64)
    oi = np.array([ok[k] for k in both], dtype=np.int64)
    return gi, oi, g_only, o_only


def check_pair_statistics_and_histograms(gpu_res, orc_hits, orc_stats, orc_hist, n_pairs, t0, width, bins,
                                         label, edge_ns=1e-2):
    """Reconciles the kernel's FP64 per-pair sums and arrival-time histograms
    with the oracle's, bin by bin.  The oracle's table, with its one-sided
    photons (rim flips) replaced by the GPU's and any matched photon whose
    time lies within edge_ns of a bin edge moved to the GPU's bin, must equal
    the GPU's: hit counts exactly, weights to 2e-3 relative."""
    gh = gpu_res.hits
    gi, oi, g_only, o_only = _split(gh, orc_hits)
    g_t = gh["time"].astype(np.float64)
    g_w = gh["weight"].astype(np.float64)
    g_p = gh["pair"].astype(np.int64)
    o_t, o_w, o_p = orc_hits["time"], orc_hits["weight"], orc_hits["pair"].astype(np.int64)

    def bin_of(t):
        return np.floor((t - t0) / width)

    exp_hist = orc_hist.copy()
    exp_cnt = orc_stats[:, 0].copy()
    exp_w = orc_stats[:, 1].copy()

    def add(p, t, w, sign):
        b = bin_of(t)
        inside = (b >= 0) & (b < bins)
        np.add.at(exp_hist, (p[inside], b[inside].astype(np.int64)), sign * w[inside])

    add(o_p[o_only], o_t[o_only], o_w[o_only], -1.0)
    add(g_p[g_only], g_t[g_only], g_w[g_only], +1.0)
    np.add.at(exp_cnt, o_p[o_only], -1.0)
    np.add.at(exp_cnt, g_p[g_only], +1.0)
    np.add.at(exp_w, o_p[o_only], -o_w[o_only])
    np.add.at(exp_w, g_p[g_only], +g_w[g_only])
    moved = bin_of(g_t[gi]) != bin_of(o_t[oi])
    if np.any(moved):
        tt = o_t[oi][moved]
        edge = t0 + width * np.round((tt - t0) / width)
        assert np.all(np.abs(tt - edge) <= edge_ns), (label, "bin differs away from an edge")
        add(o_p[oi][moved], o_t[oi][moved], o_w[oi][moved], -1.0)
        add(g_p[gi][moved], g_t[gi][moved], g_w[gi][moved], +1.0)
    s = gpu_res.stats
    np.testing.assert_array_equal(s[:, 0], exp_cnt, err_msg=label)
    np.testing.assert_allclose(s[:, 1], exp_w, rtol=2e-3, atol=1e-12, err_msg=label)
    np.testing.assert_allclose(gpu_res.hist[:, :bins], exp_hist, rtol=2e-3, atol=1e-12, err_msg=label)
    return int(np.count_nonzero(moved))

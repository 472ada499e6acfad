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
    ddist = np.abs(g["dist"].astype(np.float64) - o["dist"])
    return {"pos": dpos, "time": dt, "weight": dw, "wavelength": dwl, "dir0": dd0, "dist": ddist}


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

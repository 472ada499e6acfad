"""Learned surrogate of the photon propagation (replaces the reference's Flux
MLP fits, src/modelling.jl:113-299).

Query features (raw): log10 distance (m), cos of the angle between the
emitter axis and the emitter->target direction, log10 photon count, emitter
flag (0 isotropic, 1 Cherenkov cone).  Outputs: ln(mu/N) with mu the expected
weighted hits (absorption x PMT), and a two-component Gamma mixture
w G(a1, theta) + (1 - w) G(a2, theta) of the arrival-time residual
t - t_geo, t_geo = (d - r) n_g(800 nm) / c (the reference fits a Gamma to the
same kind of residual, src/modelling.jl:52-79 with src/photon_prop_cuda.jl:639-640),
stored as (logit w, ln a1, ln a2, ln theta).

The network (MLP 4 -> 128 -> 128 -> 128 -> 5, GELU) is trained and run by the
library's own kernels (pp_mlp_*): BF16 weights and activations, FP32
accumulation, tcgen05 tensor cores for the 128 x 128 layers, hand-written
backward and Adam.  Training pairs come from the MC kernel
(pp_propagate_device) with targets from the library's Gamma-mixture EM kernel.
Queries outside the trained feature range fall back to the MC kernel.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from . import _lib
from .batches import mixed_batch
from .medium import get_group_index
from .propagation import Propagator, RunOptions

C_VACUUM_M_PER_NS = 0.299792458
N_OUT = 5


class MLP:
    """The library's surrogate network on one device."""

    def __init__(self, device=0, seed=0):
        self._L = _lib.load()
        h = ctypes.c_void_p()
        _lib.check(self._L.pp_mlp_create(device, seed, ctypes.byref(h)))
        self._h = h
        self.device = device
        self.n_params = int(self._L.pp_mlp_num_params())

    def close(self):
        if getattr(self, "_h", None):
            self._L.pp_mlp_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, st):
        if st != _lib.PP_OK:
            raise _lib.PPError(st, (self._L.pp_mlp_last_error(self._h) or b"").decode())

    def get_params(self) -> np.ndarray:
        p = np.zeros(self.n_params, dtype=np.float32)
        self._check(self._L.pp_mlp_get_params(self._h, p.ctypes.data))
        return p

    def set_params(self, p):
        p = np.ascontiguousarray(p, dtype=np.float32)
        assert p.size == self.n_params
        self._check(self._L.pp_mlp_set_params(self._h, p.ctypes.data))

    def set_normalization(self, x_mean, x_std, y_mean, y_std):
        arr = [np.ascontiguousarray(a, dtype=np.float32) for a in (x_mean, x_std, y_mean, y_std)]
        self._check(self._L.pp_mlp_set_normalization(self._h, *[a.ctypes.data for a in arr]))

    def get_normalization(self):
        out = np.zeros(18, dtype=np.float32)
        self._check(self._L.pp_mlp_get_normalization(self._h, out.ctypes.data))
        return out[0:4], out[4:8], out[8:13], out[13:18]

    def forward(self, d_x, d_out, n, physical=False, stream=None):
        """Device inference: d_x [n, 4] raw features -> d_out [5, n] (torch tensors)."""
        s = getattr(stream, "cuda_stream", stream)
        self._check(self._L.pp_mlp_forward(self._h, d_x.data_ptr(), d_out.data_ptr(), n, int(physical), s))

    def train_step(self, d_xn, d_yt, d_mask, n, lr, want_grads=False):
        loss = ctypes.c_float()
        g = np.zeros(self.n_params, dtype=np.float32) if want_grads else None
        self._check(self._L.pp_mlp_train_step(self._h, d_xn.data_ptr(), d_yt.data_ptr(), d_mask.data_ptr(), n,
                                              float(lr), ctypes.byref(loss), g.ctypes.data if want_grads else None))
        return float(loss.value), g


def gemm_selftest(a_bf16_u16, b_bf16_u16, device=0):
    """c = a b^T through the tcgen05 path (a, b uint16 BF16 bit patterns [128,128])."""
    L = _lib.load()
    a = np.ascontiguousarray(a_bf16_u16, dtype=np.uint16)
    b = np.ascontiguousarray(b_bf16_u16, dtype=np.uint16)
    c = np.zeros((128, 128), dtype=np.float32)
    _lib.check(L.pp_mlp_gemm_selftest(device, a.ctypes.data, b.ctypes.data, c.ctypes.data))
    return c


def features(pairs) -> np.ndarray:
    """[n, 4] raw features of pairs: log10 d, cos angle, log10 N, emitter flag
    (0 isotropic, 1 Cherenkov cone, 2 cascade profile: outside the trained
    range, so the MC kernel answers)."""
    p = np.asarray(pairs)
    pos = p["pos"].astype(np.float64)
    d = p["dir"].astype(np.float64)
    cone = p["emitter"] == _lib.EMITTER_CHERENKOV_CONE
    src = pos + np.where(cone[:, None], 0.5 * p["track_len"][:, None] * d, 0.0)
    v = p["target"].astype(np.float64) - src
    dist = np.linalg.norm(v, axis=1)
    cosang = np.einsum("ij,ij->i", v / dist[:, None], d)
    flag = np.where(p["emitter"] == _lib.EMITTER_CASCADE, 2.0, cone.astype(np.float64))
    return np.stack([np.log10(dist), cosang, np.log10(np.maximum(p["n_photons"], 1)), flag],
                    axis=1).astype(np.float32)


def time_shift(pairs, medium) -> np.ndarray:
    """t_geo = (d - r) n_g(800 nm) / c for each pair (ns)."""
    f = features(pairs)
    d = 10.0 ** f[:, 0].astype(np.float64)
    ng = float(get_group_index(800.0, medium))
    return ((d - np.asarray(pairs["radius"], dtype=np.float64)) * ng / C_VACUUM_M_PER_NS).astype(np.float32)


@dataclass
class Dataset:
    x: np.ndarray      # [n, 4] raw features
    y: np.ndarray      # [n, 5] raw targets (ln(mu/N), logit w, ln a1, ln a2, ln theta)
    mask: np.ndarray   # [n, 5] 1 where the target is measured well enough to learn
    hits: np.ndarray   # [n] detected photons (unweighted)
    mu: np.ndarray     # [n] sum of weights
    sigma_mu: np.ndarray  # [n] statistical error of mu: sqrt(sum of squared weights)
    hist: np.ndarray | None = None    # [n, bins] arrival-time histograms (return_hist=True)
    tshift: np.ndarray | None = None  # [n] t_geo of each pair (ns)

    def subset(self, idx):
        return Dataset(self.x[idx], self.y[idx], self.mask[idx], self.hits[idx], self.mu[idx], self.sigma_mu[idx],
                       None if self.hist is None else self.hist[idx],
                       None if self.tshift is None else self.tshift[idx])


def mc_dataset(prop: Propagator, pairs, opts: RunOptions, min_hits_mu=1, min_hits_fit=1000, chunk=20000,
               fit_iters=60, full_weight_hits=100.0, return_hist=False) -> Dataset:
    """Propagates the pairs (MC kernel, histograms only) and turns their
    statistics and histograms into targets."""
    import torch
    dev = torch.device("cuda", prop.device)
    c = opts.to_c()
    bins = c.hist_bins
    cols = {k: [] for k in ("x", "y", "m", "h", "mu", "sg", "hist", "ts")}
    o = RunOptions(**{**opts.__dict__})
    o.write_hits = False
    o.cascade = o.cascade or bool(np.any(np.asarray(pairs["emitter"]) == _lib.EMITTER_CASCADE))
    for s0 in range(0, len(pairs), chunk):
        b = np.ascontiguousarray(pairs[s0:s0 + chunk])
        n = len(b)
        d_pairs = torch.from_numpy(b.view(np.uint8).copy()).to(dev)
        d_cnt = torch.zeros(4, dtype=torch.int64, device=dev)
        d_stats = torch.zeros((n, 8), dtype=torch.float64, device=dev)
        d_hist = torch.zeros((n, bins), dtype=torch.float64, device=dev)
        d_hits = torch.zeros(64, dtype=torch.uint8, device=dev)
        prop.propagate_device(d_pairs, n, o, d_hits, 0, d_cnt, d_stats, d_hist)
        d_ts = torch.from_numpy(time_shift(b, prop.medium)).to(dev)
        d_fit = torch.zeros((n, 5), dtype=torch.float32, device=dev)
        torch.cuda.synchronize(dev)
        _lib.check(_lib.load().pp_gamma_mixture_fit(d_hist.data_ptr(), n, bins, float(c.hist_t0),
                                                    float(c.hist_bin_width), d_ts.data_ptr(), d_fit.data_ptr(),
                                                    fit_iters, None))
        torch.cuda.synchronize(dev)
        st = d_stats.cpu().numpy()
        fit = d_fit.cpu().numpy().astype(np.float64)
        nh, mu, N = st[:, 0], st[:, 1], np.asarray(b["n_photons"], dtype=np.float64)
        with np.errstate(divide="ignore", invalid="ignore"):
            w = np.clip(fit[:, 0], 1e-4, 1 - 1e-4)
            y = np.stack([np.log(np.maximum(mu, 1e-30) / N), np.log(w / (1 - w)), np.log(fit[:, 1]),
                          np.log(fit[:, 2]), np.log(fit[:, 3])], axis=1)
        good_fit = (nh >= min_hits_fit) & np.all(np.isfinite(y[:, 1:]), axis=1)
        m = np.zeros_like(y)
        # loss weight of ln(mu/N): its Poisson variance is ~1/hits, so pairs with
        # few hits count less (full weight from full_weight_hits hits)
        m[:, 0] = np.where(nh >= max(min_hits_mu, 1), np.minimum(nh / full_weight_hits, 1.0), 0.0)
        m[:, 1] = good_fit
        m[:, 2] = good_fit & (w > 0.02)  # a component's shape is only measured if it carries weight
        m[:, 3] = good_fit & (w < 0.98)
        m[:, 4] = good_fit
        y = np.where(m > 0, y, 0.0)
        cols["x"].append(features(b))
        cols["y"].append(y.astype(np.float32))
        cols["m"].append(m.astype(np.float32))
        cols["h"].append(nh)
        cols["mu"].append(mu)
        cols["sg"].append(np.sqrt(st[:, 2]))
        if return_hist:
            cols["hist"].append(d_hist.cpu().numpy())
            cols["ts"].append(d_ts.cpu().numpy())
    ds = Dataset(*(np.concatenate(cols[k]) for k in ("x", "y", "m", "h", "mu", "sg")))
    if return_hist:
        ds.hist = np.concatenate(cols["hist"])
        ds.tshift = np.concatenate(cols["ts"])
    return ds


def training_pairs(n_pairs, photons, seed=0, d_min=2.0, d_max=150.0, distance_law="uniform"):
    """The mixed-batch geometry with a fixed photon count per pair."""
    b = mixed_batch(n_pairs, seed=seed, d_min=d_min, d_max=d_max, distance_law=distance_law)
    b["n_photons"] = int(photons)
    return b


# ---- trained-network files (the reference keeps its network in
# photon_model.bson, example_full.jl:175-178) ------------------------------
WEIGHTS_MAGIC = b"PPSURR01"


def write_weights(path, params, norm18, lo, hi):
    """Writes a trained network: the magic, int32 version 1, int32 parameter
    count, int32 inputs (4), int32 outputs (5), then little-endian FP32 arrays:
    the trained feature range lo[4], hi[4], the normalisation (x mean[4],
    x std[4], y mean[5], y std[5]) and the parameters in pp_mlp_get_params
    order."""
    params = np.ascontiguousarray(params, dtype="<f4").ravel()
    norm18 = np.ascontiguousarray(norm18, dtype="<f4").ravel()
    lo = np.ascontiguousarray(lo, dtype="<f4").ravel()
    hi = np.ascontiguousarray(hi, dtype="<f4").ravel()
    if norm18.size != 18 or lo.size != 4 or hi.size != 4:
        raise ValueError("need 18 normalisation values and a 4-feature range")
    with open(path, "wb") as f:
        f.write(WEIGHTS_MAGIC)
        f.write(np.array([1, params.size, 4, N_OUT], dtype="<i4").tobytes())
        for arr in (lo, hi, norm18, params):
            f.write(arr.tobytes())


def read_weights(path, n_params=None):
    """(params, norm18, lo, hi) of a file written by write_weights; ValueError
    for anything else (wrong magic or version, sizes that do not match the
    file or, when given, n_params)."""
    with open(path, "rb") as f:
        blob = f.read()
    if len(blob) < 24 or blob[:8] != WEIGHTS_MAGIC:
        raise ValueError(f"{path}: not a surrogate weights file")
    version, n, n_in, n_out = np.frombuffer(blob, dtype="<i4", count=4, offset=8).tolist()
    if version != 1 or n_in != 4 or n_out != N_OUT or n < 1 or (n_params is not None and n != n_params):
        raise ValueError(f"{path}: version {version}, {n} parameters, {n_in} -> {n_out} does not fit this network")
    if len(blob) != 24 + 4 * (26 + n):
        raise ValueError(f"{path}: {len(blob)} bytes, expected {24 + 4 * (26 + n)}")
    v = np.frombuffer(blob, dtype="<f4", offset=24).astype(np.float32)
    return v[26:].copy(), v[8:26].copy(), v[0:4].copy(), v[4:8].copy()


class Surrogate:
    """Trained network + its feature range; predict() answers queries inside
    the range with the network and the rest with the MC kernel."""

    def __init__(self, prop: Propagator, opts: RunOptions, device=0, seed=0):
        self.prop, self.opts = prop, opts
        self.net = MLP(device, seed)
        self.lo = None
        self.hi = None

    def save(self, path):
        """Writes the trained network and its feature range (write_weights)."""
        if self.lo is None:
            raise ValueError("the surrogate is not trained")
        xm, xs, ym, ys = self.net.get_normalization()
        write_weights(path, self.net.get_params(), np.concatenate([xm, xs, ym, ys]), self.lo, self.hi)

    @classmethod
    def load(cls, prop: Propagator, opts: RunOptions, path, device=0):
        """A surrogate with the network of a file written by save(): the same
        answers as the network that was saved, without training."""
        s = cls(prop, opts, device=device)
        params, norm, lo, hi = read_weights(path, s.net.n_params)
        s.net.set_params(params)
        s.net.set_normalization(norm[0:4], norm[4:8], norm[8:13], norm[13:18])
        s.lo, s.hi = lo.astype(np.float64), hi.astype(np.float64)
        return s

    def fit(self, data: Dataset, epochs=60, batch=4096, lr=1e-3, seed=0, log=None, lr_min=1e-5):
        """Adam with a cosine learning-rate decay from lr to lr_min."""
        import torch
        dev = torch.device("cuda", self.net.device)
        x, y, m = data.x, data.y, data.mask
        xm, xs = x.mean(0), x.std(0)
        # a feature without spread in the training set is made inert (the photon
        # count: ln(mu/N) does not depend on N, and mu = N exp(out0) scales exactly)
        xs = np.where(xs < 1e-6, 1e30, xs).astype(np.float32)
        ym = np.array([(y[:, j] * m[:, j]).sum() / max(m[:, j].sum(), 1) for j in range(N_OUT)], dtype=np.float32)
        ys = np.array([np.sqrt(((y[:, j] - ym[j]) ** 2 * m[:, j]).sum() / max(m[:, j].sum(), 1)) + 1e-6
                       for j in range(N_OUT)], dtype=np.float32)
        self.net.set_normalization(xm, xs, ym, ys)
        lo, hi = x.min(0), x.max(0)
        lo[2], hi[2] = 4.0, 7.0  # ln(mu/N) does not depend on N: any photon count of the query range
        self.lo, self.hi = lo, hi
        xn = torch.from_numpy(((x - xm) / xs).astype(np.float32)).to(dev)
        yn = torch.from_numpy(np.where(m > 0, (y - ym) / ys, 0.0).astype(np.float32)).to(dev)
        mk = torch.from_numpy(m).to(dev)
        rng = np.random.default_rng(seed)
        n = len(x)
        losses = []
        for ep in range(epochs):
            lr_e = lr_min + 0.5 * (lr - lr_min) * (1.0 + np.cos(np.pi * ep / max(epochs, 1)))
            perm = torch.from_numpy(rng.permutation(n)).to(dev)
            tot, nb = 0.0, 0
            for s in range(0, n - batch + 1, batch):
                idx = perm[s:s + batch]
                loss, _ = self.net.train_step(xn[idx].contiguous(), yn[idx].contiguous(), mk[idx].contiguous(),
                                              batch, lr_e)
                tot += loss
                nb += 1
            losses.append(tot / max(nb, 1))
            if log:
                log(ep, losses[-1])
        return losses

    def in_range(self, x):
        return np.all((x >= self.lo) & (x <= self.hi), axis=1)

    def predict_features(self, x, physical=True):
        """Network outputs [n, 5] for raw features x [n, 4] (device round trip)."""
        import torch
        dev = torch.device("cuda", self.net.device)
        n = len(x)
        d_x = torch.from_numpy(np.ascontiguousarray(x, dtype=np.float32)).to(dev)
        d_o = torch.empty((N_OUT, n), dtype=torch.float32, device=dev)
        self.net.forward(d_x, d_o, n, physical)
        return d_o.cpu().numpy().T.copy()

    def predict(self, pairs):
        """(mu, w, a1, a2, theta) per pair: the network inside the trained range,
        the MC kernel (and the EM fit) outside it.  Returns (out, used_mc)."""
        pairs = np.ascontiguousarray(pairs)
        x = features(pairs)
        ok = self.in_range(x)
        out = np.zeros((len(x), N_OUT))
        if ok.any():
            out[ok] = self.predict_features(x[ok], physical=True)
        if (~ok).any():
            mc = mc_dataset(self.prop, np.ascontiguousarray(pairs[~ok]), self.opts, min_hits_mu=0, min_hits_fit=0)
            y = mc.y.astype(np.float64)
            out[~ok] = np.stack([mc.mu, 1 / (1 + np.exp(-y[:, 1])), np.exp(y[:, 2]), np.exp(y[:, 3]),
                                 np.exp(y[:, 4])], axis=1)
        return out, ~ok

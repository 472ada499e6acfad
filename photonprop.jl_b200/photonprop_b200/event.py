"""Event likelihood of example_full.jl:338-449 (poisson_dist_per_module,
shape_mixture_per_module, extended_llh_per_module) on the device, and the
inputs it takes: the reference's model features (Modelling.source_to_input,
src/modelling.jl:269-289), per-(source, module) parameters from the learned
surrogate, and observed hit times from an MC event.

Parameters per (hypothesis, module, source) are (A, w, alpha1, alpha2,
theta, t_shift): expected photons A x N_source and the arrival-time density
w Gamma(x - t_shift; alpha1, theta) + (1 - w) Gamma(x - t_shift; alpha2,
theta).  The reference's model gives (det_fraction, 1, alpha, -, theta, 0)
with the residual times of its fit table; mode "reference" weighs the
sources of a module by det_fraction alone, as shape_mixture_per_module
does; mode "shifted" weighs them by their expected photons.
"""
from __future__ import annotations

import numpy as np

from . import _lib
from .medium import get_group_index
from .surrogate import C_VACUUM_M_PER_NS, features

_MODES = {"reference": _lib.LLH_REFERENCE, "shifted": _lib.LLH_SHIFTED}


def source_to_input(sources, targets):
    """Modelling.source_to_input(sources, targets), src/modelling.jl:269-289:
    [2, n_sources * n_targets] Float32 features (log10 distance, cos of the
    observation angle) in the reference's product order (targets inner).
    sources: pp_pair records (pos, dir); targets: (x, y, z[, r]) rows.  As in
    the reference the emitter-receiver vector points from the target to the
    source."""
    src = np.asarray(sources)
    tg = np.asarray(targets, dtype=np.float64)[:, :3]
    v = src["pos"].astype(np.float64)[:, None, :] - tg[None, :, :]
    dist = np.linalg.norm(v, axis=2)
    cosang = np.einsum("stk,sk->st", v / dist[..., None], src["dir"].astype(np.float64))
    return np.stack([np.log10(dist).ravel(), cosang.ravel()]).astype(np.float32)


def event_llh(propagator, params, hit_times, source_photons=None, mode="shifted"):
    """Extended log-likelihood per (hypothesis, module) on the device.
    params [n_hyp, n_modules, n_sources, 6]; hit_times: a list of n_modules
    arrays; source_photons [n_hyp, n_sources] or None.  Returns [n_hyp, n_modules]."""
    import torch
    dev = torch.device("cuda", propagator.device)
    p = np.ascontiguousarray(params, dtype=np.float64)
    if p.ndim == 3:
        p = p[None]
    H, M, S, _ = p.shape
    counts = np.array([len(t) for t in hit_times], dtype=np.int64)
    assert len(counts) == M
    offs = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
    times = np.concatenate([np.asarray(t, dtype=np.float64) for t in hit_times]) if offs[-1] else np.zeros(1)
    d_p = torch.from_numpy(p).to(dev)
    d_n = torch.from_numpy(np.ascontiguousarray(source_photons, dtype=np.float64).reshape(H, S)).to(dev) \
        if source_photons is not None else None
    d_o = torch.from_numpy(offs).to(dev)
    d_t = torch.from_numpy(times).to(dev)
    d_l = torch.zeros((H, M), dtype=torch.float64, device=dev)
    _lib.check(_lib.load().pp_event_llh_device(
        propagator.handle, _MODES[mode], H, S, M, d_p.data_ptr(), d_n.data_ptr() if d_n is not None else None,
        d_o.data_ptr(), d_t.data_ptr(), d_l.data_ptr(), torch.cuda.current_stream(dev).cuda_stream),
        propagator.handle)
    return d_l.cpu().numpy()


def surrogate_params(surrogate, pairs, n_sources, n_modules, medium):
    """[n_modules, n_sources, 6] parameters from the learned surrogate for the
    pairs of pp_cross_pairs_device (source-major: pairs[s * n_modules + m]):
    A = expected photons of the pair (N folded in), the mixture, and
    t_shift = the source's emission time + (d - r) n_g(800 nm) / c."""
    out, _ = surrogate.predict(pairs)
    x = features(pairs)
    d = 10.0 ** x[:, 0].astype(np.float64)
    ng = float(get_group_index(800.0, medium))
    shift = np.asarray(pairs["t0"], dtype=np.float64) + (d - pairs["radius"]) * ng / C_VACUUM_M_PER_NS
    prm = np.stack([out[:, 0], out[:, 1], out[:, 2], out[:, 3], out[:, 4], shift], axis=1)
    return prm.reshape(n_sources, n_modules, 6).transpose(1, 0, 2).copy()


def mc_hit_times(result, n_sources, n_modules):
    """Observed arrival times per module from an MC propagation of the
    cross-product pairs (hit pair index s * n_modules + m)."""
    h = result.hits
    mod = np.asarray(h["pair"], dtype=np.int64) % n_modules
    t = np.asarray(h["time"], dtype=np.float64)
    return [np.sort(t[mod == m]) for m in range(n_modules)]

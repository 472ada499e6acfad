"""Event likelihood on the device against the FP64 oracle (oracle/event.py),
and an event whose true hypothesis the likelihood prefers.  Tolerance: rtol
1e-10 (both FP64; the device sums in another order)."""
import numpy as np
import pytest

import photonprop_b200 as pp
from photonprop_b200 import event as ev
from photonprop_b200 import lightyield as ly
from photonprop_b200 import surrogate as sg
from oracle import event as OE

pytestmark = pytest.mark.gpu


def _random_case(rng, H, M, S):
    p = np.empty((H, M, S, 6))
    p[..., 0] = rng.uniform(0.0, 3.0, (H, M, S)) * (rng.uniform(size=(H, M, S)) < 0.9)
    p[..., 1] = rng.uniform(0.0, 1.0, (H, M, S))
    p[..., 2] = rng.uniform(0.8, 6.0, (H, M, S))
    p[..., 3] = rng.uniform(3.0, 30.0, (H, M, S))
    p[..., 4] = rng.uniform(0.5, 8.0, (H, M, S))
    p[..., 5] = rng.uniform(0.0, 20.0, (H, M, S))
    hits = [np.sort(rng.uniform(5.0, 200.0, rng.integers(0, 60))) for _ in range(M)]
    hits[0] = np.array([])
    hits[1] = np.array([1.0, 50.0])  # a hit before every source can contribute: ln f = -inf
    p[:, 1, :, 5] = np.maximum(p[:, 1, :, 5], 2.0)
    return p, hits


@pytest.mark.parametrize("S", [40, 700])
@pytest.mark.parametrize("mode", ["reference", "shifted"])
def test_llh_matches_oracle(propagator, S, mode):
    rng = np.random.default_rng(S)
    H, M = 3, 9
    p, hits = _random_case(rng, H, M, S)
    phot = rng.uniform(10.0, 1000.0, (H, S))
    got = ev.event_llh(propagator, p, hits, phot, mode=mode)
    for h in range(H):
        for m in range(M):
            ref = OE.module_llh(p[h, m], hits[m], phot[h], mode)
            if np.isinf(ref):
                assert got[h, m] == ref
            else:
                assert got[h, m] == pytest.approx(ref, rel=1e-10, abs=1e-9)


def test_event_likelihood_prefers_the_true_energy(propagator, medium):
    p = ly.Particle((0.0, 0.0, 0.0), (0.0, 0.0, 1.0), 0.0, 30.0, ly.ParticleType.EMinus)
    src, _ = ly.particles_to_sources(propagator, [p], (0.0, 5.0), 0.5, mode="metres", emitter="cone")
    mods = np.array([[5.0, 0.0, 8.0, 0.21], [0.0, 6.0, 9.0, 0.21], [-4.0, 0.0, 7.0, 0.21], [0.0, -8.0, 12.0, 0.21]])
    S, M = len(src), len(mods)
    ro = pp.RunOptions(mode="physical", t_max=1000.0, hist_bins=1000)
    # hypothesis parameters from an independent MC run of the same pairs
    pairs = ly.cross_pairs(propagator, src, mods, seed=1)
    ds = sg.mc_dataset(propagator, pairs, ro, min_hits_mu=0, min_hits_fit=0)
    y = ds.y.astype(np.float64)
    prm = np.stack([ds.mu, 1 / (1 + np.exp(-y[:, 1])), np.exp(y[:, 2]), np.exp(y[:, 3]), np.exp(y[:, 4]),
                    sg.time_shift(pairs, medium) + pairs["t0"]], axis=1)
    prm = prm.reshape(S, M, 6).transpose(1, 0, 2)
    # the observed event: another MC run, each weighted hit kept with probability = its weight
    obs = ly.cross_pairs(propagator, src, mods, seed=2)
    res = propagator.propagate(obs, pp.RunOptions(mode="physical", t_max=1000.0, hist_bins=0), hit_capacity=1 << 22)
    rng = np.random.default_rng(0)
    keep = rng.uniform(size=len(res.hits)) < res.hits["weight"]
    res.hits = res.hits[keep]
    times = ev.mc_hit_times(res, S, M)
    assert min(len(t) for t in times) > 30
    scales = np.array([0.33, 1.0, 3.0])
    hyp = prm[None] * np.array([1, 1, 1, 1, 1, 1])[None, None, None, :]
    hyp = np.repeat(hyp, 3, axis=0)
    hyp[..., 0] *= scales[:, None, None]
    llh = ev.event_llh(propagator, hyp, times, mode="shifted").sum(axis=1)
    assert llh[1] > llh[0] and llh[1] > llh[2], llh

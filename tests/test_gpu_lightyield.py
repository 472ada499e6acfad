"""Particles -> light sources on the device against the FP64 oracle, the
source x target cross product, and an event-driven batch through the
propagation kernel.  Photon counts are integers: exact, except where the
FP64 product lands within 1e-6 of a rounding tie."""
import numpy as np
import pytest

import photonprop_b200 as pp
from photonprop_b200 import lightyield as ly
from oracle import lightyield as OL
from oracle import tables as tb

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("mode,grid", [("reference", (0.0, 3000.0, 10.0)), ("metres", (0.0, 20.0, 0.1))])
def test_sources_match_oracle(propagator, mode, grid):
    parts = [ly.Particle((1.0, -2.0, 3.0), (0.0, 0.6, 0.8), 5.0, 1e3, ly.ParticleType.EMinus),
             ly.Particle((0.0, 0.0, 0.0), (1.0, 0.0, 0.0), 0.0, 37.5, ly.ParticleType.EPlus),
             ly.Particle((10.0, 10.0, -5.0), (0.0, 0.0, -1.0), 100.0, 2e4, ly.ParticleType.Gamma)]
    src, ng = ly.particles_to_sources(propagator, parts, grid[:2], grid[2], (300.0, 800.0), mode=mode)
    g = np.arange(grid[0], grid[1] + grid[2] / 2, grid[2])
    assert ng == len(g) and len(src) == 3 * (ng - 1)
    om = tb.cascadia(35.0, 2.0)  # the propagator's medium
    for i, p in enumerate(parts):
        ref = OL.elongated_sources(p.position, p.direction, p.time, p.energy, p.type, g, om, (300.0, 800.0), mode)
        s = src[i * (ng - 1):(i + 1) * (ng - 1)]
        exp_n = np.array([r[2] for r in ref])
        bad = np.nonzero(s["n_photons"] != exp_n)[0]
        assert len(bad) <= 1 and np.all(np.abs(s["n_photons"][bad] - exp_n[bad]) <= 1)
        np.testing.assert_allclose(s["pos"], np.array([r[0] for r in ref]), rtol=1e-6, atol=1e-5)
        np.testing.assert_allclose(s["t0"], [r[1] for r in ref], rtol=1e-6, atol=1e-5)
        assert np.all(s["emitter"] == pp._lib.EMITTER_ISOTROPIC)


def test_cross_pairs_and_event_batch(propagator):
    p = ly.Particle((0.0, 0.0, 0.0), (0.0, 0.0, 1.0), 0.0, 100.0, ly.ParticleType.EMinus)
    src, ng = ly.particles_to_sources(propagator, [p], (0.0, 10.0), 0.5, mode="metres", emitter="cone")
    assert np.all(src["track_len"] == np.float32(0.5)) and np.all(src["emitter"] == pp._lib.EMITTER_CHERENKOV_CONE)
    # three spheres on the Cherenkov cones of the track (41 deg), one far behind it
    targets = np.array([[5.0, 0.0, 7.75, 0.21], [0.0, 8.0, 13.2, 0.21], [-3.0, -3.0, 12.0, 0.21],
                        [20.0, 0.0, -20.0, 0.21]])
    pairs = ly.cross_pairs(propagator, src, targets, seed=9)
    assert len(pairs) == len(src) * 4
    L = pp._lib.load()
    for i in (0, 5, len(pairs) - 1):
        assert int(pairs["seed"][i]) == L.pp_pair_seed(9, i)
        np.testing.assert_array_equal(pairs["target"][i], targets[i % 4, :3].astype(np.float32))
        assert pairs["n_photons"][i] == src["n_photons"][i // 4]
    # the event's pairs propagate like any batch (fewer photons for speed)
    pairs["n_photons"] = np.minimum(pairs["n_photons"], 200_000)
    res = propagator.propagate(pairs, pp.RunOptions(mode="physical", t_max=500.0, hist_bins=0), hit_capacity=1 << 20)
    hits = res.stats[:, 0].reshape(len(src), 4).sum(0)
    assert np.all(hits[:3] > 100) and hits[3] < hits[:3].min() and np.all(np.isfinite(res.stats))

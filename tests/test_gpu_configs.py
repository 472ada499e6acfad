"""Parity of the CUDA path with the FP64 oracle on the benchmark
configurations themselves, through the C ABI.

  point source   the small CPU-runnable case exactly as stated (isotropic
                 point source at the origin, 1e5 photons, r = 0.21 m sphere
                 10 m along +x, 500 x 1 ns histogram, seed 0), and the same
                 geometry at 1e7 photons
  cone grid      the 25 pairs of the one-pair-per-launch workload (1 m
                 Cherenkov track along +z, spheres at {5..100} m x
                 {0..180} deg, 5 nm PMT table), photons capped per pair
  mixed batch    64 pairs of the 4096-pair benchmark batch spread over its
                 whole 2-150 m distance range, photons capped per pair
  free running   independent seeds on the GPU and the oracle: a cone pair and
                 a pair 60 m away, hit counts within 3 sigma, chi^2 p > 0.01
                 on the 1 ns arrival-time histogram

Fixed-random-number cases hold every matched photon to the tolerances of
_parity.check_matched and reconcile the kernel's FP64 per-pair sums and
histograms with the oracle's bin by bin
(_parity.check_pair_statistics_and_histograms).  The geometry replaces the
reference's one (sphere on +z, src/photon_prop_cuda.jl:588-609); the
physics is the physical mode (group-velocity time, cone emitter), which the
reference kernel does not implement.
"""
import numpy as np
import pytest

import photonprop_b200 as pp
from oracle import oracle as O
from oracle import tables as tb

from _parity import (check_matched, check_pair_statistics_and_histograms, chi2_two_sample, match_hits,
                     to_oracle_opts, to_oracle_pairs)

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def propagator_5nm(medium):
    spec = pp.CherenkovSpectrum((300.0, 800.0), 20, medium)
    prop = pp.Propagator(medium, spec, pp.p_one_pmt_acc_5nm, device=0)
    yield prop
    prop.close()


@pytest.fixture(scope="module")
def oracle_tables_5nm(propagator_5nm, oracle_medium):
    t = pp.p_one_pmt_acc_5nm
    return O.make_tables(oracle_medium, propagator_5nm.knots().astype(np.float64),
                         pmt=(t.wavelengths, t.acceptance))


def _fixed_rng_case(prop, tables, pairs, ro, label, min_hits, hit_capacity=1 << 22):
    res = prop.propagate(pairs, ro, hit_capacity=hit_capacity)
    assert not res.overflow
    oo = to_oracle_opts(ro)
    h, s, hist, steps, total = O.propagate(tables, to_oracle_pairs(pairs), oo, hit_cap=hit_capacity)
    assert total >= min_hits, (label, total)
    g, o, ng, no = match_hits(res.hits, h)
    check_matched(g, o, ng, no, label)
    moved = check_pair_statistics_and_histograms(res, h, s, hist, len(pairs), oo.hist_t0, oo.hist_bin_width,
                                                 oo.hist_bins, label)
    np.testing.assert_array_equal(res.stats[:, 6], pairs["n_photons"])
    print(label, "hits", res.n_hits, "oracle", total, "bin-edge moves", moved)
    return res, (h, s, hist, steps, total)


# ---------------------------------------------------------------------------
# the small CPU-runnable case, as stated

POINT_RO = dict(mode="physical", g=0.95, t_max=500.0, hist_t0=0.0, hist_bin_width=1.0, hist_bins=500,
                pmt_weight=False)


def test_point_source_case_exactly(propagator, oracle_tables):
    """1e5 photons, sphere at +x 10 m, seed 0, 500 x 1 ns: the same photons
    hit on both sides and the FP64 histogram matches bin by bin."""
    pair = pp.batches.point_source_pair(100_000, target=(10.0, 0.0, 0.0), seed=0)
    res, (h, *_rest) = _fixed_rng_case(propagator, oracle_tables, pair, pp.RunOptions(**POINT_RO),
                                       "point 1e5", min_hits=1)
    assert res.n_hits == len(h)  # no rim flip in this case
    assert np.array_equal(np.sort(res.hits["photon"]), np.sort(h["photon"]))


def test_point_source_geometry_at_1e7_photons(propagator, oracle_tables):
    pair = pp.batches.point_source_pair(10_000_000, target=(10.0, 0.0, 0.0), seed=0)
    res, orc = _fixed_rng_case(propagator, oracle_tables, pair, pp.RunOptions(**POINT_RO), "point 1e7",
                               min_hits=300)
    assert np.count_nonzero(res.hist[0]) > 10  # direct light at 44-48 ns and a scattered tail


# ---------------------------------------------------------------------------
# the cone grid of the one-pair-per-launch workload (5 nm PMT table)

def test_cone_grid_all_25_pairs(propagator_5nm, oracle_tables_5nm):
    pairs = pp.batches.cone_grid_pairs(n_photons=2_000_000)
    ro = pp.RunOptions(mode="physical", g=0.95, t_max=1000.0, hist_bins=1000, pmt_weight=True)
    res, (h, s, *_rest) = _fixed_rng_case(propagator_5nm, oracle_tables_5nm, pairs, ro, "cone grid",
                                          min_hits=5000)
    # every distance row has a sphere the cone reaches; the near ones are well populated
    assert s[:5, 0].max() > 1000
    # the plain one-pair-per-launch path gives the same statistics
    plain = propagator_5nm.propagate_plain(pairs, ro, hit_capacity=1 << 22)
    np.testing.assert_allclose(plain.stats, res.stats, rtol=1e-9, atol=1e-12)


# ---------------------------------------------------------------------------
# a slice of the 4096-pair benchmark batch over its whole distance range

def test_mixed_batch_full_distance_range(propagator, oracle_tables):
    b = pp.batches.mixed_batch(4096, seed=2024)
    d = np.linalg.norm(b["target"].astype(np.float64) - b["pos"].astype(np.float64), axis=1)
    sel = np.argsort(d)[np.linspace(0, len(b) - 1, 64).astype(np.int64)]
    sl = b[np.sort(sel)].copy()
    assert d[sel].min() < 3.0 and d[sel].max() > 148.0
    sl["n_photons"] = np.minimum(sl["n_photons"], 1_000_000)
    ro = pp.RunOptions(mode="physical", g=0.95, t_max=1000.0, hist_bins=1000, pmt_weight=True)
    res, (h, s, *_rest) = _fixed_rng_case(propagator, oracle_tables, sl, ro, "mixed slice", min_hits=300)
    far = np.linalg.norm(sl["target"].astype(np.float64), axis=1) > 50.0
    assert far.sum() >= 20
    assert s[far, 0].sum() > 0  # hits beyond 50 m matched too


# ---------------------------------------------------------------------------
# free running: independent streams

def _free_running(prop, tables, gpu_pair, orc_pair, ro, label, min_hits):
    r = prop.propagate(gpu_pair, ro, hit_capacity=1 << 22)
    h, s, hist, steps, total = O.propagate(tables, to_oracle_pairs(orc_pair), to_oracle_opts(ro))
    ng, no = r.n_hits, total
    assert min(ng, no) >= min_hits, (label, ng, no)
    assert abs(ng - no) <= 3 * np.sqrt(ng + no), (label, ng, no)
    bins = int(ro.hist_bins)
    cg, _ = np.histogram(r.hits["time"], bins=bins, range=(0, ro.t_max))
    co, _ = np.histogram(h["time"], bins=bins, range=(0, ro.t_max))
    chi2, dof, p = chi2_two_sample(cg, co)
    print(label, "free-running", ng, no, chi2, dof, p)
    assert p > 0.01, (label, chi2, dof, p)


def test_free_running_cone_pair(propagator, oracle_tables):
    """Cherenkov track, sphere 10 m away at 45 deg (near the cone)."""
    ro = pp.RunOptions(mode="physical", g=0.95, t_max=200.0, hist_bins=200, pmt_weight=False)
    g = pp.batches.cone_grid_pairs(n_photons=3_000_000, distances=(10.0,), polar_deg=(45.0,), seed=301)
    o = pp.batches.cone_grid_pairs(n_photons=3_000_000, distances=(10.0,), polar_deg=(45.0,), seed=302)
    assert g["seed"][0] != o["seed"][0]
    _free_running(propagator, oracle_tables, g, o, ro, "cone 10 m", min_hits=1000)


def test_free_running_far_pair(propagator, oracle_medium, oracle_tables):
    """A sphere 60 m from a Cherenkov track, on its cone (acos(1/n(400 nm)))."""
    ro = pp.RunOptions(mode="physical", g=0.95, t_max=600.0, hist_bins=600, pmt_weight=False)
    th = float(np.degrees(np.arccos(1.0 / tb.refractive_index(400.0, oracle_medium))))
    g = pp.batches.cone_grid_pairs(n_photons=8_000_000, distances=(60.0,), polar_deg=(th,), seed=303)
    o = pp.batches.cone_grid_pairs(n_photons=8_000_000, distances=(60.0,), polar_deg=(th,), seed=304)
    _free_running(propagator, oracle_tables, g, o, ro, "cone 60 m", min_hits=400)

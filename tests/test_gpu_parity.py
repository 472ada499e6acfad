"""Parity of the CUDA kernels (through the C ABI) with the FP64 oracle.

Tolerances (FP32 photon state against the FP64 oracle replaying the same
Philox numbers):
  device helpers      philox / uniform bit-exact; HG, rotation, medium rel/abs 2e-5
  matched photons     |d pos| <= 2e-3 m + 2e-5 * path, |d t| <= 1e-2 ns + 1e-5 * t,
                      |d w| <= 1e-3 w + 1e-8, |d lambda| / lambda <= 1e-5
  branch flips        photons detected on one side only <= 1 % of hits (+3)
"""
import numpy as np
import pytest

import photonprop_b200 as pp
from oracle import oracle as O
from oracle import tables as tb

from _parity import chi2_two_sample, check_matched, match_hits, to_oracle_opts, to_oracle_pairs

pytestmark = pytest.mark.gpu


_check_matched = check_matched


# ---------------------------------------------------------------------------
# device helpers (the counterpart of the reference's apply_rot test kernel)

def test_device_philox_and_uniform_bit_exact(propagator):
    rng = np.random.default_rng(1)
    ctr = rng.integers(0, 2**32, size=(256, 6), dtype=np.uint64)
    ctr[0] = 0
    ctr[1] = 0xFFFFFFFF
    out = propagator.device_eval(0, ctr.astype(np.float64))
    for i in range(256):
        want = O.philox4x32_10([int(x) for x in ctr[i, :4]], [int(x) for x in ctr[i, 4:]])
        assert [int(x) for x in out[i]] == want
    w = rng.integers(0, 2**32, size=1000, dtype=np.uint64)
    u = propagator.device_eval(1, w.astype(np.float64))[:, 0]
    np.testing.assert_array_equal(u, [O.uniform(int(x)) for x in w])
    # a step's Philox2x32-10 block and its three 21-bit uniforms
    sc = rng.integers(0, 2**32, size=(512, 3), dtype=np.uint64)
    sc[0] = 0
    sc[1] = 0xFFFFFFFF
    out = propagator.device_eval(12, sc.astype(np.float64))
    for i in range(512):
        wds = O.philox2x32_10([int(sc[i, 0]), int(sc[i, 1])], int(sc[i, 2]))
        assert [int(x) for x in out[i, :2]] == wds
        assert list(out[i, 2:]) == O.step_uniforms(wds)


def test_device_hg_costheta(propagator):
    u = np.array([O.uniform(w) for w in np.random.default_rng(2).integers(0, 2**32, 4000)])
    for g in (0.99, 0.95, 0.5, 0.0, -0.3):
        gf = float(np.float32(g))
        dev = propagator.device_eval(2, np.stack([np.full_like(u, g), u], 1))[:, 0]
        ref = np.array([O.hg_costheta(gf, x) for x in u])
        np.testing.assert_allclose(dev, ref, atol=2e-5 if g > 0.9 else 2e-6)
    # reference KAT: mean cos(theta) = g (src/tests/test_photon_prob.jl:19-21)
    dev = propagator.device_eval(2, np.stack([np.full_like(u, 0.97), u], 1))[:, 0]
    assert abs(dev.mean() - 0.97) < 0.01


def test_device_rotate_to_axis(propagator):
    kats = [([0, 0, 1.0], [0, 1.0, 0], [0, 1.0, 0]), ([0, 0, -1.0], [0, 1.0, 0], [0, -1.0, 0]),
            ([0, 1.0, 0], [0, 1.0, 0], [0, 0, -1.0])]
    x = np.array([o + n for o, n, _ in kats], dtype=np.float64)
    out = propagator.device_eval(3, x)
    for r, (_, _, want) in zip(out, kats):
        np.testing.assert_allclose(r, want, atol=1e-6)
    rng = np.random.default_rng(3)
    o = rng.normal(size=(5000, 3))
    o /= np.linalg.norm(o, axis=1, keepdims=True)
    o[:5] = [[0, 0, 1], [0, 0, -1], [1e-4, 0, -1 + 5e-9], [0, 1e-3, 1 - 5e-7], [1, 0, 0]]
    o[:5] /= np.linalg.norm(o[:5], axis=1, keepdims=True)
    n = rng.normal(size=(5000, 3))
    n /= np.linalg.norm(n, axis=1, keepdims=True)
    o32, n32 = o.astype(np.float32).astype(np.float64), n.astype(np.float32).astype(np.float64)
    out = propagator.device_eval(3, np.concatenate([o32, n32], 1))
    # reference on exactly normalised inputs: its sin(theta) = sqrt(1 - o_z^2) is
    # ill-conditioned near the poles for vectors that are unit only to FP32 rounding
    ref = np.array([O.rotate_to_axis(a / np.linalg.norm(a), b / np.linalg.norm(b)) for a, b in zip(o32, n32)])
    err = np.linalg.norm(out - ref, axis=1)
    far = np.abs(o32[:, 2] + 1) > 1e-3  # away from the south pole the rotation is well conditioned
    assert err[far].max() < 2e-6
    np.testing.assert_allclose(np.linalg.norm(out, axis=1), 1.0, atol=1e-6)


def test_device_position_update(propagator):  # src/tests/test_photon_prob.jl:67-73
    out = propagator.device_eval(4, np.array([[0, 0, 0, 0, 1.0, 0, 10.0]]))
    np.testing.assert_allclose(out[0], [0, 10.0, 0])


def test_device_medium_tables(propagator, oracle_tables, oracle_medium):
    wl = np.linspace(300.0, 800.0, 501)
    np.testing.assert_allclose(propagator.device_eval(6, wl)[:, 0], tb.refractive_index(wl, oracle_medium),
                               rtol=2e-6)
    np.testing.assert_allclose(propagator.device_eval(7, wl)[:, 0], tb.group_index(wl, oracle_medium), rtol=2e-6)
    np.testing.assert_allclose(propagator.device_eval(8, wl)[:, 0], tb.scattering_length(wl, oracle_medium),
                               rtol=2e-5)
    np.testing.assert_allclose(propagator.device_eval(9, wl)[:, 0], tb.absorption_length(wl), rtol=2e-6)
    t = pp.p_one_pmt_acc
    np.testing.assert_allclose(propagator.device_eval(10, wl)[:, 0],
                               tb.pmt_acceptance(wl, (t.wavelengths, t.acceptance)), rtol=2e-5, atol=1e-7)
    u = np.array([O.uniform(w) for w in np.random.default_rng(4).integers(0, 2**32, 2000)])
    k = propagator.knots().astype(np.float64)
    np.testing.assert_allclose(propagator.device_eval(5, u)[:, 0], tb.interp_equidistant(u, k, 0.0, 1.0),
                               rtol=1e-6)
    # the device knots are the float rounding of the FP64 spectrum table
    np.testing.assert_allclose(k, tb.cherenkov_spectrum_knots((300.0, 800.0), 20, oracle_medium), rtol=1e-7)


# ---------------------------------------------------------------------------
# fixed random numbers: per-photon parity

def test_fixed_rng_compat_reference_geometry(propagator, oracle_tables):
    """propagate_distance's geometry (sphere on +z, src/photon_prop_cuda.jl:588-609)
    in reference-compatible mode."""
    pairs = pp.batches.point_source_pair(200_000, target=(0.0, 0.0, 10.0), seed=0)
    ro = pp.RunOptions(mode="compat", hist_bins=0, pmt_weight=False)
    res = propagator.propagate(pairs, ro)
    h, s, _, steps, total = O.propagate(oracle_tables, to_oracle_pairs(pairs), to_oracle_opts(ro))
    assert total > 1000
    g, o, ng, no = match_hits(res.hits, h)
    _check_matched(g, o, ng, no, "compat")
    np.testing.assert_allclose(g["dir0"], o["dir0"], atol=1e-5)


def test_fixed_rng_physical_point_source(propagator, oracle_tables):
    pairs = pp.batches.point_source_pair(1_000_000, target=(3.0, 0.0, 0.0), seed=5)
    ro = pp.RunOptions(mode="physical", g=0.95, t_max=500.0, hist_bins=500)
    res = propagator.propagate(pairs, ro)
    h, s, hist, steps, total = O.propagate(oracle_tables, to_oracle_pairs(pairs), to_oracle_opts(ro))
    assert total > 200
    g, o, ng, no = match_hits(res.hits, h)
    _check_matched(g, o, ng, no, "physical-iso")
    # per-pair FP64 statistics follow the hits
    np.testing.assert_allclose(res.stats[0, 0], s[0, 0], rtol=0.01, atol=3)
    np.testing.assert_allclose(res.stats[0, 1], s[0, 1], rtol=0.01)


def test_fixed_rng_physical_cone_and_batch(propagator, oracle_tables):
    b = pp.batches.mixed_batch(48, seed=11, n_min=2e4, n_max=2e5, d_min=2.0, d_max=8.0)
    ro = pp.RunOptions(mode="physical", g=0.95, t_max=300.0, hist_bins=300)
    res = propagator.propagate(b, ro)
    h, s, hist, steps, total = O.propagate(oracle_tables, to_oracle_pairs(b), to_oracle_opts(ro))
    assert total > 500
    g, o, ng, no = match_hits(res.hits, h)
    _check_matched(g, o, ng, no, "physical-mixed")
    np.testing.assert_allclose(res.stats[:, 6], b["n_photons"])


def test_batched_equals_plain(propagator):
    b = pp.batches.mixed_batch(24, seed=12, n_min=1e4, n_max=3e5, d_min=2.0, d_max=6.0)
    ro = pp.RunOptions(mode="physical", hist_bins=200, t_max=200.0)
    a = propagator.propagate(b, ro).sorted_hits()
    c = propagator.propagate_plain(b, ro).sorted_hits()
    assert len(a) == len(c) > 100
    np.testing.assert_array_equal(a["photon"], c["photon"])
    np.testing.assert_array_equal(a["pair"], c["pair"])
    np.testing.assert_allclose(a["pos"], c["pos"], rtol=1e-6, atol=1e-6)
    np.testing.assert_allclose(a["time"], c["time"], rtol=1e-6)


def test_deterministic_across_runs(propagator):
    b = pp.batches.mixed_batch(16, seed=13, n_min=1e5, n_max=1e6, d_min=2.0, d_max=5.0)
    ro = pp.RunOptions(mode="physical")
    a = propagator.propagate(b, ro)
    c = propagator.propagate(b, ro)
    ha, hc = a.sorted_hits(), c.sorted_hits()
    assert ha.tobytes() == hc.tobytes()
    np.testing.assert_allclose(a.stats, c.stats, rtol=1e-12)


def test_hits_and_statistics_consistent(propagator):
    b = pp.batches.mixed_batch(32, seed=14, n_min=1e5, n_max=1e6, d_min=2.0, d_max=10.0)
    ro = pp.RunOptions(mode="physical", t_max=400.0, hist_bins=400)
    r = propagator.propagate(b, ro)
    assert not r.overflow and r.n_hits == len(r.hits)
    for p in range(len(b)):
        hp = r.hits[r.hits["pair"] == p]
        w = hp["weight"].astype(np.float64)
        t = hp["time"].astype(np.float64)
        assert r.stats[p, 0] == len(hp)
        np.testing.assert_allclose(r.stats[p, 1], w.sum(), rtol=1e-5, atol=1e-12)
        np.testing.assert_allclose(r.stats[p, 3], (w * t).sum(), rtol=1e-5, atol=1e-9)
        inwin = (t >= 0) & (t < 400.0)
        np.testing.assert_allclose(r.hist[p].sum(), w[inwin].sum(), rtol=1e-5, atol=1e-12)
        assert r.stats[p, 6] == b["n_photons"][p]
    assert np.all(r.hits["time"] < 400.0)


def test_cone_emission_geometry(propagator, oracle_medium):
    """Every detected photon of a Cherenkov track left it at acos(1/n(lambda))."""
    p = pp.batches.cone_grid_pairs(n_photons=2_000_000, distances=(2.0,), polar_deg=(45.0, 90.0))
    r = propagator.propagate(p, pp.RunOptions(mode="physical"))
    assert r.n_hits > 100
    cos_c = r.hits["dir0"] @ np.array([0.0, 0.0, 1.0])
    want = 1.0 / tb.refractive_index(r.hits["wavelength"].astype(np.float64), oracle_medium)
    np.testing.assert_allclose(cos_c, want, atol=2e-5)


def test_photon_index_beyond_32_bits(propagator, oracle_tables):
    """A pair whose photon indices cross 2^32: hits above the boundary replay
    exactly in the oracle."""
    p = pp.batches.point_source_pair((1 << 32) + (1 << 22), target=(0.0, 0.0, 2.0), seed=21)
    ro = pp.RunOptions(mode="physical", t_max=100.0, hist_bins=0)
    r = propagator.propagate(p, ro, hit_capacity=1 << 24)
    assert r.stats[0, 6] == (1 << 32) + (1 << 22)
    hi = r.hits[r.hits["photon"] >= (1 << 32)]
    assert len(hi) > 50
    op = to_oracle_pairs(p)[0]
    oo = to_oracle_opts(ro)
    for hrec in hi[:200]:
        want = O.simulate_one(oracle_tables, op, 0, int(hrec["photon"]), oo)
        if want is None:
            continue  # a rim flip
        assert abs(float(hrec["time"]) - want["time"]) < 1e-2
        np.testing.assert_allclose(hrec["pos"], want["pos"], atol=2e-3)


# ---------------------------------------------------------------------------
# free-running statistics: independent streams, 3 sigma counts and chi^2

def test_free_running_counts_and_time_histogram(propagator, oracle_tables):
    ro = pp.RunOptions(mode="physical", g=0.95, t_max=200.0, hist_bins=200, pmt_weight=False)
    n = 4_000_000
    gp = pp.batches.point_source_pair(n, target=(4.0, 0.0, 0.0), seed=101)
    op = to_oracle_pairs(pp.batches.point_source_pair(n, target=(4.0, 0.0, 0.0), seed=202))
    r = propagator.propagate(gp, ro)
    h, s, hist, steps, total = O.propagate(oracle_tables, op, to_oracle_opts(ro))
    ng, no = r.n_hits, total
    assert abs(ng - no) <= 3 * np.sqrt(ng + no), (ng, no)
    cg, _ = np.histogram(r.hits["time"], bins=200, range=(0, 200))
    co, _ = np.histogram(h["time"], bins=200, range=(0, 200))
    chi2, dof, p = chi2_two_sample(cg, co)
    print("free-running", ng, no, chi2, dof, p)
    assert p > 0.01


# ---------------------------------------------------------------------------
# reference-shaped entry points

def test_stacks_kernel_matches_oracle(propagator, medium, oracle_tables):
    """pp_cuda_propagate_photons with propagate_distance's launch
    (src/photon_prop_cuda.jl:598-606: 16 x 1024 threads, stack_len =
    cld(1e5, 16), seed 0, sphere 10 m along +z) in compat mode, against the
    FP64 oracle over the photons the launch simulates: every thread runs
    cld(N, 16384) photons (:288), photon g + i * 16384 on thread g.  The
    reference layout carries no photon index, so a stack entry is matched to
    the oracle hit with its wavelength (to 1e-5) and emission direction."""
    import torch
    blocks, threads = 16, 1024
    stack_len = -(-100_000 // blocks)
    n_gen = 100_000
    arrays = pp.initialize_photon_arrays(stack_len, blocks)
    spec = pp.CherenkovSpectrum((300.0, 800.0), 20, medium)
    src = pp.PhotonSource((0.0, 0.0, 0.0), (0.0, 0.0, 1.0), 0.0, n_gen, spec, pp.IsotropicEmission)
    pp.cuda_propagate_photons_(*arrays, stack_len, 0, src, (0.0, 0.0, 10.0), 0.21, medium, threads=threads,
                               propagator=propagator)
    torch.cuda.synchronize()
    pos, dirs, wls, dist, sp, nsim = (a.cpu().numpy() for a in arrays)
    per_thread = -(-n_gen // (blocks * threads))
    assert nsim[0] == per_thread * blocks * threads
    assert np.all(sp[sp > 0] <= (np.arange(blocks) + 1)[sp > 0] * stack_len)
    g_pos = pp.process_output(pos.reshape(-1, 3), sp).astype(np.float64)
    g_dir = pp.process_output(dirs.reshape(-1, 3), sp).astype(np.float64)
    g_wl = pp.process_output(wls, sp).astype(np.float64)
    g_dist = pp.process_output(dist, sp).astype(np.float64)
    pair = pp.batches.point_source_pair(int(nsim[0]), target=(0.0, 0.0, 10.0), seed=0)
    ro = pp.RunOptions(mode="compat", hist_bins=0, pmt_weight=False)
    h, *_ = O.propagate(oracle_tables, to_oracle_pairs(pair), to_oracle_opts(ro))
    assert len(h) > 1000
    order = np.argsort(h["wavelength"])
    o_wl = h["wavelength"][order]
    matched = 0
    used = set()
    for k in range(len(g_wl)):
        lo = np.searchsorted(o_wl, g_wl[k] * (1 - 1e-5))
        hi = np.searchsorted(o_wl, g_wl[k] * (1 + 1e-5))
        cand = order[lo:hi]
        if len(cand) == 0:
            continue
        j = cand[np.argmin(np.linalg.norm(h["dir0"][cand] - g_dir[k], axis=1))]
        if np.linalg.norm(h["dir0"][j] - g_dir[k]) > 1e-4 or j in used:
            continue
        used.add(j)
        matched += 1
        assert abs(g_dist[k] - h["dist"][j]) <= 2e-3 + 2e-5 * h["dist"][j], (k, g_dist[k], h["dist"][j])
        assert np.linalg.norm(g_pos[k] - h["pos"][j]) <= 2e-3 + 2e-5 * h["dist"][j]
    n = max(len(g_wl), len(h))
    assert n - matched <= 0.01 * n + 3, (len(g_wl), len(h), matched)


def test_propagate_distance_dataframe(propagator, medium, oracle_tables, oracle_medium):
    df = pp.propagate_distance(10.0, medium, 100_000, propagator=propagator)
    assert list(df.columns) == ["tres", "initial_theta", "ref_ix", "abs_weight", "dist_travelled", "wavelength"]
    assert len(df) > 1000
    # the reference's host finish, recomputed from the oracle's own hits
    pairs = pp.batches.point_source_pair(100_000, target=(0.0, 0.0, 10.0), seed=0)
    ro = pp.RunOptions(mode="compat", hist_bins=0, pmt_weight=False)
    h, *_ = O.propagate(oracle_tables, to_oracle_pairs(pairs), to_oracle_opts(ro))
    ref_ix = tb.refractive_index(h["wavelength"], oracle_medium)
    tgeo = (10.0 - 0.21) / (0.299792458 / tb.refractive_index(800.0, oracle_medium))
    tres = h["dist"] / (0.299792458 / ref_ix) - tgeo
    assert abs(len(df) - len(h)) <= 0.01 * len(h) + 3
    q = [0.1, 0.5, 0.9]
    np.testing.assert_allclose(np.quantile(df["tres"], q), np.quantile(tres, q), atol=0.05)
    w_ref = np.exp(-h["dist"] / tb.absorption_length(h["wavelength"]))
    np.testing.assert_allclose(np.quantile(df["abs_weight"], q), np.quantile(w_ref, q), rtol=1e-3)
    assert np.all(df["initial_theta"] <= 1.0 + 1e-6)  # theta drawn in (-1, 1) rad (reference)


# ---------------------------------------------------------------------------
# edge cases and errors

def test_empty_and_zero_photon_pairs(propagator):
    r = propagator.propagate(np.zeros(0, dtype=pp.PAIR_DTYPE), pp.RunOptions())
    assert r.n_hits == 0 and r.stats.shape == (0, 8)
    p = pp.batches.mixed_batch(8, seed=5, n_min=1e4, n_max=1e5)
    p["n_photons"][[0, 3, 7]] = 0
    r = propagator.propagate(p, pp.RunOptions())
    assert np.all(r.stats[[0, 3, 7], 0] == 0) and np.all(r.stats[[0, 3, 7], 6] == 0)
    assert set(np.unique(r.hits["pair"])) <= {1, 2, 4, 5, 6}
    r2 = propagator.propagate_plain(p, pp.RunOptions())
    assert r2.n_hits == r.n_hits


def test_hit_overflow_reports_true_count(propagator):
    p = pp.batches.point_source_pair(2_000_000, target=(0.0, 0.0, 1.0), seed=3)
    full = propagator.propagate(p, pp.RunOptions(mode="physical", t_max=50.0))
    assert full.n_hits > 1000
    r = propagator.propagate(p, pp.RunOptions(mode="physical", t_max=50.0), hit_capacity=100)
    assert r.overflow and r.n_hits == full.n_hits and len(r.hits) == 100
    np.testing.assert_allclose(r.stats, full.stats, rtol=1e-9)
    r = propagator.propagate(p, pp.RunOptions(mode="physical", t_max=50.0, write_hits=False), hit_capacity=0)
    assert not r.overflow and r.n_hits == full.n_hits and len(r.hits) == 0


def test_normalize_flag(propagator):
    p = pp.batches.point_source_pair(1_000_000, target=(3.0, 0.0, 0.0), seed=9)
    a = propagator.propagate(p, pp.RunOptions(hist_bins=100, t_max=100.0))
    b = propagator.propagate(p, pp.RunOptions(hist_bins=100, t_max=100.0, normalize=True))
    np.testing.assert_allclose(b.hist, a.hist / 1e6, rtol=1e-12)


def test_invalid_arguments_raise(propagator):
    p = pp.batches.point_source_pair(1000)
    for bad in (pp.RunOptions(g=1.0), pp.RunOptions(max_steps=0), pp.RunOptions(hist_bins=-1),
                pp.RunOptions(hist_bins=10, hist_bin_width=0.0), pp.RunOptions(block_size=100)):
        with pytest.raises(pp.PPError) as e:
            propagator.propagate(p, bad)
        assert e.value.status == 1
    cone = pp.batches.cone_grid_pairs(1000, distances=(5.0,), polar_deg=(0.0,))
    with pytest.raises(pp.PPError, match="ArgumentError"):
        propagator.propagate(cone, pp.RunOptions(mode="compat"))
    q = p.copy()
    q["n_photons"] = -1
    with pytest.raises(pp.PPError):
        propagator.propagate(q, pp.RunOptions())
    q = p.copy()
    q["radius"] = 0
    with pytest.raises(pp.PPError):
        propagator.propagate(q, pp.RunOptions())
    # the limits of the Philox counter: photon index < 2^40, step < 2^24 - 1
    q = p.copy()
    q["n_photons"] = (1 << 40) + 1
    with pytest.raises(pp.PPError, match="2\\^40"):
        propagator.propagate(q, pp.RunOptions())
    with pytest.raises(pp.PPError, match="max_steps"):
        propagator.propagate(p, pp.RunOptions(max_steps=(1 << 24) - 1))
    r = propagator.propagate(p, pp.RunOptions(max_steps=(1 << 24) - 2))  # the largest accepted
    np.testing.assert_array_equal(r.stats[:, 6], p["n_photons"])
    q = p.copy()
    q["emitter"] = 7
    with pytest.raises(pp.PPError, match="unknown emitter"):
        propagator.propagate(q, pp.RunOptions())
    q = cone.copy()
    q["dir"] = (0.0, 0.0, 2.0)
    with pytest.raises(pp.PPError, match="unit direction"):
        propagator.propagate(q, pp.RunOptions())
    with pytest.raises(pp.PPError, match="t_max"):
        propagator.propagate(p, pp.RunOptions(t_max=float("inf")))


def test_device_api_graph_replay_matches_host_api(propagator):
    import torch
    b = pp.batches.mixed_batch(64, seed=31, n_min=1e4, n_max=5e5, d_min=2.0, d_max=10.0)
    ro = pp.RunOptions(mode="physical", t_max=300.0, hist_bins=300)
    host = propagator.propagate(b, ro)
    dev = torch.device("cuda:0")
    d_pairs = torch.from_numpy(b.view(np.uint8).copy()).to(dev)
    cap = 1 << 18
    d_hits = torch.zeros(cap * 64, dtype=torch.uint8, device=dev)
    d_cnt = torch.zeros(4, dtype=torch.int64, device=dev)
    d_stats = torch.zeros((len(b), 8), dtype=torch.float64, device=dev)
    d_hist = torch.zeros((len(b), 300), dtype=torch.float64, device=dev)
    s = torch.cuda.Stream()
    before = pp.launch_count()
    for _ in range(3):  # first call captures the graph, the others replay it
        propagator.propagate_device(d_pairs, len(b), ro, d_hits, cap, d_cnt, d_stats, d_hist, stream=s)
    s.synchronize()
    assert pp.launch_count() - before == 9
    assert int(d_cnt[0]) == host.n_hits
    np.testing.assert_allclose(d_stats.cpu().numpy(), host.stats, rtol=1e-9)
    np.testing.assert_allclose(d_hist.cpu().numpy(), host.hist, rtol=1e-9, atol=1e-15)
    hits = d_hits.cpu().numpy()[:host.n_hits * 64].view(pp.HIT_DTYPE)
    hs = hits[np.lexsort((hits["photon"], hits["pair"]))]
    assert hs.tobytes() == host.sorted_hits().tobytes()


def test_autotune_and_cache(propagator, tmp_path):
    b = pp.batches.mixed_batch(64, seed=41, n_min=1e5, n_max=1e6)
    ro = pp.RunOptions(mode="physical")
    path = str(tmp_path / "tune.txt")
    best = propagator.autotune(b, ro, cache_path=path)
    assert best["block_size"] in (128, 256, 512) and best["photons_per_s"] > 0
    again = propagator.autotune(b, ro, cache_path=path)  # read back from the cache
    assert again["block_size"] == best["block_size"] and again["chunk_photons"] == best["chunk_photons"]
    r = propagator.propagate(b, ro)
    assert r.n_hits > 0


def test_full_size_benchmark_batch_properties(propagator):
    """The 4096-pair benchmark batch at full size (5.75e9 photons), through
    size-independent properties: batched and plain paths give the same hits
    and statistics (the photons are a fixed function of the seeds), every
    hit record agrees with its pair's FP64 sums, histograms hold the
    in-window weight, and each pair counts all its photons."""
    b = pp.batches.mixed_batch(4096, seed=2024)
    ro = pp.RunOptions(mode="physical", g=0.95, t_max=1000.0, hist_bins=1000)
    a = propagator.propagate(b, ro, hit_capacity=1 << 21)
    c = propagator.propagate_plain(b, ro, hit_capacity=1 << 21)
    assert not a.overflow and a.n_hits > 100_000
    # the two kernels run the same device code; allow for a photon grazing a
    # sphere to flip should the compiler contract one of them differently
    ha, hc = a.sorted_hits(), c.sorted_hits()
    ka = set(zip(ha["pair"].tolist(), ha["photon"].tolist()))
    kc = set(zip(hc["pair"].tolist(), hc["photon"].tolist()))
    assert len(ka ^ kc) <= 1e-5 * len(ka) + 2
    if ka == kc:
        np.testing.assert_allclose(ha["pos"], hc["pos"], rtol=1e-5, atol=1e-5)
        np.testing.assert_allclose(ha["time"], hc["time"], rtol=1e-6)
    np.testing.assert_allclose(a.stats[:, 1:6], c.stats[:, 1:6], rtol=1e-3, atol=1e-6)
    np.testing.assert_array_equal(a.stats[:, 6], b["n_photons"])
    per_pair = np.bincount(ha["pair"], minlength=len(b))
    np.testing.assert_array_equal(a.stats[:, 0], per_pair)
    w = ha["weight"].astype(np.float64)
    np.testing.assert_allclose(a.stats[:, 1], np.bincount(ha["pair"], weights=w, minlength=len(b)),
                               rtol=1e-5, atol=1e-9)
    t = ha["time"].astype(np.float64)
    inwin = (t >= 0) & (t < 1000.0)
    np.testing.assert_allclose(a.hist.sum(axis=1), np.bincount(ha["pair"][inwin], weights=w[inwin],
                                                               minlength=len(b)), rtol=1e-5, atol=1e-9)


def test_cascade_emitter_sampler_matches_oracle(propagator):
    """cos(theta) of the cascade emitter: the device's FP32 tables against the
    oracle's FP64 tables (built independently with scipy)."""
    from oracle import fits as F
    rng = np.random.default_rng(21)
    u = rng.uniform(size=20000)
    n = rng.uniform(1.30, 1.40, size=20000)
    got = propagator.device_eval(11, np.stack([u, n], axis=1))[:, 0]
    np.testing.assert_allclose(got, F.cascade_cos_theta(u, n), rtol=0, atol=3e-5)


def test_fixed_rng_cascade_emitter(propagator, oracle_tables):
    b = pp.batches.mixed_batch(32, seed=17, n_min=2e4, n_max=2e5, d_min=2.0, d_max=8.0)
    b["emitter"] = pp._lib.EMITTER_CASCADE
    b["track_len"] = 0.0
    ro = pp.RunOptions(mode="physical", g=0.95, t_max=300.0, hist_bins=300)
    res = propagator.propagate(b, ro)
    h, s, hist, steps, total = O.propagate(oracle_tables, to_oracle_pairs(b), to_oracle_opts(ro))
    assert total > 200
    g, o, ng, no = match_hits(res.hits, h)
    _check_matched(g, o, ng, no, "physical-cascade")
    # compat mode has no cascade emitter (the reference rejects non-isotropic emission)
    with pytest.raises(pp.PPError):
        propagator.propagate(b[:1], pp.RunOptions(mode="compat"))


def test_cascade_pairs_on_the_device_api_need_the_flag(propagator):
    import torch
    b = pp.batches.mixed_batch(8, seed=19, n_min=1e5, n_max=2e5, d_min=2.0, d_max=4.0)
    b["emitter"] = pp._lib.EMITTER_CASCADE
    ref = propagator.propagate(b, pp.RunOptions(mode="physical", hist_bins=0))
    d_pairs = torch.from_numpy(b.view(np.uint8).copy()).cuda()
    cap = 1 << 18
    d_hits = torch.zeros(cap * 64, dtype=torch.uint8, device="cuda")
    d_cnt = torch.zeros(4, dtype=torch.int64, device="cuda")
    d_st = torch.zeros((len(b), 8), dtype=torch.float64, device="cuda")
    for flag in (False, True):
        ro = pp.RunOptions(mode="physical", hist_bins=0, cascade=flag)
        propagator.propagate_device(d_pairs, len(b), ro, d_hits, cap, d_cnt, d_st, None,
                                    stream=torch.cuda.current_stream())
        torch.cuda.synchronize()
        status = int(d_cnt[2].item())
        if flag:
            assert status & 4 == 0
            np.testing.assert_allclose(d_st.cpu().numpy(), ref.stats, rtol=1e-9, atol=1e-12)
        else:
            assert status & 4  # flagged: emitted on the cone instead


def test_reachability_cut_is_exact(propagator, oracle_tables):
    """Physical mode ends a photon once its sphere is farther than the path it
    has left before t_max.  With t_max = 100 ns (about 22 m of path) and
    spheres 10-20 m away most photons end that way; the oracle, which steps
    every photon to t_max, must find exactly the same hits."""
    b = pp.batches.mixed_batch(24, seed=23, n_min=2e5, n_max=5e5, d_min=10.0, d_max=20.0)
    ro = pp.RunOptions(mode="physical", g=0.95, t_max=100.0, hist_bins=100)
    res = propagator.propagate(b, ro)
    h, s, hist, steps, total = O.propagate(oracle_tables, to_oracle_pairs(b), to_oracle_opts(ro))
    assert total > 100
    g, o, ng, no = match_hits(res.hits, h)
    assert ng == 0 and no == 0, (ng, no)
    _check_matched(g, o, ng, no, "physical-cut")

"""The FP64 oracle against the reference's own known-answer tests
(src/tests/test_photon_prob.jl), the Random123 Philox vectors and the
committed oracle golden outputs.  CPU only."""
import json
import os

import numpy as np
import pytest

from oracle import oracle as O
from oracle import tables as tb

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
KATS = json.load(open(os.path.join(GOLDEN, "reference_kats.json")))
REF = KATS["reference"]
GOLD = json.load(open(os.path.join(GOLDEN, "oracle_golden.json")))


def _stream(n, seed=0):
    """n uniforms from the Philox stream the kernels use (photon i, block 0)."""
    out = []
    for i in range(n // 4 + 1):
        out.extend(O.uniform(w) for w in O.philox4x32_10([i, 0, 0, 0], [seed, 0]))
    return np.array(out[:n])


@pytest.mark.parametrize("kat", KATS["philox4x32_10"])
def test_philox_random123_vectors(kat):
    assert O.philox4x32_10(kat["ctr"], kat["key"]) == kat["out"]


@pytest.mark.parametrize("kat", KATS["philox2x32_10"])
def test_philox2x32_random123_vectors(kat):
    assert O.philox2x32_10(kat["ctr"], kat["key"]) == kat["out"]


def test_step_uniforms_bit_fields():
    # 21-bit fields 63..43, 42..22, 21..1 of w0:w1, each (k + 1/2) 2^-21
    for w0, w1 in ((0, 0), (0xFFFFFFFF, 0xFFFFFFFF), (0x80000000, 1), (0x12345678, 0x9ABCDEF0)):
        b = (w0 << 32) | w1
        want = [(((b >> s) & 0x1FFFFF) + 0.5) / 2**21 for s in (43, 22, 1)]
        got = O.step_uniforms([w0, w1])
        assert got == want
        assert all(0.0 < u < 1.0 and float(np.float32(u)) == u for u in got)


def test_step_uniforms_distribution():
    rng = np.random.default_rng(5)
    w = rng.integers(0, 2**32, size=(20000, 2), dtype=np.uint64)
    u = np.array([O.step_uniforms(O.philox2x32_10([int(a), int(b)], 7)) for a, b in w[:4000]])
    for j in range(3):
        assert abs(u[:, j].mean() - 0.5) < 0.015
        assert abs(u[:, j].var() - 1 / 12) < 0.005
    assert abs(np.corrcoef(u.T)[0, 1]) < 0.05 and abs(np.corrcoef(u.T)[1, 2]) < 0.05


def test_scatter_turn_frame():
    # physical-mode turn: unit output at polar angle acos(c) from the old
    # direction, and the same turn as rotate_to_axis up to an azimuth
    rng = np.random.default_rng(9)
    for _ in range(200):
        u = rng.normal(size=3)
        u /= np.linalg.norm(u)
        c = rng.uniform(-1, 1)
        phi = rng.uniform(0, 2 * np.pi)
        n = np.array([np.cos(phi) * np.sqrt(1 - c * c), np.sin(phi) * np.sqrt(1 - c * c), c])
        r = O.scatter_turn(u, n)
        assert abs(np.linalg.norm(r) - 1) < 1e-12
        assert abs(r @ u - c) < 1e-12
        r2 = O.rotate_to_axis(u, n)
        assert abs(r2 @ u - c) < 1e-12
    # the frame's first axis is the meridian: azimuth 0 tilts toward -z for an upward direction
    u = np.array([0.6, 0.0, 0.8])
    r = O.scatter_turn(u, [1.0, 0.0, 0.0])
    np.testing.assert_allclose(r, [0.8, 0.0, -0.6], atol=1e-12)


def test_uniform_open_interval_and_exact_float32():
    for w in (0, 1, 511, 512, 0x7FFFFFFF, 0xFFFFFFFF):
        u = O.uniform(w)
        assert 0.0 < u < 1.0
        assert float(np.float32(u)) == u  # exactly representable in FP32


def test_uniform_range():  # src/tests/test_photon_prob.jl:13-17
    k = REF["uniform_range"]
    u = _stream(k["n"])
    a, b = k["a"], k["b"]
    unis = a + u * (b - a)
    assert unis.min() >= a and unis.max() <= b


def test_hg_mean():  # src/tests/test_photon_prob.jl:19-21
    k = REF["hg_mean"]
    u = _stream(k["n"], seed=7)
    c = np.array([O.hg_costheta(k["g"], x) for x in u])
    assert abs(c.mean() - k["expected_mean"]) < k["atol"]
    assert c.min() >= -1 and c.max() <= 1


@pytest.mark.parametrize("name", ["rotate_identity", "rotate_flip", "rotate_y_to_minus_z"])
def test_rotate_to_axis_kats(name):  # src/tests/test_photon_prob.jl:24-41
    k = REF[name]
    r = O.rotate_to_axis(k["old"], k["new"])
    np.testing.assert_allclose(r, k["expected"], atol=1e-12)


def test_rotate_unit_norm():  # src/tests/test_photon_prob.jl:43-53
    k = REF["rotate_unit_norm"]
    a = np.array(k["old"]) / np.linalg.norm(k["old"])
    b = np.array(k["new"]) / np.linalg.norm(k["new"])
    assert abs(np.linalg.norm(O.rotate_to_axis(a, b)) - 1.0) < 1e-12


def rodrigues_rotation(a, b, operand):
    """rodrigues_rotation, src/photon_prop_cuda.jl:161-169."""
    ax = np.cross(a, b)
    axn = np.linalg.norm(ax)
    ax = ax / axn
    th = np.arcsin(axn)
    return operand * np.cos(th) + np.cross(ax, operand) * np.sin(th) + ax * (1 - np.cos(th)) * np.dot(ax, operand)


def test_rotate_vs_rodrigues():  # src/tests/test_photon_prob.jl:55-64
    k = REF["rotate_vs_rodrigues"]
    a = np.array(k["old"]) / np.linalg.norm(k["old"])
    u = _stream(64, seed=3)
    for i in range(0, 64, 2):
        ct = O.hg_costheta(k["g"], u[i])
        phi = 2 * np.pi * u[i + 1]
        st = np.sqrt(1 - ct * ct)
        new = np.array([np.cos(phi) * st, np.sin(phi) * st, ct])
        np.testing.assert_allclose(O.rotate_to_axis(a, new), rodrigues_rotation(np.array([0, 0, 1.0]), a, new),
                                   atol=1e-12)


def test_position_update():  # src/tests/test_photon_prob.jl:67-73
    k = REF["position_update"]
    np.testing.assert_allclose(O.update_position(k["pos"], k["dir"], k["step"]), k["expected"])


def test_interp_sorted_kats():  # src/tests/test_photon_prob.jl:75-85
    k = REF["interp_sorted"]
    for x, want in k["cases"]:
        assert O.interp_sorted(x, k["xs"], k["ys"]) == pytest.approx(want)
        assert float(tb.interp_sorted(x, k["xs"], k["ys"])) == pytest.approx(want)


def test_interp_sorted_lower_edge():
    # x == xs[1] (1-based) reads out of bounds in the reference; clamped here
    assert O.interp_sorted(0.0, [0.0, 1.0, 2.0], [5.0, 6.0, 7.0]) == 5.0


def test_interp_equidistant_kats():  # src/tests/test_photon_prob.jl:86-89
    k = REF["interp_equidistant"]
    for x, want in k["cases"]:
        assert O.interp_equidistant(x, k["knots"], k["lower"], k["upper"]) == pytest.approx(want)
        assert float(tb.interp_equidistant(x, k["knots"], k["lower"], k["upper"])) == pytest.approx(want)


def test_medium_spot_values_against_golden(oracle_medium):
    g = GOLD
    w = g["wavelengths"]
    np.testing.assert_allclose(tb.refractive_index(w, oracle_medium), g["refractive_index"], rtol=1e-14)
    np.testing.assert_allclose(tb.group_index(w, oracle_medium), g["group_index"], rtol=1e-14)
    np.testing.assert_allclose(tb.scattering_length(w, oracle_medium), g["scattering_length"], rtol=1e-14)
    np.testing.assert_allclose(tb.absorption_length(w), g["absorption_length"], rtol=1e-14)


def test_medium_physical_ranges(oracle_medium):
    # phase index 1.372 @300 -> 1.340 @800 nm; scattering 18.5 m @300, 37.7 @400, 129 m @800
    n = tb.refractive_index([300.0, 800.0], oracle_medium)
    assert n[0] == pytest.approx(1.372, abs=1e-3) and n[1] == pytest.approx(1.340, abs=1e-3)
    s = tb.scattering_length([300.0, 400.0, 800.0], oracle_medium)
    np.testing.assert_allclose(s, [18.5, 37.7, 129.1], rtol=2e-3)
    # group index exceeds phase index for normal dispersion
    assert np.all(tb.group_index(np.linspace(300, 800, 51), oracle_medium) >
                  tb.refractive_index(np.linspace(300, 800, 51), oracle_medium))


def test_spectrum_knots_golden_and_shape(oracle_medium):
    k = tb.cherenkov_spectrum_knots((300.0, 800.0), 20, oracle_medium)
    np.testing.assert_allclose(k, GOLD["cherenkov_knots_20"], rtol=1e-13)
    assert k[0] == 300.0 and k[-1] == 800.0 and np.all(np.diff(k) > 0)
    # 1/lambda^2 spectrum: the median wavelength sits well below the midpoint
    med = tb.interp_equidistant(0.5, k, 0.0, 1.0)
    assert 420 < med < 440


def test_gl50_exact_for_polynomials():
    # Gauss-Legendre with 50 nodes integrates polynomials up to degree 99 exactly
    assert tb.integrate_gauss_quad(lambda x: x ** 7 - 3 * x ** 2, -1.0, 2.0) == pytest.approx(
        (2 ** 8 - 1) / 8 - (8 + 1), rel=1e-12)


def _golden_tables():
    m = tb.cascadia(35.0, 2.0)
    knots = np.array(GOLD["cherenkov_knots_20"])
    pmt = tb.load_pmt_table(os.path.join(os.path.dirname(__file__), "..", "photonprop.jl_b200",
                                         "photonprop_b200", "data", "pmt_acceptance.csv"))
    return O.make_tables(m, knots, pmt=pmt)


def _cmp_hits(h, rows):
    assert len(rows) <= len(h)
    for r, want in zip(h, rows):
        assert int(r["photon"]) == want["photon"] and int(r["step"]) == want["step"]
        np.testing.assert_allclose(r["pos"], want["pos"], rtol=1e-12, atol=1e-12)
        assert r["time"] == pytest.approx(want["time"], rel=1e-12)
        assert r["weight"] == pytest.approx(want["weight"], rel=1e-12)


def test_oracle_compat_run_golden():
    g = GOLD["compat_run"]
    p = O.pairs_array(1)
    p[0]["target"] = g["pair"]["target"]
    p[0]["radius"] = g["pair"]["radius"]
    p[0]["n_photons"] = g["pair"]["n_photons"]
    h, s, _, steps, total = O.propagate(_golden_tables(), p, O.make_opts(mode=O.MODE_COMPAT, g=g["g"], hist_bins=0),
                                        n_threads=2)
    assert total == g["n_hits"] and steps == g["steps"]
    np.testing.assert_allclose(s[0], g["stats"], rtol=1e-12)
    _cmp_hits(h, g["first_hits"])


def test_oracle_physical_run_golden():
    g = GOLD["physical_run"]
    p = O.pairs_array(1)
    p[0]["target"] = g["pair"]["target"]
    p[0]["radius"] = g["pair"]["radius"]
    p[0]["n_photons"] = g["pair"]["n_photons"]
    o = O.make_opts(mode=O.MODE_PHYSICAL, g=g["g"], t_max=g["t_max"], hist_bins=500, flags=O.OPT_PMT_WEIGHT)
    h, s, hist, steps, total = O.propagate(_golden_tables(), p, o, n_threads=3)
    assert total == g["n_hits"] and steps == g["steps"]
    np.testing.assert_allclose(s[0], g["stats"], rtol=1e-12)
    _cmp_hits(h, g["hits"])
    for i, v in g["hist_nonzero"]:
        assert hist[0, i] == pytest.approx(v, rel=1e-12)


def test_oracle_thread_count_invariance():
    T = _golden_tables()
    p = O.pairs_array(2)
    p["target"] = [(0.0, 0.0, 5.0), (3.0, 0.0, 0.0)]
    p["radius"] = 0.21
    p["n_photons"] = [5000, 7000]
    p["seed"] = [11, 12]
    o = O.make_opts(mode=O.MODE_PHYSICAL, g=0.9, t_max=300.0, hist_bins=300)
    a = O.propagate(T, p, o, n_threads=1)
    b = O.propagate(T, p, o, n_threads=4)
    assert a[4] == b[4] and a[3] == b[3]
    np.testing.assert_array_equal(a[0], b[0])
    np.testing.assert_array_equal(a[1], b[1])


def test_oracle_empty_zero_photon_and_limited_pairs():
    """Edge cases the kernels are held to: pairs without photons add nothing
    and keep their rows zero; a photon limit replays exactly the first
    photons of each pair (the pilot launch of the fit stage relies on this)."""
    T = _golden_tables()
    o = O.make_opts(mode=O.MODE_PHYSICAL, g=0.9, t_max=300.0, hist_bins=300)
    h, s, hist, steps, total = O.propagate(T, O.pairs_array(0), o, n_threads=2)
    assert total == 0 and steps == 0 and len(h) == 0
    p = O.pairs_array(3)
    p["target"] = [(0.0, 0.0, 2.0), (0.0, 0.0, 2.0), (0.0, 2.5, 0.0)]
    p["radius"] = 0.21
    p["n_photons"] = [0, 4000, 3000]
    p["seed"] = [5, 6, 7]
    h, s, hist, steps, total = O.propagate(T, p, o, n_threads=2)
    assert total > 0 and not np.any(h["pair"] == 0)
    assert np.all(s[0] == 0.0) and np.all(hist[0] == 0.0)
    np.testing.assert_array_equal(s[:, 0], [np.sum(h["pair"] == k) for k in range(3)])
    hl, sl, _, _, total_l = O.propagate(T, p, o, photon_limit=1500, n_threads=2)
    full = h[h["photon"] < 1500]
    assert total_l == len(full)
    key = lambda a: np.lexsort((a["photon"], a["pair"]))  # noqa: E731
    np.testing.assert_array_equal(hl[key(hl)]["photon"], full[key(full)]["photon"])
    np.testing.assert_array_equal(hl[key(hl)]["pos"], full[key(full)]["pos"])


def test_oracle_flat_parallel_uses_every_thread():
    """The oracle's work is one flat index space of (pair, 256-photon chunk)
    items, so a batch of many pairs with fewer photons each than one chunk
    still keeps every requested thread busy, and the result does not depend
    on how the chunks fall on threads."""
    T = _golden_tables()
    rng = np.random.default_rng(3)
    p = O.pairs_array(64)
    p["target"] = rng.uniform(-3, 3, size=(64, 3))
    p["radius"] = 0.21
    p["n_photons"] = rng.integers(0, 700, size=64)
    p["seed"] = np.arange(64) + 100
    o = O.make_opts(mode=O.MODE_PHYSICAL, g=0.9, t_max=200.0, hist_bins=200)
    a = O.propagate(T, p, o, n_threads=1)
    assert O.last_threads_used == 1
    b = O.propagate(T, p, o, n_threads=4)
    assert O.last_threads_used == 4
    assert a[4] == b[4] > 0 and a[3] == b[3]
    np.testing.assert_array_equal(a[0], b[0])
    np.testing.assert_array_equal(a[1], b[1])
    np.testing.assert_array_equal(a[2], b[2])
    np.testing.assert_array_equal(b[1][:, 6], p["n_photons"])


def test_oracle_batch_generator_matches_product():
    """oracle/batches.py draws the benchmark batch without the product
    library (the CPU arm of the benchmark must not load it); it must be the
    product's batch number for number."""
    import photonprop_b200 as pp
    from oracle import batches as ob
    for seed, n in ((2024, 4096), (7, 33)):
        a = pp.batches.mixed_batch(n, seed=seed)
        b = ob.mixed_batch(n, seed=seed)
        for f in ("pos", "t0", "dir", "track_len", "target", "radius", "n_photons", "seed", "emitter"):
            np.testing.assert_array_equal(np.asarray(a[f], dtype=b[f].dtype), b[f], err_msg=f)
    idx = np.array([0, 1, 2, 4095, 2**40], dtype=np.uint64)
    for g in (0, 1, 2**63 + 5):
        np.testing.assert_array_equal(ob.pair_seed(g, idx), [pp.propagation.pair_seed(g, int(i)) for i in idx])
    wl, acc = ob.pmt_table()
    np.testing.assert_array_equal(wl, pp.p_one_pmt_acc.wavelengths)
    np.testing.assert_array_equal(acc, pp.p_one_pmt_acc.acceptance)
    s = ob.sampled(b, 1e-3)
    assert np.all(s["n_photons"] == np.minimum(b["n_photons"], np.maximum(1, np.ceil(b["n_photons"] * 1e-3))))

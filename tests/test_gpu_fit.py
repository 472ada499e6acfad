"""Fit stage on the device against the FP64 oracle (oracle/fits.py).

The fused path (pp_propagate_fit / pp_fit_hits_device) is checked on the
GPU's own hit records: the oracle recomputes every hit's Cherenkov weight,
arrival-time residual and the per-(pair, angle) moments in FP64 and fits
them.  Tolerances: moments rtol 2e-4 (the device evaluates the weight in
FP32 with MUFU exp2/log2; sums are FP64); Gamma fits from the same moments
rtol 1e-9 (both FP64 Newton); fits from oracle moments rtol 2e-3 (the
Gamma shape amplifies the moment error by 1 / (ln mean - mean ln))."""
import numpy as np
import pytest

import photonprop_b200 as pp
from photonprop_b200 import modelling as md
from oracle import fits as F
from oracle import tables as tb

pytestmark = pytest.mark.gpu

ANGLES = np.array([0.0, 0.4, 0.75, 1.2, 1.9, 2.6, np.pi])


def _pairs(mode):
    ds = [1.5, 2.5, 4.0, 6.0]
    return np.concatenate([pp.batches.point_source_pair(1_500_000, target=(0.0, 0.0, d), seed=pp.propagation.pair_seed(7, i))
                           for i, d in enumerate(ds)])


def _oracle_moments(hits, pairs, mode, om):
    n800 = tb.refractive_index(800.0, om) if mode == "compat" else tb.group_index(800.0, om)
    out = np.zeros((len(pairs), len(ANGLES), 4))
    tab = F.int_table()
    for p in range(len(pairs)):
        h = hits[hits["pair"] == p]
        d0 = h["dir0"].astype(np.float64)
        ct = np.clip(d0[:, 2], -1, 1)
        theta = np.arccos(ct)
        wl = h["wavelength"].astype(np.float64)
        n = tb.refractive_index(wl, om)
        d = np.linalg.norm(pairs["target"][p].astype(np.float64) - pairs["pos"][p].astype(np.float64))
        tgeo = (d - float(pairs["radius"][p])) * n800 / 0.299792458
        t0 = 0.0 if mode == "compat" else float(pairs["t0"][p])
        tres = h["time"].astype(np.float64) - t0 - tgeo
        w = h["weight"].astype(np.float64)
        for j, a in enumerate(ANGLES):
            out[p, j] = F.moments(tres, F.get_dir_reweight(theta, a, n, tab) * w)
    return out


@pytest.mark.parametrize("mode", ["compat", "physical"])
def test_fused_fit_matches_oracle_on_the_same_hits(propagator, oracle_medium, mode):
    pairs = _pairs(mode)
    ro = pp.RunOptions(mode=mode, pmt_weight=True, hist_bins=0, t_max=300.0)
    res = propagator.propagate(pairs, ro, hit_capacity=1 << 21)
    assert not res.overflow and res.n_hits > 2000
    fr = md.propagate_fit(propagator, pairs, ANGLES, ro)
    assert fr.n_hits == res.n_hits
    np.testing.assert_allclose(fr.stats, res.stats, rtol=1e-9)
    ref = _oracle_moments(res.hits, pairs, mode, oracle_medium)
    np.testing.assert_allclose(fr.moments, ref, rtol=2e-4, atol=1e-12)
    for p in range(len(pairs)):
        for j in range(len(ANGLES)):
            m = fr.moments[p, j]
            a, th = F.gamma_fit_moments(m[1], m[2], m[3])
            np.testing.assert_allclose(fr.fits[p, j, :2], [a, th], rtol=1e-9)
            assert fr.fits[p, j, 2] == pytest.approx(m[0] / pairs["n_photons"][p], rel=1e-12)
            ra, rth = F.gamma_fit_moments(*ref[p, j, 1:])
            np.testing.assert_allclose(fr.fits[p, j, :2], [ra, rth], rtol=2e-3)


def test_device_fit_over_device_hits(propagator):
    import torch
    pairs = _pairs("compat")
    ro = pp.RunOptions(mode="compat", pmt_weight=True, hist_bins=0)
    fr = md.propagate_fit(propagator, pairs, ANGLES, ro)
    cap = 1 << 21
    d_pairs = torch.from_numpy(pairs.view(np.uint8).copy()).cuda()
    d_hits = torch.empty(cap * 64, dtype=torch.uint8, device="cuda")
    d_cnt = torch.zeros(4, dtype=torch.int64, device="cuda")
    d_stats = torch.zeros((len(pairs), 8), dtype=torch.float64, device="cuda")
    propagator.propagate_device(d_pairs, len(pairs), ro, d_hits, cap, d_cnt, d_stats, None,
                                stream=torch.cuda.current_stream())
    d_m = torch.zeros((len(pairs), len(ANGLES), 4), dtype=torch.float64, device="cuda")
    d_f = torch.zeros((len(pairs), len(ANGLES), 3), dtype=torch.float64, device="cuda")
    L = pp._lib.load()
    pp._lib.check(L.pp_fit_hits_device(propagator.handle, d_pairs.data_ptr(), len(pairs), pp._lib.MODE_COMPAT,
                                       d_hits.data_ptr(), cap, d_cnt.data_ptr(), ANGLES.ctypes.data, len(ANGLES),
                                       d_m.data_ptr(), d_f.data_ptr(), torch.cuda.current_stream().cuda_stream),
                  propagator.handle)
    torch.cuda.synchronize()
    np.testing.assert_allclose(d_m.cpu().numpy(), fr.moments, rtol=1e-12)
    np.testing.assert_allclose(d_f.cpu().numpy(), fr.fits, rtol=1e-9)


def test_fit_photon_dist_over_columns_matches_oracle(propagator):
    import pandas as pd
    rng = np.random.default_rng(3)
    n = 40000
    wl = rng.uniform(300.0, 700.0, n)
    df = pd.DataFrame({"tres": rng.gamma(2.5, 6.0, n) - 1.0, "initial_theta": rng.uniform(0, np.pi, n),
                       "ref_ix": rng.uniform(1.33, 1.36, n), "abs_weight": rng.uniform(0.05, 1.0, n),
                       "dist_travelled": rng.uniform(1, 20, n), "wavelength": wl})
    out = md.fit_photon_dist(ANGLES, df, 10_000_000, propagator=propagator)
    assert list(out.columns) == ["obs_angle", "fit_alpha", "fit_theta", "det_fraction"]
    pmt = np.interp(wl, pp.p_one_pmt_acc.wavelengths, pp.p_one_pmt_acc.acceptance)
    rows, _ = F.fit_photon_dist(ANGLES, df["tres"].to_numpy(), df["initial_theta"].to_numpy(),
                                df["ref_ix"].to_numpy(), df["abs_weight"].to_numpy(), pmt, 10_000_000)
    np.testing.assert_allclose(out.to_numpy(), rows, rtol=2e-4)


def test_gamma_fit_recovers_sample_mle(propagator):
    import pandas as pd
    from scipy import stats
    rng = np.random.default_rng(4)
    x = rng.gamma(3.5, 4.0, 50000)
    n = len(x)
    df = pd.DataFrame({"tres": x, "initial_theta": np.full(n, 0.8), "ref_ix": np.full(n, 1.34),
                       "abs_weight": np.ones(n), "wavelength": np.full(n, 420.0)})
    out = md.fit_photon_dist([0.3], df, n, propagator=propagator)
    sa, _, sth = stats.gamma.fit(x, floc=0)
    assert out["fit_alpha"][0] == pytest.approx(sa, rel=1e-4)
    assert out["fit_theta"][0] == pytest.approx(sth, rel=1e-4)


def test_make_photon_fits_table(propagator, tmp_path):
    df = md.make_photon_fits(300_000, 3, 4, 30.0, propagator=propagator, seed=2)
    assert list(df.columns) == ["obs_angle", "fit_alpha", "fit_theta", "det_fraction", "distance"]
    assert len(df) == 12
    s2 = md.SobolSeq(0.0, float(np.float32(np.log10(np.float32(30.0)))))
    dist = [np.float32(10 ** s2.next()) for _ in range(3)]
    np.testing.assert_allclose(df["distance"].to_numpy(), np.repeat(dist, 4), rtol=1e-7)
    np.testing.assert_allclose(df["obs_angle"].to_numpy()[:4], [np.pi / 2, 0.75 * np.pi, 0.25 * np.pi, 0.375 * np.pi])
    assert np.isfinite(df["fit_alpha"]).all() and (df["det_fraction"] > 0).all()
    # closer spheres catch more light
    det = df.groupby("distance")["det_fraction"].sum()
    assert det.sort_index().is_monotonic_decreasing
    md.write_fit_table(df, tmp_path / "fits.parquet")
    back = md.read_parquet(tmp_path / "fits.parquet")
    np.testing.assert_array_equal(back.to_numpy(), df.to_numpy())


@pytest.mark.parametrize("n_photons,n_pairs", [(1_000_000, 8), (60_000, 16)])
def test_waves_match_one_launch(propagator, n_photons, n_pairs):
    """Waves planned from the pilot launch's estimates (1e6 photons per pair),
    and waves planned from geometry alone (pairs too small for a pilot), whose
    first wave overflows and is repacked with the exact counts."""
    pairs = np.concatenate([pp.batches.point_source_pair(n_photons, target=(0.0, 0.0, 3.0),
                                                         seed=pp.propagation.pair_seed(11, i)) for i in range(n_pairs)])
    ro = pp.RunOptions(mode="compat", pmt_weight=True, hist_bins=0)
    one = md.propagate_fit(propagator, pairs, ANGLES, ro, hit_capacity=1 << 21)
    assert one.n_hits < 1 << 21
    waves = md.propagate_fit(propagator, pairs, ANGLES, ro, hit_capacity=one.n_hits // 3)
    assert waves.n_hits == one.n_hits
    np.testing.assert_allclose(waves.stats, one.stats, rtol=1e-9)
    np.testing.assert_allclose(waves.moments, one.moments, rtol=1e-9)
    np.testing.assert_allclose(waves.fits, one.fits, rtol=1e-7)

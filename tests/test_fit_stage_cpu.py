"""Fit stage on the CPU: the oracle's restatement of the reference's
Cherenkov angular distribution, its closed-form integral and the weighted
Gamma fit, pinned against independent computations (quadrature, scipy's
Gamma MLE); the library's FP64 host functions against the oracle; the Sobol
points; the fit-table Parquet I/O."""
import numpy as np
import pytest
from scipy import integrate, stats

import photonprop_b200 as pp
from photonprop_b200 import modelling as md
from oracle import fits as F


@pytest.mark.parametrize("n", [1.1, 1.25, 1.33, 1.34, 1.35, 1.5])
def test_closed_form_integral_is_quadrature_plus_the_reference_join(n):
    c0 = 1.0 / n
    f = lambda x: F.cherenkov_ang_dist(x, n)
    q = integrate.quad(f, -1, c0, limit=200, epsabs=1e-13)[0] + integrate.quad(f, c0, 1, limit=200, epsabs=1e-13)[0]
    assert F.cherenkov_ang_dist_int_exact(n) == pytest.approx(q + F.join_offset(n), rel=1e-10)
    # the join makes the reference's normalisation about 1 % smaller than the true integral
    assert 0.005 < (q - F.cherenkov_ang_dist_int_exact(n)) / q < 0.02


def test_interpolated_integral_hits_the_nodes():
    t = F.int_table()
    for i in (0, 7, 24, 40):
        n = F.INT_N0 + F.INT_DN * i
        assert F.cherenkov_ang_dist_int(n, t) == pytest.approx(F.cherenkov_ang_dist_int_exact(n), rel=1e-12)
    assert np.isnan(F.cherenkov_ang_dist_int(1.05, t)) and np.isnan(F.cherenkov_ang_dist_int(1.51, t))


def test_oracle_gamma_fit_matches_scipy_mle():
    rng = np.random.default_rng(5)
    for a, th in [(1.7, 3.0), (4.5, 0.8), (25.0, 2.0)]:
        x = rng.gamma(a, th, size=20000)
        sa, _, sth = stats.gamma.fit(x, floc=0)
        oa, oth = F.gamma_fit(x, np.ones_like(x))
        assert oa == pytest.approx(sa, rel=1e-4) and oth == pytest.approx(sth, rel=1e-4)
        # integer weights are replicated samples
        w = rng.integers(1, 4, size=2000)
        xr = np.repeat(x[:2000], w)
        sa, _, sth = stats.gamma.fit(xr, floc=0)
        oa, oth = F.gamma_fit(x[:2000], w)
        assert oa == pytest.approx(sa, rel=1e-4) and oth == pytest.approx(sth, rel=1e-4)


def test_library_host_functions_match_oracle():
    rng = np.random.default_rng(1)
    ct = rng.uniform(-1, 1, 200)
    n = rng.uniform(1.1, 1.5, 200)
    np.testing.assert_allclose(md.cherenkov_ang_dist(ct, n), F.cherenkov_ang_dist(ct, n), rtol=1e-13)
    np.testing.assert_allclose(md.cherenkov_ang_dist_int(n), F.cherenkov_ang_dist_int(n), rtol=1e-12)
    for x in (1.1, 1.3, 1.34, 1.5):
        assert md.cherenkov_ang_dist_int(x, -1.0, 1.0) == pytest.approx(F.cherenkov_ang_dist_int_exact(x), rel=1e-12)
        assert md.cherenkov_ang_dist_int(x, -0.3, 0.6) == pytest.approx(
            F.cherenkov_ang_dist_int_exact(x, -0.3, 0.6), rel=1e-12)
    with pytest.raises(ValueError):
        md.cherenkov_ang_dist_int(1.6)
    th = rng.uniform(0, np.pi, 500)
    for a in (0.0, 0.7, 2.5):
        np.testing.assert_allclose(md.get_dir_reweight(th, a, n[0]), F.get_dir_reweight(th, a, n[0]), rtol=1e-12)


def test_sobol_points_are_sobol_jl_first_dimension():
    from scipy.stats import qmc
    ref = qmc.Sobol(1, scramble=False).random_base2(7)[1:65, 0]  # Sobol.jl skips the initial 0
    s = md.SobolSeq(0.0, 1.0)
    np.testing.assert_array_equal([s.next() for _ in range(64)], ref)
    s = md.SobolSeq(0.0, np.pi)
    assert [s.next() for _ in range(3)] == pytest.approx([np.pi / 2, 0.75 * np.pi, 0.25 * np.pi])


def test_fit_table_parquet_round_trip(tmp_path):
    import pandas as pd
    rng = np.random.default_rng(2)
    n = 500
    df = pd.DataFrame({"obs_angle": rng.uniform(0, np.pi, n), "fit_alpha": rng.uniform(1, 50, n),
                       "fit_theta": rng.uniform(0.1, 10, n), "det_fraction": 10 ** rng.uniform(-9, -2, n),
                       "distance": 10 ** rng.uniform(0, 2.4, n)})
    p = tmp_path / "photon_fits.parquet"
    md.write_fit_table(df, p)
    back = md.read_parquet(p)
    assert list(back.columns) == list(md.FIT_TABLE_COLUMNS)
    np.testing.assert_array_equal(back.to_numpy(), df[list(md.FIT_TABLE_COLUMNS)].to_numpy())
    ftr, ttr, fte, tte = md.read_from_parquet(p, rng=np.random.default_rng(0))
    assert ftr.shape[0] == 2 and ttr.shape[0] == 3 and ftr.shape[1] + fte.shape[1] == n
    assert ftr.shape[1] == int(0.8 * n) and ftr.dtype == np.float32
    # the transforms of get_data, and their inverses
    tr = md.default_trafos()
    d32 = df.astype(np.float32)
    allf = np.concatenate([ftr, fte], axis=1)
    got = np.sort(allf[0])
    np.testing.assert_allclose(got, np.sort(np.log10(d32["distance"].to_numpy())), rtol=1e-6)
    t = tr[("det_fraction", "log_det_fraction_scaled")]
    x = d32["det_fraction"].to_numpy().astype(np.float64)
    np.testing.assert_allclose(md.reverse_transformation(md.apply_transformation(x, t), t), x, rtol=1e-12)


def test_cascade_sampler_matches_oracle_and_profile():
    """The library's FP64 cascade sampler equals the oracle's (independent
    tables), and samples drawn on a fine grid of u follow the normalised
    profile a exp(b |x - 1/n|^c) + d on [-1, 1] (quadrature CDF)."""
    L = pp._lib.load()
    rng = np.random.default_rng(3)
    for u, n in zip(rng.uniform(size=200), rng.uniform(1.3, 1.4, size=200)):
        assert L.pp_cascade_cos_theta(u, n) == pytest.approx(float(F.cascade_cos_theta(u, n)), abs=1e-12)
    n = 1.34
    us = (np.arange(200000) + 0.5) / 200000
    x = np.sort(F.cascade_cos_theta(us, np.full_like(us, n)))
    f = lambda t: F.cherenkov_ang_dist(t, n)
    c0 = 1 / n
    tot = integrate.quad(f, -1, c0, limit=200)[0] + integrate.quad(f, c0, 1, limit=200)[0]
    for q in (-0.5, 0.0, 0.5, 0.7, c0, 0.78, 0.9):
        cdf = (integrate.quad(f, -1, min(q, c0), limit=200)[0]
               + (integrate.quad(f, c0, q, limit=200)[0] if q > c0 else 0.0)) / tot
        assert np.searchsorted(x, q) / len(x) == pytest.approx(cdf, abs=2e-4)


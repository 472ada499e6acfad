"""Light yield on the CPU: the library's FP64 host functions (shower
profile, track length, Frank-Tamm normalisation, fractional contributions,
water density) against the oracle (oracle/lightyield.py), which uses numpy's
Gauss-Legendre nodes and scipy's Gamma function."""
import numpy as np
import pytest

import photonprop_b200 as pp
from photonprop_b200 import lightyield as ly
from oracle import lightyield as OL
from oracle import tables as tb


@pytest.fixture(scope="module")
def media():
    return pp.make_cascadia_medium_properties(), tb.cascadia()


@pytest.mark.parametrize("mode", ["reference", "metres"])
def test_density_and_profile(media, mode):
    m, om = media
    assert ly.medium_density(m, mode) == pytest.approx(OL.density(om, mode), rel=1e-13)
    if mode == "metres":
        assert 1000.0 < ly.medium_density(m, mode) < 1030.0  # water near 2 degC
    else:
        assert ly.medium_density(m, mode) == pytest.approx(12.849, rel=1e-3)  # the reference's expression
    z = np.array([1.0, 10.0, 100.0, 500.0, 3000.0])
    for pt in ly.ParticleType:
        for e in (1.0, 1e3, 1e5):
            np.testing.assert_allclose(ly.longitudinal_profile(e, z, m, pt, mode),
                                       OL.longitudinal_profile(e, z, om, pt, mode), rtol=1e-12)


def test_track_length_and_frank_tamm(media):
    m, om = media
    for pt in ly.ParticleType:
        for e in (0.5, 10.0, 1e4):
            assert ly.cherenkov_track_length(e, pt) == pytest.approx(OL.cherenkov_track_length(e, pt), rel=1e-14)
            assert ly.cherenkov_track_length_dev(e, pt) == pytest.approx(OL.cherenkov_track_length_dev(e, pt),
                                                                         rel=1e-14)
    assert ly.frank_tamm_norm((300.0, 800.0), m) == pytest.approx(tb.frank_tamm_norm((300.0, 800.0), om), rel=1e-12)
    assert np.isnan(pp._lib.load().pp_cherenkov_track_length(13, 1.0))


@pytest.mark.parametrize("mode", ["reference", "metres"])
def test_fractional_contrib(media, mode):
    m, om = media
    grid = np.arange(0.0, 3001.0, 50.0) if mode == "reference" else np.arange(0.0, 20.01, 0.25) * 100
    for pt in ly.ParticleType:
        a = ly.fractional_contrib_long(1e3, grid, m, pt, mode)
        b = OL.fractional_contrib_long(1e3, grid, om, pt, mode)
        np.testing.assert_allclose(a, b, rtol=1e-10, atol=1e-300)
        assert a[0] == 0.0 and abs(a.sum() - 1.0) < 1e-6


def test_point_lightsource(media):
    m, _ = media
    p = ly.Particle((0.0, 0.0, 0.0), (0.0, 0.0, 1.0), 0.0, 1e3, ly.ParticleType.EMinus)
    s = ly.particle_to_lightsource(p, m, (300.0, 800.0))
    assert s.photons == round(ly.frank_tamm_norm((300.0, 800.0), m) * ly.cherenkov_track_length(1e3, p.type))

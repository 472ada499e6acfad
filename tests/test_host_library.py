"""The C-ABI library on the host (no GPU): it loads, exports every symbol the
header declares, and its FP64 host physics agrees with the oracle."""
import ctypes
import os
import re

import numpy as np
import pytest

import photonprop_b200 as pp
from photonprop_b200 import _lib
from oracle import tables as tb

HEADER = os.path.join(os.path.dirname(__file__), "..", "include", "photonprop_b200.h")


def header_functions():
    src = open(HEADER).read()
    return sorted(set(re.findall(r"PP_API\s+[\w\s\*]+?\b(pp_\w+)\s*\(", src)))


def test_library_exports_every_header_symbol():
    L = _lib.load()
    names = header_functions()
    assert len(names) >= 20
    for n in names:
        assert hasattr(L, n), n
    assert sorted(_lib.EXPORTED) == names


def test_struct_layouts_match_header():
    assert _lib.PAIR_DTYPE.itemsize == 80
    assert _lib.HIT_DTYPE.itemsize == 64
    assert ctypes.sizeof(_lib.RunOpts) == 48
    assert ctypes.sizeof(_lib.MediumDesc) == 6 * 8 + 8 + 2 * 32 * 8
    assert ctypes.sizeof(_lib.PmtDesc) == 8 + 2 * 256 * 8


def test_abi_version_and_launch_counter():
    L = _lib.load()
    assert L.pp_abi_version() == 1
    assert b"sm_100a" in L.pp_version()
    assert pp.launch_count() >= 0


@pytest.mark.parametrize("wl", [300.0, 333.3, 400.0, 512.0, 650.0, 800.0])
def test_host_medium_matches_oracle(medium, oracle_medium, wl):
    assert pp.get_refractive_index(wl, medium) == pytest.approx(float(tb.refractive_index(wl, oracle_medium)),
                                                                rel=1e-14)
    assert pp.get_group_index(wl, medium) == pytest.approx(float(tb.group_index(wl, oracle_medium)), rel=1e-14)
    assert pp.get_scattering_length(wl, medium) == pytest.approx(
        float(tb.scattering_length(wl, oracle_medium)), rel=1e-13)
    assert pp.get_absorption_length(wl, medium) == pytest.approx(float(tb.absorption_length(wl)), rel=1e-14)


def test_host_knots_match_oracle(medium, oracle_medium):
    for n in (2, 5, 20, 64):
        k = pp.CherenkovSpectrum((300.0, 800.0), n, medium).knots
        np.testing.assert_allclose(k, tb.cherenkov_spectrum_knots((300.0, 800.0), n, oracle_medium), rtol=1e-12)


def test_cascadia_medium():
    m = pp.make_cascadia_medium_properties()
    assert m.salinity == 34.82 and m.temperature == 1.8
    assert m.pressure == pytest.approx(269.44088 / 1.01325)
    assert m.vol_conc_small_part == 0.0075 and m.vol_conc_large_part == 0.0075


def test_pmt_acceptance_table():
    t = pp.p_one_pmt_acc
    assert len(t.wavelengths) == 57  # PMTAcc.csv rows
    i = int(np.argmax(t.acceptance))
    assert t.wavelengths[i] == pytest.approx(402.42, abs=0.01) and t.acceptance[i] == pytest.approx(0.2708, abs=1e-4)
    xs = np.linspace(250, 750, 37)
    np.testing.assert_allclose(t(xs), tb.pmt_acceptance(xs, (t.wavelengths, t.acceptance)), rtol=1e-14, atol=1e-16)
    t5 = pp.p_one_pmt_acc_5nm
    assert len(t5.wavelengths) == 81 and t5.wavelengths[0] == 300 and t5.wavelengths[-1] == 700
    np.testing.assert_allclose(t5.acceptance, t(t5.wavelengths), rtol=1e-12)


def test_custom_absorption_table(medium):
    m = pp.WaterProperties(35.0, 265.9, 2.0, 0.0075, 0.0075, absorption_table=([300.0, 800.0], [10.0, 20.0]))
    assert pp.get_absorption_length(550.0, m) == pytest.approx(15.0)
    with pytest.raises(ValueError):
        pp.WaterProperties(35.0, 265.9, 2.0, 0.0075, 0.0075, absorption_table=([800.0, 300.0], [1.0, 2.0])).desc()


def test_pair_seed_is_deterministic_and_distinct():
    a = [pp.pair_seed(0, i) for i in range(1000)]
    assert len(set(a)) == 1000
    assert a == [pp.pair_seed(0, i) for i in range(1000)]
    assert pp.pair_seed(1, 0) != pp.pair_seed(0, 0)


def test_default_opts():
    o = pp.RunOptions(mode="compat").to_c()
    assert (o.mode, o.max_steps, o.hist_bins) == (0, 10, 0)
    assert o.g == pytest.approx(0.99)
    o = pp.RunOptions(mode="physical").to_c()
    assert (o.mode, o.max_steps, o.hist_bins, o.flags) == (1, 1000, 500, 1)
    assert o.g == pytest.approx(0.95) and o.t_max == 500.0
    o = pp.RunOptions(mode="physical", pmt_weight=False, normalize=True, write_hits=False, g=0.5).to_c()
    assert o.flags == 2 | 4 and o.g == pytest.approx(0.5)
    # the cascade-emitter kernel variant is a flag the device entry points take from the caller
    o = pp.RunOptions(mode="physical", cascade=True, block_size=128, blocks_per_sm=6, chunk_photons=4096).to_c()
    assert o.flags == 1 | 16 and (o.block_size, o.blocks_per_sm, o.chunk_photons) == (128, 6, 4096)
    with pytest.raises(ValueError):
        pp.RunOptions(mode="nope").to_c()


def test_process_output_reference_semantics():
    # two blocks of stack 4: block 0 holds 2 hits (1-based pointer 2), block 1 none
    out = np.arange(8.0)
    np.testing.assert_array_equal(pp.process_output(out, [2, 0]), [0.0, 1.0])
    np.testing.assert_array_equal(pp.process_output(out, [0, 7]), [4.0, 5.0, 6.0])
    np.testing.assert_array_equal(pp.process_output(out, [4, 8]), out)
    assert len(pp.process_output(out, [0, 0])) == 0


def test_mixed_batch_shape():
    b = pp.batches.mixed_batch(512, seed=3)
    n = b["n_photons"]
    assert n.min() >= 1e4 and n.max() <= 1e7
    d = np.linalg.norm(b["target"], axis=1)
    assert d.min() >= 2.0 and d.max() <= 150.0
    cone = b["emitter"] == 1
    assert 0.35 < cone.mean() < 0.65
    np.testing.assert_allclose(np.linalg.norm(b["dir"], axis=1), 1.0, rtol=1e-6)
    assert len(set(b["seed"].tolist())) == 512
    # reproducible
    b2 = pp.batches.mixed_batch(512, seed=3)
    assert b.tobytes() == b2.tobytes()


def test_cone_grid_pairs():
    g = pp.batches.cone_grid_pairs(n_photons=1000)
    assert len(g) == 25
    mid = np.array([0, 0, 0.5])
    d = np.linalg.norm(g["target"] - mid, axis=1)
    np.testing.assert_allclose(sorted(set(np.round(d, 4))), [5, 10, 20, 50, 100])


def test_create_without_gpu_fails_loudly(medium):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    spec = pp.CherenkovSpectrum((300.0, 800.0), 20, medium)
    with pytest.raises(pp.PPError):
        pp.Propagator(medium, spec)

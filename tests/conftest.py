import os
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG_ROOT = os.path.join(REPO, "photonprop.jl_b200")
for p in (REPO, PKG_ROOT):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


HAS_GPU = _has_gpu()


def pytest_collection_modifyitems(config, items):
    if HAS_GPU:
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


@pytest.fixture(scope="session")
def medium():
    import photonprop_b200 as pp
    return pp.make_seawater(35.0, 2.0)


@pytest.fixture(scope="session")
def oracle_medium():
    from oracle import tables as tb
    return tb.cascadia(35.0, 2.0)


@pytest.fixture(scope="session")
def propagator(medium):
    import photonprop_b200 as pp
    spec = pp.CherenkovSpectrum((300.0, 800.0), 20, medium)
    prop = pp.Propagator(medium, spec, pp.p_one_pmt_acc, device=0)
    yield prop
    prop.close()


@pytest.fixture(scope="session")
def oracle_tables(propagator, oracle_medium):
    """Oracle tables with the device's float knots (so both draw the same
    wavelength from the same uniform)."""
    import numpy as np
    import photonprop_b200 as pp
    from oracle import oracle as O
    knots = propagator.knots().astype(np.float64)
    pmt = (pp.p_one_pmt_acc.wavelengths, pp.p_one_pmt_acc.acceptance)
    return O.make_tables(oracle_medium, knots, pmt=pmt)

"""Event likelihood on the CPU: the reference's model features and the
oracle's likelihood against a direct evaluation."""
import numpy as np
import pytest
from scipy import stats

import photonprop_b200 as pp
from photonprop_b200 import event as ev
from oracle import event as OE


def test_source_to_input_reference_features():
    src = np.zeros(2, dtype=pp._lib.PAIR_DTYPE)
    src["pos"] = [(0, 0, 0), (0, 0, 10)]
    src["dir"] = [(0, 0, 1), (1, 0, 0)]
    tg = np.array([[3.0, 0.0, 4.0], [0.0, 0.0, -10.0]])
    x = ev.source_to_input(src, tg)
    assert x.shape == (2, 4)
    np.testing.assert_allclose(x[0], np.log10([5.0, 10.0, np.hypot(3, 6), 20.0]), rtol=1e-6)
    # emitter-receiver vector from the target to the source, as the reference has it
    v = np.array([[0, 0, 0], [0, 0, 0], [0, 0, 10], [0, 0, 10]], float) - tg[[0, 1, 0, 1]]
    d = np.array([[0, 0, 1], [0, 0, 1], [1, 0, 0], [1, 0, 0]], float)
    np.testing.assert_allclose(x[1], np.einsum("ij,ij->i", v / np.linalg.norm(v, axis=1)[:, None], d), atol=1e-6)




def test_oracle_module_llh_single_gamma():
    x = np.array([3.0, 7.5, 12.0])
    p = np.array([[2.0, 1.0, 3.0, 0.0, 2.5, 1.0]])
    got = OE.module_llh(p, x, photons=np.array([4.0]), mode="shifted")
    ref = stats.poisson.logpmf(3, 8.0) + np.sum(stats.gamma.logpdf(x - 1.0, 3.0, scale=2.5))
    assert got == pytest.approx(ref, rel=1e-12)

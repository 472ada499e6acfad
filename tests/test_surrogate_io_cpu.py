"""Trained-surrogate files (write_weights / read_weights): round trip and
rejection of files that do not fit the network.  CPU only; the GPU test
(test_gpu_surrogate.py) checks that a loaded network answers like the saved one."""
import numpy as np
import pytest

from photonprop_b200 import surrogate as sg


def _arrays(n=1000, seed=0):
    rng = np.random.default_rng(seed)
    return (rng.normal(size=n).astype(np.float32), rng.normal(size=18).astype(np.float32),
            np.array([0.3, -1.0, 4.0, 0.0], np.float32), np.array([2.2, 1.0, 7.0, 2.0], np.float32))


def test_round_trip(tmp_path):
    p, norm, lo, hi = _arrays()
    f = tmp_path / "net.bin"
    sg.write_weights(f, p, norm, lo, hi)
    assert f.stat().st_size == 24 + 4 * (26 + p.size)
    q, norm2, lo2, hi2 = sg.read_weights(f, n_params=p.size)
    for a, b in ((p, q), (norm, norm2), (lo, lo2), (hi, hi2)):
        np.testing.assert_array_equal(a, b)


def test_rejects_foreign_and_damaged_files(tmp_path):
    p, norm, lo, hi = _arrays(64)
    good = tmp_path / "net.bin"
    sg.write_weights(good, p, norm, lo, hi)
    blob = good.read_bytes()
    bad_magic = tmp_path / "magic.bin"
    bad_magic.write_bytes(b"XXXXXXXX" + blob[8:])
    truncated = tmp_path / "short.bin"
    truncated.write_bytes(blob[:-4])
    for f in (bad_magic, truncated):
        with pytest.raises(ValueError):
            sg.read_weights(f)
    with pytest.raises(ValueError):  # another network size
        sg.read_weights(good, n_params=65)
    with pytest.raises(ValueError):
        sg.write_weights(tmp_path / "x.bin", p, norm[:17], lo, hi)

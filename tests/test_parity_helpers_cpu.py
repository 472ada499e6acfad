"""The reconciliation checks of _parity.py on CPU, with the oracle's own
output standing in for the kernel's: they pass on equal tables and fail on a
mistake planted in the oracle's tables."""
import numpy as np
import pytest

import photonprop_b200 as pp
from oracle import oracle as O
from oracle import tables as tb

from _parity import check_pair_statistics_and_histograms, to_oracle_opts, to_oracle_pairs


class _Result:
    def __init__(self, hits, stats, hist, n):
        self.hits, self.stats, self.hist, self.n_hits, self.overflow = hits, stats, hist, n, False


def _run():
    m = tb.cascadia(35.0, 2.0)
    knots = tb.cherenkov_spectrum_knots((300.0, 800.0), 20, m).astype(np.float32).astype(np.float64)
    T = O.make_tables(m, knots)
    pairs = pp.batches.mixed_batch(6, seed=3, n_min=2e4, n_max=6e4, d_min=2.0, d_max=4.0)
    ro = pp.RunOptions(mode="physical", g=0.95, t_max=200.0, hist_bins=200, pmt_weight=False)
    oo = to_oracle_opts(ro)
    h, s, hist, _, total = O.propagate(T, to_oracle_pairs(pairs), oo)
    g = np.zeros(len(h), dtype=pp.HIT_DTYPE)
    for f in ("pos", "time", "dir0", "weight", "dir", "wavelength", "dist", "pair", "photon"):
        g[f] = h[f]
    return _Result(g, s.copy(), hist.copy(), total), h, s, hist, oo


def test_reconciliation_accepts_equal_tables():
    res, h, s, hist, oo = _run()
    assert len(h) > 50
    check_pair_statistics_and_histograms(res, h, s, hist, len(s), oo.hist_t0, oo.hist_bin_width, oo.hist_bins,
                                         "equal")
    # a rim flip on the kernel's side: one hit fewer there, its sums and bin with it
    drop = 0
    keep = np.ones(len(res.hits), dtype=bool)
    keep[drop] = False
    p, t, w = int(h["pair"][drop]), h["time"][drop], h["weight"][drop]
    res2 = _Result(res.hits[keep], s.copy(), hist.copy(), res.n_hits - 1)
    res2.stats[p, 0] -= 1
    res2.stats[p, 1] -= w
    res2.hist[p, int(np.floor(t))] -= w
    check_pair_statistics_and_histograms(res2, h, s, hist, len(s), oo.hist_t0, oo.hist_bin_width, oo.hist_bins,
                                         "flip")


@pytest.mark.parametrize("what", ["bin", "count", "weight"])
def test_reconciliation_rejects_planted_mistakes(what):
    res, h, s, hist, oo = _run()
    s2, hist2 = s.copy(), hist.copy()
    p = int(h["pair"][0])
    b = int(np.floor(h["time"][0]))
    if what == "bin":  # a hit's weight in the neighbouring bin
        hist2[p, b] -= h["weight"][0]
        hist2[p, b + 1] += h["weight"][0]
    elif what == "count":
        s2[p, 0] += 1
    else:
        s2[p, 1] *= 1.01
    with pytest.raises(AssertionError):
        check_pair_statistics_and_histograms(res, h, s2, hist2, len(s), oo.hist_t0, oo.hist_bin_width,
                                             oo.hist_bins, what)

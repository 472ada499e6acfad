"""Continuous-batching serving loop (pp_server_* through the C ABI)."""
import numpy as np
import pytest

import photonprop_b200 as pp
from photonprop_b200 import serving

pytestmark = pytest.mark.gpu

OPTS = pp.RunOptions(mode="physical", t_max=400.0, hist_bins=400)


def _key(h):
    return np.lexsort((h["photon_lo"], h["pair"]))


def test_request_alone_equals_request_in_the_mix(propagator):
    req = pp.batches.mixed_batch(8, seed=501, n_min=1e5, n_max=1e6, d_min=2.0, d_max=10.0)
    others = [pp.batches.mixed_batch(int(n), seed=600 + i, n_min=1e4, n_max=1e6)
              for i, n in enumerate(np.random.default_rng(0).integers(1, 64, 40))]
    with serving.Server(propagator, OPTS) as srv:
        alone = srv.result(srv.submit(req))
        ids = [srv.submit(o) for o in others[:20]]
        rid = srv.submit(req)
        ids += [srv.submit(o) for o in others[20:]]
        mixed = srv.result(rid)
        for i in ids:
            srv.result(i)
        c = srv.counters()
    assert c["completed"] == c["submitted"] == 42 and c["batches"] < 42  # requests were batched together
    assert len(alone.hits) == len(mixed.hits) > 50 and not alone.overflow
    np.testing.assert_allclose(mixed.stats, alone.stats, rtol=1e-9, atol=1e-12)
    np.testing.assert_allclose(mixed.hist, alone.hist, rtol=1e-9, atol=1e-15)
    a, b = alone.hits[_key(alone.hits)], mixed.hits[_key(mixed.hits)]
    assert a.tobytes() == b.tobytes()


def test_served_request_matches_direct_call(propagator):
    req = pp.batches.mixed_batch(16, seed=502, n_min=1e5, n_max=1e6, d_min=2.0, d_max=10.0)
    with serving.Server(propagator, OPTS) as srv:
        r = srv.result(srv.submit(req))
    d = propagator.propagate(req, OPTS)
    np.testing.assert_allclose(r.stats, d.stats, rtol=1e-9, atol=1e-12)
    np.testing.assert_allclose(r.hist, d.hist, rtol=1e-9, atol=1e-15)
    dh = d.sorted_hits()
    rh = r.hits[_key(r.hits)]
    np.testing.assert_array_equal(rh["pair"], dh["pair"])
    np.testing.assert_array_equal(rh["photon_lo"], dh["photon"].astype(np.uint32))
    np.testing.assert_array_equal(rh["pos"], dh["pos"])
    np.testing.assert_array_equal(rh["time"], dh["time"])


def test_admission_by_hbm_budget(propagator):
    req = pp.batches.mixed_batch(4, seed=503, n_min=1e4, n_max=1e5)
    # a budget that holds one request at a time: everything still completes, one per batch
    with serving.Server(propagator, OPTS, hbm_budget_bytes=8 << 20, hit_safety=200.0) as srv:
        ids = [srv.submit(req) for _ in range(6)]
        res = [srv.result(i) for i in ids]
        c = srv.counters()
    assert c["completed"] == 6 and c["reserved_bytes"] == 0
    for r in res[1:]:
        np.testing.assert_allclose(r.stats, res[0].stats, rtol=1e-9, atol=1e-12)
    with serving.Server(propagator, OPTS, hbm_budget_bytes=1 << 16) as srv:
        big = pp.batches.point_source_pair(10_000_000, target=(2.0, 0.0, 0.0))
        with pytest.raises(pp.PPError) as e:
            srv.submit(big)  # can never fit the budget
        assert e.value.status == pp._lib.PP_ERR_ARG


def test_wait_is_bounded_and_overflow_is_reported(propagator):
    req = pp.batches.point_source_pair(50_000_000, target=(1.0, 0.0, 0.0), seed=9)
    with serving.Server(propagator, OPTS, hit_safety=1e-6) as srv:
        rid = srv.submit(req)
        with pytest.raises(pp.PPError) as e:
            srv.wait(rid, timeout_s=0.0)
        assert e.value.status == pp._lib.PP_ERR_TIMEOUT
        r = srv.result(rid, timeout_s=60.0)
    assert r.overflow and len(r.hits) < r.stats[0, 0]  # slots ran out; statistics stay complete
    full = propagator.propagate(req, OPTS, hit_capacity=1 << 22)
    np.testing.assert_allclose(r.stats, full.stats, rtol=1e-9)


def test_open_loop_latency(propagator):
    arrivals, reqs = serving.requests(rate_hz=200.0, duration_s=2.0, seed=7)
    with serving.Server(propagator, OPTS) as srv:
        w_arr, w_req = serving.requests(rate_hz=200.0, duration_s=0.5, seed=8)
        serving.run_open_loop(srv, w_arr, w_req)  # warm-up: first launches and graph set-up
        out, res = serving.run_open_loop(srv, arrivals, reqs)
    print("open loop", out)
    assert out["requests"] == len(reqs) and out["overflow_requests"] == 0
    assert out["p99_ms"] < 50.0

"""pp_propagate_device_noalloc: the allocation-free batched entry point.

Callers whose device memory is all held by their own pool (Julia's CUDA.jl
allocator, PyTorch's caching allocator, a serving loop that reserves HBM up
front) cannot let the library call cudaMalloc: the allocation can fail while
the pool holds the memory, and cudaMalloc/cudaFree can synchronise the device
in the middle of the caller's work.  This entry point keeps its work-queue
scratch in a fixed static device array instead.  The tests call it through
the C ABI twice in a row and compare each result with pp_propagate_device on
the same inputs; they pass alone in a fresh process (where the first call
performs the one-time address look-up) and after the rest of the suite.
"""
import numpy as np
import pytest

import photonprop_b200 as pp

pytestmark = pytest.mark.gpu


def _outputs(torch, n_pairs, bins, cap, dev):
    return (torch.zeros(cap * 64, dtype=torch.uint8, device=dev), torch.zeros(4, dtype=torch.int64, device=dev),
            torch.zeros((n_pairs, 8), dtype=torch.float64, device=dev),
            torch.zeros((n_pairs, bins), dtype=torch.float64, device=dev))


def _sorted_hits(d_hits, n):
    h = d_hits.cpu().numpy()[:n * 64].view(pp.HIT_DTYPE)
    return h[np.lexsort((h["photon"], h["pair"]))]


def test_noalloc_matches_device_entry_on_two_calls(propagator):
    import torch
    dev = torch.device("cuda:0")
    b = pp.batches.mixed_batch(256, seed=77, n_min=1e4, n_max=3e5, d_min=2.0, d_max=20.0)
    ro = pp.RunOptions(mode="physical", t_max=400.0, hist_bins=400)
    cap = 1 << 18
    d_pairs = torch.from_numpy(b.view(np.uint8).copy()).to(dev)
    s = torch.cuda.Stream()

    ref = _outputs(torch, len(b), 400, cap, dev)
    propagator.propagate_device(d_pairs, len(b), ro, ref[0], cap, ref[1], ref[2], ref[3], stream=s)
    s.synchronize()
    n_ref = int(ref[1][0])
    assert n_ref > 100
    ref_hits = _sorted_hits(ref[0], n_ref)

    out = _outputs(torch, len(b), 400, cap, dev)
    for call in range(2):
        torch.cuda.synchronize()
        free_before = torch.cuda.mem_get_info(dev)[0]
        propagator.propagate_device_noalloc(d_pairs, len(b), ro, out[0], cap, out[1], out[2], out[3], stream=s)
        s.synchronize()
        if call == 1:  # the first call may load the module; later calls allocate nothing
            assert torch.cuda.mem_get_info(dev)[0] == free_before
        assert int(out[1][0]) == n_ref, call
        assert int(out[1][1]) == int(ref[1][1]), call  # photon steps
        np.testing.assert_allclose(out[2].cpu().numpy(), ref[2].cpu().numpy(), rtol=1e-9, atol=1e-15)
        np.testing.assert_allclose(out[3].cpu().numpy(), ref[3].cpu().numpy(), rtol=1e-9, atol=1e-15)
        h = _sorted_hits(out[0], n_ref)
        np.testing.assert_array_equal(h["photon"], ref_hits["photon"])
        np.testing.assert_array_equal(h["pair"], ref_hits["pair"])
        np.testing.assert_allclose(h["pos"], ref_hits["pos"], rtol=1e-6, atol=1e-6)
        np.testing.assert_allclose(h["time"], ref_hits["time"], rtol=1e-6)
        np.testing.assert_allclose(h["weight"], ref_hits["weight"], rtol=1e-6, atol=1e-12)


def test_noalloc_rejects_batches_above_the_scratch_limit(propagator):
    import torch
    dev = torch.device("cuda:0")
    b = pp.batches.point_source_pair(1000)
    d_pairs = torch.from_numpy(b.view(np.uint8).copy()).to(dev)
    out = _outputs(torch, 1, 10, 16, dev)
    with pytest.raises(pp.PPError, match="PP_NOALLOC_MAX_PAIRS") as e:
        propagator.propagate_device_noalloc(d_pairs, pp._lib.NOALLOC_MAX_PAIRS + 1, pp.RunOptions(hist_bins=10),
                                            out[0], 16, out[1], out[2], out[3])
    assert e.value.status == pp._lib.PP_ERR_ARG

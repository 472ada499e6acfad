"""The multi-rank path: world_size 2 over gloo.  Each rank propagates its
shard and the gathered table and hits must equal one process propagating
every pair.  On CPU the FP64 oracle stands in for the per-rank compute; with
a GPU present both ranks run the real library on that one GPU in turn (no
kernel waits on another rank, so sharing one GPU is safe)."""
import os
import socket

import numpy as np
import pytest


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _oracle_fn():
    from oracle import oracle as O
    from oracle import tables as tb
    import photonprop_b200 as pp
    from photonprop_b200.propagation import PropagationResult
    m = tb.cascadia(35.0, 2.0)
    T = O.make_tables(m, tb.cherenkov_spectrum_knots((300.0, 800.0), 20, m),
                      pmt=(pp.p_one_pmt_acc.wavelengths, pp.p_one_pmt_acc.acceptance))

    def fn(pairs, opts):
        op = O.pairs_array(len(pairs))
        for f in ("pos", "t0", "dir", "track_len", "target", "radius", "n_photons", "seed", "emitter"):
            op[f] = pairs[f]
        c = opts.to_c()
        oo = O.make_opts(mode=c.mode, max_steps=c.max_steps, g=float(np.float32(c.g)), t_max=c.t_max,
                         hist_bins=c.hist_bins, flags=c.flags & 3)
        h, s, hist, _, total = O.propagate(T, op, oo, n_threads=2)
        hits = np.zeros(len(h), dtype=pp.HIT_DTYPE)
        for f in ("pos", "time", "dir0", "weight", "dir", "wavelength", "dist"):
            hits[f] = h[f]
        hits["pair"] = h["pair"]
        hits["photon"] = h["photon"]
        return PropagationResult(hits, total, s, hist, False)
    return fn


def _gpu_fn():
    import photonprop_b200 as pp
    medium = pp.make_seawater(35.0, 2.0)
    prop = pp.Propagator(medium, pp.CherenkovSpectrum((300.0, 800.0), 20, medium), pp.p_one_pmt_acc, device=0)

    def fn(pairs, opts):
        return prop.propagate(pairs, opts)
    return fn


def _worker(rank, world, port, out_dir, use_gpu=False, backend="gloo"):
    import sys
    repo = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path[:0] = [repo, os.path.join(repo, "photonprop.jl_b200")]
    import datetime
    import torch.distributed as dist
    import photonprop_b200 as pp
    from photonprop_b200.parallel import propagate_sharded
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    device = None
    if backend == "nccl":  # the exchange's tensors on the GPU
        import torch
        torch.cuda.set_device(0)
        device = torch.device("cuda", 0)
        dist.init_process_group("nccl", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60),
                                device_id=device)
    else:
        dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    pairs = pp.batches.mixed_batch(24, seed=123, n_min=1e4, n_max=1e5, d_min=2.0, d_max=6.0)
    opts = pp.RunOptions(mode="physical", t_max=200.0, hist_bins=200)
    res = propagate_sharded(pairs, opts, _gpu_fn() if use_gpu else _oracle_fn(), device=device)
    np.savez(os.path.join(out_dir, f"rank{rank}.npz"), stats=res.stats, hist=res.hist, hits=res.hits.view(np.uint8),
             n_hits=res.n_hits)
    dist.barrier()
    dist.destroy_process_group()


def test_shard_pairs_balanced_and_disjoint():
    import photonprop_b200 as pp
    from photonprop_b200.parallel import shard_pairs
    b = pp.batches.mixed_batch(4096, seed=5)
    for w in (2, 4, 8):
        sh = shard_pairs(b, w)
        allidx = np.concatenate(sh)
        assert sorted(allidx.tolist()) == list(range(4096))
        loads = np.array([b["n_photons"][s].sum() for s in sh])
        assert loads.max() / loads.mean() < 1.01


def _two_ranks(tmp_path, use_gpu, world=2, backend="gloo"):
    import torch.multiprocessing as mp
    port = _free_port()
    mp.start_processes(_worker, args=(world, port, str(tmp_path), use_gpu, backend), nprocs=world, join=True,
                       start_method="spawn")
    import photonprop_b200 as pp
    pairs = pp.batches.mixed_batch(24, seed=123, n_min=1e4, n_max=1e5, d_min=2.0, d_max=6.0)
    opts = pp.RunOptions(mode="physical", t_max=200.0, hist_bins=200)
    ref = _gpu_fn()(pairs, opts) if use_gpu else _oracle_fn()(pairs, opts)
    # FP64 atomics add in any order on the GPU: equal to rounding there, bit for bit on the oracle
    rtol = 1e-12 if use_gpu else 0.0
    for r in range(world):
        d = np.load(tmp_path / f"rank{r}.npz")
        np.testing.assert_allclose(d["stats"], ref.stats, rtol=rtol, atol=0)
        np.testing.assert_allclose(d["hist"], ref.hist, rtol=rtol, atol=0)
        hits = d["hits"].view(pp.HIT_DTYPE)
        hs = hits[np.lexsort((hits["photon"], hits["pair"]))]
        rs = ref.hits[np.lexsort((ref.hits["photon"], ref.hits["pair"]))]
        assert int(d["n_hits"]) == ref.n_hits and hs.tobytes() == rs.tobytes()
    return ref


def test_two_rank_gloo_matches_single_process(tmp_path):
    _two_ranks(tmp_path, use_gpu=False)


@pytest.mark.gpu
def test_two_rank_gloo_gpu_shards_match_single_process(tmp_path):
    ref = _two_ranks(tmp_path, use_gpu=True)
    assert ref.n_hits > 100


@pytest.mark.gpu
def test_one_rank_nccl_device_exchange_matches_single_process(tmp_path):
    """The exchange with its tensors on the GPU over NCCL (one rank: this
    run has one GPU, and two ranks of NCCL on one GPU are not allowed)."""
    ref = _two_ranks(tmp_path, use_gpu=True, world=1, backend="nccl")
    assert ref.n_hits > 100


def test_exchange_moves_each_row_once():
    from photonprop_b200.parallel import exchange_bytes
    # 4096 pairs x (8 + 1000) FP64 values: each rank receives the other ranks' rows once
    assert exchange_bytes(4096, 1000, 2) == 2048 * 1008 * 8
    assert exchange_bytes(4096, 1000, 8) == 7 * 512 * 1008 * 8

"""Multi-GPU propagation: one process per GPU, pairs sharded across ranks.

Pairs are independent and a pair's photons depend only on its seed, so any
split reproduces the single-GPU result exactly.  shard_pairs() balances the
expected cost (photons) with a longest-processing-time greedy split;
propagate_sharded() runs each rank's shard and, when every rank needs the
whole table, exchanges it with one all-reduce (sum) of the zero-padded FP64
statistics and histograms — each pair's row is non-zero on exactly one rank,
so the sum is exact.  Hits are gathered as objects (they are small).
"""
from __future__ import annotations

import numpy as np

from . import _lib
from .propagation import PropagationResult


def shard_pairs(pairs, world_size: int):
    """Index arrays of the pairs each rank propagates (sorted, disjoint,
    covering all pairs), balancing the photon counts."""
    n = np.asarray(pairs["n_photons"], dtype=np.int64)
    order = np.lexsort((np.arange(len(n)), -n))  # largest first, ties by index
    load = np.zeros(world_size, dtype=np.int64)
    owner = np.empty(len(n), dtype=np.int64)
    for i in order:
        r = int(np.argmin(load))
        owner[i] = r
        load[r] += n[i]
    return [np.nonzero(owner == r)[0] for r in range(world_size)]


def propagate_sharded(pairs, opts, propagate_fn, group=None, device=None, gather=True):
    """Propagates this rank's shard with propagate_fn(pairs_subset, opts) ->
    PropagationResult and, if gather, returns the full result on every rank."""
    import torch
    import torch.distributed as dist
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    pairs = np.ascontiguousarray(pairs, dtype=_lib.PAIR_DTYPE)
    idx = shard_pairs(pairs, world)[rank]
    local = propagate_fn(pairs[idx], opts)
    if not gather:
        return idx, local
    n = len(pairs)
    bins = local.hist.shape[1] if local.hist.ndim == 2 else 0
    table = np.zeros((n, _lib.N_STATS + bins))
    table[idx, :_lib.N_STATS] = local.stats
    if bins:
        table[idx, _lib.N_STATS:] = local.hist
    t = torch.from_numpy(table)
    if device is not None:
        t = t.to(device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    table = t.cpu().numpy()
    hits = local.hits.copy()
    if len(hits):
        hits["pair"] = idx[hits["pair"].astype(np.int64)]
    parts = [None] * world
    dist.all_gather_object(parts, (hits, local.n_hits, local.overflow), group=group)
    all_hits = np.concatenate([p[0] for p in parts]) if parts else hits
    return PropagationResult(all_hits, int(sum(p[1] for p in parts)), table[:, :_lib.N_STATS],
                             table[:, _lib.N_STATS:], any(p[2] for p in parts))

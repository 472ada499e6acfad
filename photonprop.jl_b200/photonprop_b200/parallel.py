"""Multi-GPU propagation: one process per GPU, pairs sharded across ranks.

Pairs are independent and a pair's photons depend only on its seed, so any
split reproduces the single-GPU result exactly.  shard_pairs() balances the
expected cost (photons) with a longest-processing-time greedy split;
propagate_sharded() runs each rank's shard and, when every rank needs the
whole result, exchanges only what each rank owns: one all-gather of the
rank's own rows of the FP64 statistics and histograms (padded to the largest
shard, n_pairs x (8 + bins) x 8 bytes in total, e.g. 33 MB for 4096 pairs
with 1000 bins) and one all-gather of its hit records (64 bytes each, padded
to the largest rank's count after an all-gather of the counts).  Rows are
never summed, so the result is bit-identical to one process.
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


def exchange_bytes(n_pairs: int, bins: int, world_size: int) -> int:
    """Bytes of statistics and histograms each rank receives (its own rows
    excluded) in propagate_sharded's all-gather, with shards of equal
    length."""
    rows = -(-n_pairs // world_size)
    return (world_size - 1) * rows * (_lib.N_STATS + bins) * 8


def _all_gather_padded(t, rows_per_rank, group):
    """All-gather of a [rows, ...] tensor whose row count differs by rank
    (rows_per_rank known everywhere): pads to the largest, returns the list
    of each rank's rows."""
    import torch
    import torch.distributed as dist
    world = len(rows_per_rank)
    m = max(max(rows_per_rank), 1)
    pad = torch.zeros((m,) + tuple(t.shape[1:]), dtype=t.dtype, device=t.device)
    pad[: t.shape[0]] = t
    parts = [torch.empty_like(pad) for _ in range(world)]
    dist.all_gather(parts, pad, group=group)
    return [p[:r] for p, r in zip(parts, rows_per_rank)]


def propagate_sharded(pairs, opts, propagate_fn, group=None, device=None, gather=True):
    """Propagates this rank's shard with propagate_fn(pairs_subset, opts) ->
    PropagationResult and, if gather, returns the full result on every rank
    (tensors travel on `device`: a CUDA device for NCCL, None for gloo)."""
    import torch
    import torch.distributed as dist
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    pairs = np.ascontiguousarray(pairs, dtype=_lib.PAIR_DTYPE)
    shards = shard_pairs(pairs, world)
    idx = shards[rank]
    local = propagate_fn(pairs[idx], opts)
    if not gather:
        return idx, local
    n = len(pairs)
    bins = local.hist.shape[1] if local.hist.ndim == 2 else 0
    rows = np.zeros((len(idx), _lib.N_STATS + bins))
    rows[:, :_lib.N_STATS] = local.stats
    if bins:
        rows[:, _lib.N_STATS:] = local.hist
    t = torch.from_numpy(rows)
    if device is not None:
        t = t.to(device)
    parts = _all_gather_padded(t, [len(s) for s in shards], group)
    table = np.zeros((n, _lib.N_STATS + bins))
    for s, p in zip(shards, parts):
        table[s] = p.cpu().numpy()
    # hit records: counts first, then the records as bytes
    hits = local.hits.copy()
    if len(hits):
        hits["pair"] = idx[hits["pair"].astype(np.int64)]
    meta = torch.tensor([len(hits), local.n_hits, int(local.overflow)], dtype=torch.int64)
    if device is not None:
        meta = meta.to(device)
    metas = [torch.empty_like(meta) for _ in range(world)]
    dist.all_gather(metas, meta, group=group)
    metas = [m.cpu().numpy() for m in metas]
    h = torch.from_numpy(np.ascontiguousarray(hits).view(np.uint8).reshape(len(hits), _lib.HIT_DTYPE.itemsize))
    if device is not None:
        h = h.to(device)
    hparts = _all_gather_padded(h, [int(m[0]) for m in metas], group)
    all_hits = np.concatenate([np.ascontiguousarray(p.cpu().numpy()).reshape(-1).view(_lib.HIT_DTYPE)
                               for p in hparts])
    return PropagationResult(all_hits, int(sum(int(m[1]) for m in metas)), table[:, :_lib.N_STATS],
                             table[:, _lib.N_STATS:], any(bool(m[2]) for m in metas))

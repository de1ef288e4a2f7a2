"""Multi-GPU layout of the transport.

Histories are independent, so the path shards without any exchange during
transport: one process per GPU takes a contiguous range of the EDE stream,
cut at history boundaries so that a history's photons are tallied on one
rank, and keeps the global index of its first event (``event_base``), so its
random streams -- and therefore its tallies -- are the ones the unsharded
run would produce.  The only exchange is one sum of the tallies at the end
(``merge_tallies``: an all-reduce over NCCL, or gloo on CPU).
"""
from __future__ import annotations

import numpy as np


def shard_bounds(hist: np.ndarray, rank: int, world: int) -> tuple[int, int]:
    """[start, stop) event range of ``rank`` for events ordered by history
    (1-based, non-decreasing, as the EDE tally produces them).  Histories are
    split as evenly as possible; a history never straddles two ranks."""
    hist = np.asarray(hist)
    if world <= 0 or not 0 <= rank < world:
        raise ValueError("rank must be in [0, world)")
    n = len(hist)
    if n == 0:
        return 0, 0
    if np.any(np.diff(hist) < 0):
        raise ValueError("events must be ordered by history")
    lo, hi = int(hist[0]), int(hist[-1])
    span = hi - lo + 1
    first = lo + (span * rank) // world
    last = lo + (span * (rank + 1)) // world  # exclusive history bound
    start = int(np.searchsorted(hist, first, side="left"))
    stop = int(np.searchsorted(hist, last, side="left")) if rank + 1 < world else n
    return start, stop


def merge_tallies(tallies: dict, group=None) -> dict:
    """Sum integer tallies (PRF image, per-history counts, PHS, counters)
    across ranks.  Values are numpy arrays; returns the merged arrays (on
    every rank).  Integer sums are exact, so the merge is deterministic."""
    import torch
    import torch.distributed as dist

    backend = dist.get_backend(group)
    device = torch.device("cuda", torch.cuda.current_device()) if backend == "nccl" else torch.device("cpu")
    out = {}
    for k in sorted(tallies):
        a = np.ascontiguousarray(tallies[k])
        t = torch.from_numpy(a.astype(np.int64)).to(device)
        dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
        out[k] = t.cpu().numpy().astype(a.dtype)
    return out

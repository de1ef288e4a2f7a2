"""Multi-process (gloo, world size 2) test of the sharded transport layout.

Each rank transports its history range of one EDE stream with the global
event index of its first event, then the tallies are summed with one
all-reduce.  The merged PRF, per-history counts and counters must equal the
unsharded run bit for bit.  On CPU the per-rank transport is the oracle
(the checker); the sharding and merge logic is the product's
(hybridmantis_b200.sharding).
"""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from hybridmantis_b200.sharding import shard_bounds


def _events():
    rng = np.random.default_rng(42)
    n_hist = 9
    per = rng.integers(1, 4, n_hist)
    hist = np.repeat(np.arange(1, n_hist + 1), per).astype(np.int32)
    n = len(hist)
    x = 250.5 + rng.normal(0, 3, n)
    z = 75.0 - np.minimum(rng.exponential(60, n), 149.0)
    N = rng.integers(20, 90, n).astype(np.int32)
    return x, z, hist, N, n_hist


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out_dir):
    import torch.distributed as dist

    from hybridmantis_b200.sharding import merge_tallies
    from oracle import pyoracle as po

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        x, z, hist, N, n_hist = _events()
        a, b = shard_bounds(hist, rank, world)
        g = po.Geometry()
        r = po.run_oracle(g, x[a:b], x[a:b], z[a:b], hist[a:b], N[a:b], base=a, prim_size=n_hist, records=False)
        merged = merge_tallies({"prf": r.image, "prim": r.per_primary, "counters": r.counters})
        if rank == 0:
            np.savez(os.path.join(out_dir, "merged.npz"), **merged)
    finally:
        dist.destroy_process_group()


def test_shard_bounds_cut_at_history_boundaries():
    hist = np.array([1, 1, 2, 3, 3, 3, 4, 5, 5, 6])
    parts = [shard_bounds(hist, r, 3) for r in range(3)]
    assert parts[0][0] == 0 and parts[-1][1] == len(hist)
    for (a0, b0), (a1, b1) in zip(parts, parts[1:]):
        assert b0 == a1
        assert hist[b0 - 1] != hist[a1]  # no history on two ranks
    with pytest.raises(ValueError):
        shard_bounds(np.array([2, 1]), 0, 2)


def test_two_rank_merge_equals_unsharded(tmp_path):
    from oracle import pyoracle as po

    port = _free_port()
    mp.start_processes(_worker, args=(2, port, str(tmp_path)), nprocs=2, join=True, start_method="spawn")
    merged = np.load(tmp_path / "merged.npz")
    x, z, hist, N, n_hist = _events()
    whole = po.run_oracle(po.Geometry(), x, x, z, hist, N, prim_size=n_hist, records=False)
    assert np.array_equal(merged["prf"], whole.image)
    assert np.array_equal(merged["prim"], whole.per_primary)
    assert np.array_equal(merged["counters"], whole.counters)

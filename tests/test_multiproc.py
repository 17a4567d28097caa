"""The N > 1 path on the CPU: world_size-2 gloo process groups over 127.0.0.1
run the sharding helpers bench.py and multi-GPU callers use (byte-balanced
string shards, max-over-ranks timing, gathered per-string results)."""

import socket

import numpy as np
import pytest

from trex_b200.sharding import gather_results, max_over_ranks, rank_seed, run_sharded, shard_bounds


def test_shard_bounds_balance_bytes():
    rng = np.random.default_rng(0)
    lens = rng.integers(0, 5000, size=10_000)
    off = np.zeros(len(lens) + 1, np.int64)
    np.cumsum(lens, out=off[1:])
    for world in (1, 2, 3, 8):
        b = shard_bounds(off, world)
        assert b[0] == 0 and b[-1] == len(lens) and np.all(np.diff(b) >= 0)
        cost = np.array([off[b[r + 1]] - off[b[r]] + 64 * (b[r + 1] - b[r]) for r in range(world)])
        assert cost.max() - cost.min() <= 5000 + 64   # at most one string apart
    assert list(shard_bounds(np.zeros(1, np.int64), 4)) == [0, 0, 0, 0, 0]
    assert rank_seed(7, 0) != rank_seed(7, 1)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import torch.distributed as dist
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world)
    try:
        res = {}
        res["max"] = max_over_ranks(1.5 + rank, dist)
        res["gather"] = gather_results(np.arange(10 * rank, 10 * rank + 2 + rank, dtype=np.int64), dist)
        rng = np.random.default_rng(3)
        lens = rng.integers(0, 100, size=1001)
        off = np.zeros(len(lens) + 1, np.int64)
        np.cumsum(lens, out=off[1:])
        seen = []
        res["sharded"] = run_sharded(off, lambda lo, hi: seen.append((lo, hi)) or lens[lo:hi].astype(np.int64),
                                     dist)
        res["range"] = seen[0]
        res["seed"] = rank_seed(2024, rank)
        out.put((rank, res))
    finally:
        dist.destroy_process_group()


def test_gloo_world_size_2():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = dict(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    rng = np.random.default_rng(3)
    lens = rng.integers(0, 100, size=1001)
    for r in (0, 1):
        assert got[r]["max"] == 2.5
        assert list(got[r]["gather"]) == [0, 1, 10, 11, 12]
        assert np.array_equal(got[r]["sharded"], lens)
    assert got[0]["range"][0] == 0 and got[0]["range"][1] == got[1]["range"][0]
    assert got[1]["range"][1] == 1001
    assert got[0]["seed"] != got[1]["seed"]

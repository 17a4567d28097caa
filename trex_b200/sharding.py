"""Multi-GPU sharding of string batches: one process per GPU.

Strings are independent, so a batch shards by strings with no data-path
collective: every rank walks a contiguous range of strings whose bytes are
balanced across ranks (each string also costs a fixed overhead, counted as
``per_string`` bytes), and the per-string results are gathered afterwards.
The reference is single-GPU; this is the plumbing `bench.py --gpus N` and
multi-GPU callers use (process groups over NCCL, or gloo on the CPU).
"""

from __future__ import annotations

from typing import Callable, Optional

import numpy as np


def shard_bounds(offsets: np.ndarray, world: int, per_string: int = 64) -> np.ndarray:
    """String index bounds [world + 1] of `world` contiguous shards with about
    equal bytes (+ per_string per string): shard r = strings [b[r], b[r+1])."""
    off = np.asarray(offsets, dtype=np.int64)
    n = len(off) - 1
    if world < 1:
        raise ValueError("world must be >= 1")
    if n <= 0:
        return np.zeros(world + 1, dtype=np.int64)
    # cumulative cost at the end of each string
    cost = (off[1:] - off[0]) + per_string * np.arange(1, n + 1, dtype=np.int64)
    total = int(cost[-1])
    targets = (total * np.arange(1, world, dtype=np.float64) / world)
    inner = np.searchsorted(cost, targets, side="left") + 1
    b = np.concatenate([[0], np.minimum(inner, n), [n]]).astype(np.int64)
    return np.maximum.accumulate(b)


def shard_of(offsets: np.ndarray, rank: int, world: int, per_string: int = 64):
    """(lo, hi) string range of this rank."""
    b = shard_bounds(offsets, world, per_string)
    return int(b[rank]), int(b[rank + 1])


def rank_seed(seed: int, rank: int) -> int:
    """Seed of a rank's own synthetic batch (weak scaling: every rank its own data)."""
    return int(seed) + 7919 * int(rank)


def max_over_ranks(value: float, dist=None, device=None) -> float:
    """The largest value over all ranks (times are reported as the max over ranks)."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def gather_results(local: np.ndarray, dist=None, device=None) -> np.ndarray:
    """Concatenates every rank's per-string results in rank order (on every rank)."""
    local = np.ascontiguousarray(local)
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return local
    import torch
    world = dist.get_world_size()
    n = torch.tensor([local.shape[0]], dtype=torch.int64, device=device)
    sizes = [torch.zeros_like(n) for _ in range(world)]
    dist.all_gather(sizes, n)
    sizes = [int(s.item()) for s in sizes]
    m = max(sizes)
    buf = torch.zeros((m,) + local.shape[1:], dtype=torch.from_numpy(local[:0]).dtype, device=device)
    if local.shape[0]:
        buf[:local.shape[0]] = torch.from_numpy(local).to(device)
    parts = [torch.zeros_like(buf) for _ in range(world)]
    dist.all_gather(parts, buf)
    return np.concatenate([p[:s].cpu().numpy() for p, s in zip(parts, sizes)])


def run_sharded(offsets: np.ndarray, run_shard: Callable[[int, int], np.ndarray], dist=None,
                device=None, per_string: int = 64) -> np.ndarray:
    """Runs this rank's shard (run_shard(lo, hi) -> per-string results of strings
    [lo, hi)) and returns all ranks' results in string order."""
    if dist is None or not dist.is_initialized():
        return np.asarray(run_shard(0, len(offsets) - 1))
    lo, hi = shard_of(offsets, dist.get_rank(), dist.get_world_size(), per_string)
    return gather_results(np.asarray(run_shard(lo, hi)), dist, device)


def dfa_shard_runner(dfa_set, data: np.ndarray, offsets: np.ndarray,
                     dfa_id: Optional[np.ndarray] = None, seg_len: int = 0):
    """run_shard for run_sharded: the strings [lo, hi) of a host batch through
    the B200 ragged kernel of this rank's GPU (DFASet.run_host); returns the
    accept flags."""
    off = np.asarray(offsets, dtype=np.int64)

    def run(lo: int, hi: int) -> np.ndarray:
        if hi <= lo:
            return np.zeros(0, dtype=np.uint8)
        a, b = int(off[lo]), int(off[hi])
        sub_off = off[lo:hi + 1] - a
        ids = None if dfa_id is None else np.ascontiguousarray(dfa_id[lo:hi])
        _, acc, _, _ = dfa_set.run_host(np.ascontiguousarray(data[a:b]), sub_off, ids, seg_len=seg_len)
        return np.asarray(acc[:hi - lo], dtype=np.uint8)

    return run

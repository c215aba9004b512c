"""Data-parallel sharding of a pair batch across ranks (one process per GPU).

GASAL2's pairs are independent, so N GPUs each align their own shard and no
collective runs in the data path (weak scaling: every rank keeps a full-size
shard).  The only collectives are for timing: every rank reports its
CUDA-event time and the job's time is the maximum over ranks.
"""
from __future__ import annotations

import os

import numpy as np


def rank_info():
    """(rank, world_size, local_rank) from the torchrun environment."""
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def shard_seed(base_seed: int, rank: int) -> int:
    """Seed of a rank's synthetic shard: distinct, deterministic per rank."""
    return base_seed + 1000 * rank


def shard_range(n_total: int, rank: int, world: int):
    """Contiguous [lo, hi) slice of n_total pairs for a rank (strong-scaling
    split of a fixed batch; sizes differ by at most one)."""
    q, r = divmod(n_total, world)
    lo = rank * q + min(rank, r)
    return lo, lo + q + (1 if rank < r else 0)


def cell_shard_range(cells, rank: int, world: int):
    """Contiguous [lo, hi) slice of a batch for a rank, balanced by work: the
    cut points are where the running sum of per-pair cells (qlen * tlen)
    crosses k/world of the total, so every rank gets about the same number of
    DP cells rather than of pairs (a strong-scaling split of one batch whose
    lengths are uneven).  Every pair lands in exactly one slice."""
    cells = np.asarray(cells, dtype=np.float64)
    n = len(cells)
    if n == 0:
        return 0, 0
    csum = np.cumsum(cells)
    total = csum[-1]
    if total <= 0:
        return shard_range(n, rank, world)
    def cut(k):
        if k <= 0:
            return 0
        if k >= world:
            return n
        # slice k-1 ends after the pair whose running sum first reaches k/world of the total
        return int(np.searchsorted(csum, total * k / world, side="left")) + 1
    lo, hi = cut(rank), cut(rank + 1)
    lo = min(lo, n)
    hi = min(max(hi, lo), n)
    return lo, hi


def max_over_ranks(value: float, dist=None, device=None) -> float:
    """Job time = slowest rank's time (all_reduce MAX); identity without a
    process group."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_throughput(pairs_per_rank: int, world: int, steps: int, max_ms: float) -> float:
    """Whole-job pairs/s: every rank's pairs over the slowest rank's time."""
    return pairs_per_rank * world * steps / (max_ms * 1e-3)

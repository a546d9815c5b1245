"""Multi-GPU plumbing: one process per GPU over torch.distributed.

MD runs independent replicas (the system is not decomposed; no data-path
collective).  The batched fit shards the configurations across ranks, each rank
assembles the normal equations of its shard on its own GPU, and one SUM
all-reduce of A (64 x 64) and b (64) combines them -- the only exchange step
(NCCL on GPUs, gloo on CPU).  Timings are the maximum over ranks.
"""
from __future__ import annotations

import numpy as np


def shard_bounds(counts, rank: int, world: int) -> tuple[int, int]:
    """Contiguous range [lo, hi) of configurations for rank, balanced by atom
    count (cut where the running atom total crosses rank/world of the whole)."""
    counts = np.asarray(counts, dtype=np.int64)
    csum = np.concatenate([[0], np.cumsum(counts)])
    total = csum[-1]
    cuts = [0] + [int(np.searchsorted(csum, total * r / world, side="left")) for r in range(1, world)] + [len(counts)]
    for r in range(1, world + 1):
        cuts[r] = max(cuts[r], cuts[r - 1])
    return cuts[rank], cuts[rank + 1]


def allreduce_sum(*arrays, device=None):
    """Elementwise sum over ranks of float64 numpy arrays (one collective)."""
    import torch
    import torch.distributed as dist
    flat = np.concatenate([np.asarray(a, dtype=np.float64).ravel() for a in arrays])
    t = torch.from_numpy(flat).to(device if device is not None else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    out = t.cpu().numpy()
    res, k = [], 0
    for a in arrays:
        a = np.asarray(a)
        res.append(out[k:k + a.size].reshape(a.shape))
        k += a.size
    return res


def max_over_ranks(x: float, device=None) -> float:
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x)], dtype=torch.float64, device=device if device is not None else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())

"""The multi-rank paths on CPU (gloo, world size 2): configuration sharding,
the single all-reduce of the normal equations, and max-over-ranks timing."""
import os
import socket

import numpy as np
import pytest

from mdp_b200 import fit, parallel


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def test_shard_bounds_cover_and_balance():
    counts = np.random.default_rng(0).integers(16, 513, size=4096)
    for world in (1, 2, 3, 8):
        b = [parallel.shard_bounds(counts, r, world) for r in range(world)]
        assert b[0][0] == 0 and b[-1][1] == len(counts)
        assert all(b[r][1] == b[r + 1][0] for r in range(world - 1))
        load = [counts[lo:hi].sum() for lo, hi in b]
        assert max(load) - min(load) <= 2 * counts.max()


def _worker(rank, world, port, out):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        cfgs, e, f = fit.batch_configs(12, seed=4, lo=16, hi=64)
        rng = np.random.default_rng(0)
        n = np.array([c.natoms for c in cfgs])
        bi = rng.normal(size=(len(cfgs), 5))
        bd = rng.normal(size=(n.sum(), 3, 5))
        lo, hi = parallel.shard_bounds(n, rank, world)
        a0 = np.concatenate([[0], np.cumsum(n)])
        R, t = fit.rows_numpy(cfgs[lo:hi], bi[lo:hi], bd[a0[lo]:a0[hi]], e[lo:hi], f[a0[lo]:a0[hi]])
        A, b = parallel.allreduce_sum(R.T @ R, R.T @ t)
        ms = parallel.max_over_ranks(10.0 + rank)
        if rank == 0:
            Rf, tf = fit.rows_numpy(cfgs, bi, bd, e, f)
            np.save(out, np.array([np.max(np.abs(A - Rf.T @ Rf)), np.max(np.abs(b - Rf.T @ tf)), ms]))
    finally:
        dist.destroy_process_group()


def test_two_rank_normal_equations_equal_one_rank(tmp_path):
    import torch.multiprocessing as mp
    out = str(tmp_path / "res.npy")
    mp.spawn(_worker, args=(2, _free_port(), out), nprocs=2, join=True)
    da, db, ms = np.load(out)
    assert da < 1e-10 and db < 1e-10
    assert ms == 11.0

"""Batched-fitting host logic on the CPU: the configuration generator against
the stored fixture inputs, the workload's shape, and the row assembly."""
import os
import sys

import numpy as np
import pytest

from conftest import GOLDEN, fit_names
from mdp_b200 import fit

sys.path.insert(0, GOLDEN)
import make_golden  # noqa: E402


@pytest.mark.parametrize("name", fit_names())
def test_fixture_inputs_regenerate(name):
    sparse = {c[0]: c for c in make_golden.SPARSE_FIT_CASES}
    if name in sparse:
        _, n, edge, seed, tj = sparse[name]
        cfg = make_golden.sparse_config(n, edge, seed)
        d = np.load(os.path.join(GOLDEN, name + ".npz"))
        assert np.array_equal(cfg.x, d["x"]) and np.array_equal(cfg.box, d["box"])
        return
    cases = {c[0]: c + ((0.0, 0.0, 0.0),) for c in make_golden.FIT_CASES}
    cases.update({c[0]: c for c in make_golden.TRI_FIT_CASES})
    _, kind, target, strain, sigma, seed, tj, flags, tilt = cases[name]
    cfg = fit.make_config(kind, target, strain, sigma, np.random.default_rng(seed))
    if any(tilt):
        cfg = make_golden.sheared(cfg, tilt)
        assert cfg.box.shape == (3, 3)
    d = np.load(os.path.join(GOLDEN, name + ".npz"))
    assert np.array_equal(cfg.x, d["x"]) and np.array_equal(cfg.box, d["box"])


def test_workload_shape():
    cfgs, e, f = fit.batch_configs(4096)
    n = np.array([c.natoms for c in cfgs])
    assert len(cfgs) == 4096 and n.min() >= 16 and n.max() <= 512
    assert 1.0e6 < n.sum() < 1.15e6
    assert min(c.box.min() for c in cfgs) >= fit.MIN_WIDTH
    assert {c.kind for c in cfgs} == {"bcc", "fcc", "a15"}
    assert f.shape == (n.sum(), 3) and e.shape == (4096,)
    for c in cfgs[:50]:
        assert np.all(c.x >= 0) and np.all(c.x < c.box)


def test_rows_and_solve_recover_a_linear_model():
    rng = np.random.default_rng(0)
    cfgs, _, _ = fit.batch_configs(6, seed=1, lo=16, hi=40)
    k = 5
    n = np.array([c.natoms for c in cfgs])
    bi = rng.normal(size=(6, k))
    bd = rng.normal(size=(n.sum(), 3, k))
    beta = rng.normal(size=1 + k)
    e = beta[0] * n + bi @ beta[1:]
    f = np.einsum("ick,k->ic", bd, beta[1:])   # f = beta . bd (bd = -dB/dx)
    R, t = fit.rows_numpy(cfgs, bi, bd, e, f)
    got = fit.solve(R.T @ R, R.T @ t)
    assert np.allclose(got, beta, rtol=1e-9, atol=1e-9)

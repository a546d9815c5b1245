"""Batched descriptors and normal equations on the GPU against the reference's
ComputeSnap chain (golden fixtures) and against numpy assembly of the same rows."""
import glob
import os

import numpy as np
import pytest

from mdp_b200 import configs, fit

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
FIX = sorted(glob.glob(os.path.join(HERE, "golden", "fit_*.npz")))


def _params(d):
    bnorm, bzero, switch = [int(v) for v in d["flags"]]
    return configs.snap_params(int(d["twojmax"]), seed=0, bnormflag=bnorm, bzeroflag=bzero, switchflag=switch)


def _cfg(d):
    return fit.FitConfig(x=d["x"], box=d["box"], kind=str(d["kind"]))


def _rel(a, b):
    return np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300)


@pytest.mark.parametrize("path", FIX, ids=[os.path.basename(p)[:-4] for p in FIX])
def test_descriptors_match_reference(path):
    d = np.load(path)
    bf = fit.BatchFit(_params(d))
    bf.set_batch([_cfg(d)])
    bi, bd, bv, bl = bf.descriptors()
    bf.close()
    assert _rel(bi[0], d["bi"]) < 1e-10
    assert _rel(bl, d["blist"]) < 1e-10
    assert _rel(bd, np.transpose(d["bd"], (1, 2, 0))) < 1e-10
    assert _rel(bv[0], d["bv"]) < 1e-10


def test_batch_equals_single_configurations():
    ds = [np.load(p) for p in FIX if "2j8" in p]
    p = _params(ds[0])
    bf = fit.BatchFit(p)
    bf.set_batch([_cfg(d) for d in ds])
    bi, bd, bv, bl = bf.descriptors()
    bf.close()
    a0 = 0
    for c, d in enumerate(ds):
        n = d["x"].shape[0]
        assert _rel(bi[c], d["bi"]) < 1e-10
        assert _rel(bd[a0:a0 + n], np.transpose(d["bd"], (1, 2, 0))) < 1e-10
        assert _rel(bl[:, a0:a0 + n], d["blist"]) < 1e-10
        a0 += n


@pytest.fixture(scope="module")
def small_batch():
    cfgs, e, f = fit.batch_configs(24, seed=5, lo=16, hi=160)
    we = np.linspace(0.5, 2.0, len(cfgs))
    wf = np.linspace(1.5, 0.7, len(cfgs))
    p = configs.snap_params(8, seed=0)
    bf = fit.BatchFit(p)
    bf.set_batch(cfgs, e, f, we, wf)
    yield bf, cfgs, e, f, we, wf
    bf.close()


def test_fp64_assembly_matches_numpy(small_batch):
    bf, cfgs, e, f, we, wf = small_batch
    bi, bd, bv, bl = bf.descriptors()
    R, t = fit.rows_numpy(cfgs, bi, bd, e, f, we, wf)
    A, b, ms = bf.run("fp64")
    assert _rel(A, R.T @ R) < 1e-12
    assert _rel(b, R.T @ t) < 1e-12
    # the captured graph replays to the same bits
    A2, b2, _ = bf.run("fp64")
    assert np.array_equal(A, A2) and np.array_equal(b, b2)


def test_chunked_pipeline_equals_one_chunk(small_batch):
    bf, cfgs, e, f, we, wf = small_batch
    A, b, _ = bf.run("fp64")
    bi, bd, bv, bl = bf.descriptors()
    assert bf.nchunks() == 1
    bf.set_chunk_bytes(2e6)          # a few configurations per chunk
    try:
        assert bf.nchunks() > 3
        A2, b2, _ = bf.run("fp64")
        bi2, bd2, bv2, bl2 = bf.descriptors()
    finally:
        bf.set_chunk_bytes(24e9)
    assert _rel(A2, A) < 1e-13 and _rel(b2, b) < 1e-13
    assert np.array_equal(bd2, bd) and np.array_equal(bi2, bi) and np.array_equal(bv2, bv)


def test_bf16_split_assembly(small_batch):
    bf, cfgs, e, f, we, wf = small_batch
    A, b, _ = bf.run("fp64")
    Ab, bb, _ = bf.run("bf16")
    assert np.linalg.norm(Ab - A) / np.linalg.norm(A) < 1e-4
    assert np.linalg.norm(bb - b) / np.linalg.norm(b) < 1e-4


def test_tuned_shapes_give_the_same_system(small_batch):
    bf, *_ = small_batch
    A, b, _ = bf.run("fp64")
    choice = bf.tune()
    assert choice["du_threads"] in (32, 64, 128) and choice["gram_rows"] in (256, 1024, 4096, 16384)
    A2, b2, _ = bf.run("fp64")
    assert _rel(A2, A) < 1e-12 and _rel(b2, b) < 1e-12


def test_fit_recovers_known_coefficients():
    """Energies and forces of plain 2J=8 SNAP with known beta: the FP64 fit
    returns beta (the rows are consistent, so the least-squares residual is 0)."""
    from mdp_b200.snap import snap_compute
    p = configs.snap_params(8, seed=3)
    cfgs, _, _ = fit.batch_configs(40, seed=9, lo=16, hi=200)
    e = np.zeros(len(cfgs))
    f = []
    for c, cf in enumerate(cfgs):
        out = snap_compute(p, cf.x, cf.box, 1.0, 96, precision="fp64")
        e[c] = out["eatom"].sum()
        f.append(out["fatom"])
    f = np.concatenate(f)
    bf = fit.BatchFit(p)
    bf.set_batch(cfgs, e, f)
    A, b, _ = bf.run("fp64")
    beta = fit.solve(A, b)
    bf.close()
    assert np.max(np.abs(beta - p.coeff)) < 1e-6 * np.max(np.abs(p.coeff))


@pytest.mark.parametrize("tj", [4, 6, 8])
def test_descriptors_contract_to_the_oracle(tj):
    """At every 2J the fit takes (4, 6, 8): the batch's
    per-atom bispectrum and dB/dR, contracted with beta, give the oracle's
    per-atom energies (beta_0 + beta . B_i) and forces (beta . bd_i)."""
    from oracle import oracle
    p = configs.snap_params(tj, seed=11)
    cfg = configs.ta_config((3, 3, 3), temp=300, jitter=0.1, seed=4)
    xa, al, nl, nn = oracle.neighbor_list(cfg.x, cfg.box, p.rcut, 1.0, 64)
    e, f, _ = oracle.snap_force(xa, al, nl, nn, p)
    bf = fit.BatchFit(p)
    bf.set_batch([fit.FitConfig(x=cfg.x, box=np.asarray(cfg.box, dtype=float), kind="bcc")])
    bi, bd, _, bl = bf.descriptors()
    bf.close()
    beta0, beta = p.coeff[0], np.asarray(p.coeff[1:])
    assert _rel(beta0 + beta @ bl, e) < 1e-10
    assert _rel(bd @ beta, f) < 1e-10
    assert _rel(bi[0], bl.sum(axis=1)) < 1e-12

"""Edge cases of the plain force path: an isolated atom (no neighbours at
all), a dimer, a sparse gas with ragged neighbour counts, many atoms
having none, and a crystal slab beside a gas in one box (the dE/dr kernel
copies a window's Y rows into shared memory when its 128 pairs span at most
16 atoms and reads them in place otherwise: both kinds of window, and the
windows between them, occur in one launch).  The oracle is checked against the reference's CPU code on the
CPU (when the reference build is present); the GPU path is checked against
the oracle: identical ghosts and neighbour sets, per-atom energy, forces and
virial within 1e-10 of the largest magnitude (or absolutely, where the
reference values are zero)."""
import numpy as np
import pytest

from mdp_b200 import configs
from oracle import oracle, refpy

SKIN, NEIGHMAX = 1.0, 64


def _isolated():
    return np.array([[3.0, 4.0, 5.0]]), np.array([20.0, 20.0, 20.0])


def _dimer():
    return np.array([[5.0, 5.0, 5.0], [7.1, 6.2, 5.9]]), np.array([20.0, 21.0, 22.0])


def _gas():
    rng = np.random.default_rng(5)
    return rng.uniform(0.0, 32.0, (40, 3)), np.array([32.0, 32.0, 32.0])


def _slab_and_gas():
    rng = np.random.default_rng(11)
    x, box = configs.lattice((4, 4, 4), "bcc", configs.TA_LATTICE)
    x = x + rng.normal(0.0, 0.05, x.shape)
    box = np.array([4.0 * box[0], box[1], box[2]])
    gas = np.column_stack([rng.uniform(box[0] / 4 + 1.0, box[0] - 1.0, 40),
                           rng.uniform(0.0, box[1], 40), rng.uniform(0.0, box[2], 40)])
    return np.mod(np.vstack([x, gas]), box), box


CASES = {"isolated": _isolated, "dimer": _dimer, "gas": _gas, "slab_gas": _slab_and_gas}


def close(a, b, tol=1e-10):
    return np.abs(a - b).max() <= tol * max(np.abs(b).max(), 1.0)


def sorted_rows(nl, nn):
    return [tuple(sorted(nl[i, : nn[i]].tolist())) for i in range(len(nn))]


@pytest.mark.parametrize("name", sorted(CASES))
def test_case_shapes(name):
    x, box = CASES[name]()
    p = configs.snap_params(8, seed=9)
    xa, al, nl, nn = oracle.neighbor_list(x, box, p.rcut, SKIN, NEIGHMAX)
    if name == "isolated":
        assert nn.tolist() == [0]
    if name == "gas":
        assert (nn == 0).sum() >= 5 and nn.max() >= 2      # isolated atoms and clusters
    if name == "slab_gas":
        assert nn[:128].min() >= 20 and np.mean(nn[128:]) < 8   # dense rows, then sparse ones


@pytest.mark.skipif(not refpy.available(), reason="reference build absent")
@pytest.mark.parametrize("name", sorted(CASES))
def test_oracle_matches_reference(name):
    x, box = CASES[name]()
    p = configs.snap_params(8, seed=9)
    xa, al, nl, nn = refpy.neighbor_list(x, box, p.rcut, SKIN, NEIGHMAX, neighcell=0)
    xo, alo, nlo, nno = oracle.neighbor_list(x, box, p.rcut, SKIN, NEIGHMAX)
    assert np.array_equal(xo, xa) and np.array_equal(alo, al)
    assert sorted_rows(nlo, nno) == sorted_rows(nl, nn)
    e, f, v = refpy.snap_force(xa, al, nl, nn, p)
    eo, fo, vo = oracle.snap_force(xo, alo, nlo, nno, p)
    assert close(eo, e) and close(fo, f) and close(vo, v)


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(CASES))
def test_gpu_matches_oracle(cuda_lib, name):
    from mdp_b200.snap import snap_compute
    x, box = CASES[name]()
    p = configs.snap_params(8, seed=9)
    xo, alo, nlo, nno = oracle.neighbor_list(x, box, p.rcut, SKIN, NEIGHMAX)
    eo, fo, vo = oracle.snap_force(xo, alo, nlo, nno, p)
    out = snap_compute(p, x, box, SKIN, NEIGHMAX, want_neighbors=True)
    assert out["anum"] == xo.shape[0]
    assert np.array_equal(out["xall"], xo) and np.array_equal(out["alist"], alo)
    assert sorted_rows(out["neighlist"], out["neighnum"]) == sorted_rows(nlo, nno)
    assert close(out["eatom"], eo) and close(out["fatom"], fo) and close(out["vatom"], vo)
    o32 = snap_compute(p, x, box, SKIN, NEIGHMAX, precision="fp32")
    assert np.all(np.isfinite(o32["fatom"])) and np.abs(o32["fatom"] - fo).max() < 1e-4

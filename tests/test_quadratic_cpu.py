"""CPU: the quadratic-SNAP fixtures and their algebra.

The fixtures (tests/golden/quad_*.npz) hold the reference's ComputePairSnap
chain (snappotential.cpp:236-410) run with quadraticflag = 1.  Checked here,
without a GPU:

* the reference build reproduces each fixture exactly from its inputs;
* each per-atom energy equals beta0 + beta . B_i + B_i^T Q B_i / 2 with Q the
  symmetric matrix whose upper triangle is the coefficient tail packed by rows
  (cpuSnapTallyEnergyFull, cpuSnap.cpp:1745-1770), B_i taken from the
  reference's ComputeSnap chain -- the packing the GPU path's k_snap_quad
  reads;
* the quadratic terms move the forces by more than the GPU tolerance by many
  orders, so the GPU test exercises them.
"""
import glob
import os

import numpy as np
import pytest

from conftest import GOLDEN, load_golden
from mdp_b200 import configs
from oracle import refpy

NAMES = sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN, "quad_*.npz")))

pytestmark = pytest.mark.skipif(not refpy.available(), reason="oracle/_ref not built")


def params(g, **kw):
    bnorm, bzero, switch = (int(v) for v in g["flags"])
    return configs.snap_params(int(g["twojmax"]), seed=int(g["coeff_seed"]), bnormflag=bnorm, bzeroflag=bzero,
                               switchflag=switch, **kw)


def args(g):
    return g["xall"], g["alist"], g["neighlist"], g["neighnum"]


@pytest.mark.parametrize("name", NAMES)
def test_reference_reproduces_fixture(name):
    g = load_golden(name)
    p = params(g, quadraticflag=1)
    assert np.array_equal(p.coeff, g["coeff"])
    e, f, v = refpy.snap_force_pairsnap(*args(g), p)
    assert np.array_equal(e, g["eatom"]) and np.array_equal(f, g["fatom"]) and np.array_equal(v, g["vatom"])


@pytest.mark.parametrize("name", NAMES)
def test_energy_is_packed_quadratic_form(name):
    g = load_golden(name)
    p = params(g, quadraticflag=1)
    nb = p.ncoeff
    _, _, _, B = refpy.snap_descriptors(*args(g), p)
    beta0, beta, tail = p.coeff[0], p.coeff[1:nb + 1], p.coeff[nb + 1:]
    assert tail.size == nb * (nb + 1) // 2
    Q = np.zeros((nb, nb))
    Q[np.triu_indices(nb)] = tail          # row-major upper triangle
    Q = Q + np.triu(Q, 1).T
    e = beta0 + beta @ B + 0.5 * np.einsum("ki,kl,li->i", B, Q, B)
    assert np.abs(e - g["eatom"]).max() < 1e-11 * max(1.0, np.abs(g["eatom"]).max())


@pytest.mark.parametrize("name", NAMES)
def test_quadratic_terms_are_material(name):
    g = load_golden(name)
    p = params(g)                            # the same linear coefficients, no quadratic tail
    e, f, _ = refpy.snap_force_pairsnap(*args(g), p)
    df = np.abs(f - g["fatom"]).max() / np.abs(g["fatom"]).max()
    de = np.abs(e - g["eatom"]).max()
    assert df > 1e-3 and de > 1e-4, (df, de)

"""CPU: the multi-element fixtures and what the reference's chain does with
several element types.

* The reference build reproduces each tests/golden/chem_*.npz exactly.
* With one element listed, or two identical elements without chemflag, the
  multi-element chain gives the single-element results bit for bit.
* chemflag = 0: the reference's forces are minus the gradient of its
  energy (central differences, 1e-6 eV/A).
* chemflag = 1: they are not.  cpuSnapComputeYi (cpuSnap4.cpp:762-784) gives
  each coupling one element triple and a multiplicity factor (3 when
  j1 = j2 = j, 2 when one index repeats) that is exact only when the
  coefficients are symmetric under the element permutations it stands for;
  with independent coefficients per triple the Y-based forces differ from
  the derivative of the energy of cpuSnapComputeEi (cpuSnap4.cpp:250-420) by
  a sizeable fraction of the forces.  The GPU path therefore evaluates the
  energy from the element-triple bispectrum and the forces from the
  reference's Y, as the reference does, and matches both.
"""
import dataclasses
import glob
import os

import numpy as np
import pytest

from conftest import GOLDEN, load_golden
from mdp_b200 import configs
from oracle import refpy

NAMES = sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN, "chem_*.npz")))

pytestmark = pytest.mark.skipif(not refpy.available(), reason="oracle/_ref not built")


def params(g):
    bnorm, bzero, switch, wsa = (int(v) for v in g["flags"])
    return configs.snap_params_elements(int(g["twojmax"]), g["radelems"], g["wjelems"], chemflag=int(g["chemflag"]),
                                        seed=int(g["coeff_seed"]), bnormflag=bnorm, bzeroflag=bzero,
                                        switchflag=switch, wselfallflag=wsa)


@pytest.mark.parametrize("name", NAMES)
def test_reference_reproduces_fixture(name):
    g = load_golden(name)
    p = params(g)
    assert np.array_equal(p.coeff, g["coeff"])
    e, f, v = refpy.snap_force_me(g["xall"], g["alist"], g["neighlist"], g["neighnum"], g["types"], p)
    assert np.array_equal(e, g["eatom"]) and np.array_equal(f, g["fatom"]) and np.array_equal(v, g["vatom"])


def _small():
    cfg = configs.ta_config((3, 3, 3), temp=300.0, jitter=0.05, seed=1)
    types = np.random.default_rng(0).integers(1, 3, cfg.natoms).astype(np.int32)
    return cfg, types


def test_single_element_reductions():
    cfg, types = _small()
    p = configs.snap_params(6, seed=3)
    xa, al, nl, nn = refpy.neighbor_list(cfg.x, cfg.box, p.rcut, 1.0, 80, neighcell=0)
    e, f, _ = refpy.snap_force(xa, al, nl, nn, p)
    one = dataclasses.replace(p, radelems=(0.5,), wjelems=(1.0,))
    e1, f1, _ = refpy.snap_force_me(xa, al, nl, nn, np.ones(cfg.natoms, np.int32), one)
    two = dataclasses.replace(p, radelems=(0.5, 0.5), wjelems=(1.0, 1.0), coeff=np.concatenate([p.coeff, p.coeff]))
    e2, f2, _ = refpy.snap_force_me(xa, al, nl, nn, types, two)
    assert np.array_equal(e, e1) and np.array_equal(f, f1)
    assert np.array_equal(e, e2) and np.array_equal(f, f2)


def fd_error(p, cfg, types, h=1e-5):
    def run(x):
        xa, al, nl, nn = refpy.neighbor_list(x, cfg.box, p.rcut, 1.0, 80, neighcell=0)
        e, f, _ = refpy.snap_force_me(xa, al, nl, nn, types, p)
        return e.sum(), f
    _, f = run(cfg.x)
    err = 0.0
    for i in (0, 5, 17):
        for k in range(3):
            xp = cfg.x.copy(); xp[i, k] += h
            xm = cfg.x.copy(); xm[i, k] -= h
            err = max(err, abs((run(xp)[0] - run(xm)[0]) / (2 * h) + f[i, k]))
    return err, np.abs(f).max()


def test_chemflag0_forces_are_the_energy_gradient():
    cfg, types = _small()
    p = configs.snap_params_elements(6, (0.5, 0.45), (1.0, 0.8), chemflag=0, seed=5, bzeroflag=1)
    err, fmax = fd_error(p, cfg, types)
    assert err < 1e-6 * max(1.0, fmax), err


def test_chemflag1_forces_are_not_the_energy_gradient():
    cfg, types = _small()
    p = configs.snap_params_elements(6, (0.5, 0.45), (1.0, 0.8), chemflag=1, seed=5)
    err, fmax = fd_error(p, cfg, types)
    assert err > 0.1 * fmax, (err, fmax)

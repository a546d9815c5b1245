"""Sheared (triclinic) periodic cells through the plain FP64 force path:
ghosts, neighbour sets and per-atom energy, forces and virial against the
reference's CPU code (tri_* golden fixtures)."""
import os
import sys

import numpy as np
import pytest

from conftest import GOLDEN, golden_params, load_golden, tri_names
from oracle import oracle

sys.path.insert(0, GOLDEN)
import make_golden  # noqa: E402

TOL_FP64 = 1e-10
NAMES = tri_names()


def rel_inf(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def sorted_rows(nl, nn):
    return [tuple(sorted(nl[i, : nn[i]].tolist())) for i in range(len(nn))]


def test_fixtures_present():
    assert len(NAMES) == 2


@pytest.mark.parametrize("name", NAMES)
def test_inputs_regenerate_and_cell_is_sheared(name):
    g = load_golden(name)
    case = {c[0]: c for c in make_golden.TRI_CASES}[name]
    _, cells, tj, temp, jit, seed, cseed, tilt = case
    x, H = make_golden.tri_config(cells, temp, jit, seed, tilt)
    assert np.array_equal(x, g["x"]) and np.array_equal(H, g["box"])
    assert np.abs(H - np.diag(np.diag(H))).max() > 0.1


@pytest.mark.parametrize("name", NAMES)
def test_reference_list_forms_agree(name):
    g = load_golden(name)
    assert sorted_rows(g["neighlist"], g["neighnum"]) == sorted_rows(g["neighlist_cell"], g["neighnum_cell"])


@pytest.mark.parametrize("name", NAMES)
def test_oracle_matches_reference(name):
    g = load_golden(name)
    p = golden_params(g)
    xa, al, nl, nn = oracle.neighbor_list(g["x"], g["box"], p.rcut, float(g["skin"]), int(g["neighmax"]))
    assert np.array_equal(xa, g["xall"]) and np.array_equal(al, g["alist"])
    assert sorted_rows(nl, nn) == sorted_rows(g["neighlist"], g["neighnum"])
    e, f, v = oracle.snap_force(xa, al, nl, nn, p)
    assert rel_inf(e, g["eatom"]) < TOL_FP64
    assert rel_inf(f, g["fatom"]) < TOL_FP64
    assert rel_inf(v, g["vatom"]) < TOL_FP64


@pytest.mark.gpu
@pytest.mark.parametrize("name", NAMES)
def test_gpu_matches_reference(cuda_lib, name):
    from mdp_b200.snap import snap_compute
    g = load_golden(name)
    p = golden_params(g)
    out = snap_compute(p, g["x"], g["box"], float(g["skin"]), int(g["neighmax"]), want_neighbors=True)
    assert out["anum"] == g["xall"].shape[0]
    assert np.array_equal(out["xall"], g["xall"]), "ghost coordinates differ from the reference"
    assert np.array_equal(out["alist"], g["alist"]), "ghost numbering differs from the reference"
    assert sorted_rows(out["neighlist"], out["neighnum"]) == sorted_rows(g["neighlist"], g["neighnum"])
    assert rel_inf(out["eatom"], g["eatom"]) < TOL_FP64
    assert rel_inf(out["fatom"], g["fatom"]) < TOL_FP64
    assert rel_inf(out["vatom"], g["vatom"]) < TOL_FP64

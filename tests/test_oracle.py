"""CPU tests: the oracle restatement against the golden fixtures generated
from the reference's own CPU code, and against the reference build when it is
present (oracle/_ref)."""
import numpy as np
import pytest

from conftest import golden_names, golden_params, load_golden
from mdp_b200 import configs
from oracle import oracle, refpy


def rel_inf(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def sorted_rows(nl, nn):
    return [tuple(sorted(nl[i, : nn[i]].tolist())) for i in range(len(nn))]


@pytest.mark.parametrize("name", golden_names())
def test_inputs_regenerate(name):
    g = load_golden(name)
    cfg = configs.ta_config(tuple(g["cells"]), temp=float(g["temp"]), jitter=float(g["jitter"]), seed=int(g["seed"]))
    assert np.array_equal(cfg.x, g["x"]) and np.array_equal(cfg.v, g["v"]) and np.array_equal(cfg.box, g["box"])
    golden_params(g)


@pytest.mark.parametrize("name", golden_names())
def test_oracle_neighbors_bit_exact(name):
    g = load_golden(name)
    p = golden_params(g)
    xa, al, nl, nn = oracle.neighbor_list(g["x"], g["box"], p.rcut, float(g["skin"]), int(g["neighmax"]))
    assert np.array_equal(xa, g["xall"]), "ghost positions differ"
    assert np.array_equal(al, g["alist"]), "ghost owners differ"
    assert sorted_rows(nl, nn) == sorted_rows(g["neighlist"], g["neighnum"])


@pytest.mark.parametrize("name", golden_names())
def test_oracle_forces_match_reference(name):
    g = load_golden(name)
    p = golden_params(g)
    e, f, v = oracle.snap_force(g["xall"], g["alist"], g["neighlist"], g["neighnum"], p)
    assert rel_inf(e, g["eatom"]) < 1e-12
    assert rel_inf(f, g["fatom"]) < 1e-10
    assert rel_inf(v, g["vatom"]) < 1e-10


def test_oracle_md_trajectory():
    g = load_golden("bcc128_2j6")
    p = golden_params(g)
    x, v = g["x"].copy(), g["v"].copy()
    box, dt, n = g["box"], float(g["md_dt"]), g["x"].shape[0]
    dtfm = 0.5 * dt * configs.FTM2V / configs.TA_MASS
    skin, nm = float(g["skin"]), int(g["neighmax"])
    xa, al, nl, nn = oracle.neighbor_list(x, box, p.rcut, skin, nm)
    xhold = x.copy()
    e, f, va = oracle.snap_force(xa, al, nl, nn, p)
    for step in range(int(g["md_steps"])):
        xstart = x.copy()
        v = v + dtfm * f
        x = x + dt * v
        if np.max(np.sum((x - xhold) ** 2, axis=1)) > 0.25 * skin * skin:
            x = np.where(x < 0, x + box, x)
            x = np.where(x >= box, np.maximum(x - box, 0.0), x)
            xa, al, nl, nn = oracle.neighbor_list(x, box, p.rcut, skin, nm)
            xhold = x.copy()
        else:
            xa = xa.copy(); xa[:n] = x; xa[n:] += (x - xstart)[al[n:]]
        e, f, va = oracle.snap_force(xa, al, nl, nn, p)
        v = v + dtfm * f
    assert rel_inf(x, g["md_x"]) < 1e-10
    assert rel_inf(v, g["md_v"]) < 1e-8
    assert rel_inf(e, g["md_e"]) < 1e-10


def test_cell_list_completeness_quirk():
    """The reference's cell-form list equals its O(N^2) list when its cells are
    at least rcut+skin wide, and drops skin-shell pairs otherwise; the project
    (and the oracle) always produce the complete list."""
    for name in golden_names():
        g = load_golden(name)
        full = sorted_rows(g["neighlist"], g["neighnum"])
        cell = sorted_rows(g["neighlist_cell"], g["neighnum_cell"])
        for a, b in zip(full, cell):
            assert set(b) <= set(a)


@pytest.mark.skipif(not refpy.available(), reason="reference build (oracle/_ref) not present")
def test_oracle_vs_reference_random_flags():
    rng = np.random.default_rng(5)
    for tj in (4, 6, 8):
        flags = dict(bnormflag=int(rng.integers(2)), bzeroflag=int(rng.integers(2)), switchflag=int(rng.integers(2)))
        p = configs.snap_params(tj, seed=int(rng.integers(1 << 30)), **flags)
        cfg = configs.ta_config((3, 3, 3), temp=500, jitter=0.15, seed=int(rng.integers(1 << 30)))
        xa, al, nl, nn = refpy.neighbor_list(cfg.x, cfg.box, p.rcut, 1.0, 80, neighcell=0)
        e, f, v = refpy.snap_force(xa, al, nl, nn, p)
        e2, f2, v2 = oracle.snap_force(xa, al, nl, nn, p)
        assert rel_inf(e2, e) < 1e-12 and rel_inf(f2, f) < 1e-10 and rel_inf(v2, v) < 1e-10


def test_tables_match_reference_counts():
    for tj, (ncg, nu, nb, nz) in {4: (305, 55, 14, 185), 6: (1321, 140, 30, 779), 8: (4098, 285, 55, 2386)}.items():
        s = oracle.table_sizes(tj)
        assert (s["idxcg"], s["idxu"], s["idxb"], s["idxz"]) == (ncg, nu, nb, nz)


def test_zbl_restatement_matches_reference_generated_code():
    """The numpy ZBL restatement against MDP's own generated code for the Ta
    potential of its snapTA06A example (inner 4, outer 4.8, Z 73)."""
    from oracle import refpy, zbl
    if not refpy.available():
        pytest.skip("oracle/_ref not built")
    import ctypes as C
    L = refpy.lib()
    L.ref_zbl_pairs.argtypes = [C.c_void_p] * 3 + [C.c_int]
    rng = np.random.default_rng(3)
    r = np.concatenate([rng.uniform(1.5, 4.8, 4000), np.linspace(3.9, 4.1, 101)])
    u_dir = rng.normal(size=(r.size, 3))
    xij = np.ascontiguousarray(u_dir / np.linalg.norm(u_dir, axis=1)[:, None] * r[:, None])
    u_ref, ux_ref = np.zeros(r.size), np.zeros((r.size, 3))
    L.ref_zbl_pairs(u_ref.ctypes.data, ux_ref.ctypes.data, xij.ctypes.data, r.size)
    u, ux = zbl.zbl_pair(xij)
    assert np.abs(u - u_ref).max() <= 1e-12 * np.abs(u_ref).max()
    assert np.abs(ux - ux_ref).max() <= 1e-11 * np.abs(ux_ref).max()

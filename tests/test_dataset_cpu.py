"""CPU: MDP's JSON training-data reader and the cell replication of the
real-data fit (mdp_b200.dataset)."""
import json
import os

import numpy as np
import pytest

from mdp_b200 import configs, dataset
from oracle import oracle
from oracle.refroot import reference_root

_REF = reference_root()
TA_JSON = os.path.join(_REF, "fitting", "snap", "Ta", "JSON") if _REF else ""


def write_json(path, frames, header="# A test JSON file for QM data\n"):
    """Frames in MDP's JSON training format (readJSON.jl:8-165)."""
    data = []
    for fr in frames:
        d = {"NumAtoms": fr.natoms, "Lattice": fr.lattice.tolist(), "Positions": fr.x.tolist(),
             "AtomTypes": ["Ta"] * fr.natoms}
        if fr.e is not None:
            d["Energy"] = fr.e
        if fr.f is not None:
            d["Forces"] = fr.f.tolist()
        if fr.stress is not None:
            d["Stress"] = fr.stress.tolist()
        data.append(d)
    with open(path, "w") as fh:
        fh.write(header + json.dumps({"Dataset": {"Data": data}}))


def bcc2(a=3.316, tilt=(0.0, 0.0, 0.0), jitter=0.0, seed=0):
    """Two-atom BCC cell (narrower than the cutoff), optionally sheared."""
    H = np.array([[a, 0, 0], [tilt[0] * a, a, 0], [tilt[1] * a, tilt[2] * a, a]])
    s = np.array([[0.0, 0.0, 0.0], [0.5, 0.5, 0.5]])
    x = s @ H + np.random.default_rng(seed).normal(0, jitter, (2, 3))
    return dataset.Frame(natoms=2, lattice=H, x=x)


def test_reader_fields_and_order(tmp_path):
    rng = np.random.default_rng(1)
    frames = []
    for n in (2, 5, 3):
        fr = dataset.Frame(natoms=n, lattice=np.diag(rng.uniform(5, 9, 3)) + rng.normal(0, 0.2, (3, 3)),
                           x=rng.uniform(0, 5, (n, 3)), e=float(rng.normal()), f=rng.normal(size=(n, 3)),
                           stress=rng.normal(size=(3, 3)))
        frames.append(fr)
    write_json(tmp_path / "b.json", frames[1:])
    write_json(tmp_path / "a.json", frames[:1])
    (tmp_path / "notes.txt").write_text("not data")
    got = dataset.read_json_folder(str(tmp_path))
    assert [g.natoms for g in got] == [2, 5, 3]          # files in name order, frames in file order
    for g, fr in zip(got, frames):
        np.testing.assert_array_equal(g.lattice, fr.lattice)
        np.testing.assert_array_equal(g.x, fr.x)
        np.testing.assert_array_equal(g.f, fr.f)
        np.testing.assert_array_equal(g.stress, fr.stress)
        assert g.e == fr.e
        assert np.all(g.types == 1)


def test_reader_rejects_inconsistent_atom_count(tmp_path):
    (tmp_path / "bad.json").write_text(json.dumps({"Dataset": {"Data": [
        {"NumAtoms": 3, "Lattice": np.eye(3).tolist(), "Positions": [[0, 0, 0]]}]}}))
    with pytest.raises(ValueError, match="NumAtoms"):
        dataset.read_json(str(tmp_path / "bad.json"))


def test_replication_covers_cutoff_and_keeps_atoms_first():
    fr = bcc2(tilt=(0.1, -0.05, 0.08), jitter=0.05, seed=3)
    cfg, m = dataset.replicate(fr, 4.67637)
    assert np.all(dataset.cell_widths(cfg.box) > 4.67637)
    assert m == cfg.natoms // 2 and m > 1
    np.testing.assert_allclose(cfg.x[:2], dataset.wrap(fr.x, fr.lattice), atol=1e-12)
    s = cfg.x @ np.linalg.inv(cfg.box)                  # every copy inside the replicated cell
    assert s.min() >= -1e-12 and s.max() < 1.0


def test_replicated_energy_per_atom_is_invariant():
    """The replicated cell reproduces the narrow cell's physics: energy per atom
    and the original atoms' forces are the same for m and 27m copies."""
    p = configs.snap_params(4, seed=5)
    fr = bcc2(tilt=(0.07, 0.0, -0.04), jitter=0.08, seed=4)
    res = []
    for scale in (1, 2):
        cfg, m = dataset.replicate(fr, p.rcut)
        H = cfg.box
        if scale == 2:                                    # three copies along each vector
            cfg = dataset.replicate(dataset.Frame(natoms=cfg.natoms, lattice=H, x=cfg.x), 2.0 * np.linalg.norm(H[0]))[0]
        xa, al, nl, nn = oracle.neighbor_list(cfg.x, cfg.box, p.rcut, 1.0, 64)
        e, f, _ = oracle.snap_force(xa, al, nl, nn, p)
        res.append((e.sum() / cfg.natoms, f[:2]))
    assert abs(res[0][0] - res[1][0]) < 1e-12 * abs(res[0][0])
    np.testing.assert_allclose(res[0][1], res[1][1], atol=1e-11)


def test_batch_weights_reproduce_original_rows():
    """A frame replicated m times gets its energy row per atom and force rows
    scaled by 1/sqrt(m): the same normal-equation contribution."""
    fr = bcc2(jitter=0.05, seed=2)
    fr.e, fr.f = -23.0, np.arange(6.0).reshape(2, 3)
    g = dataset.Group("g", [fr], we=100.0, wf=2.0)
    cfgs, e, f, we, wf, copies, gid = dataset.batch_of([g], 4.67637)
    m = copies[0]
    assert cfgs[0].natoms == 2 * m
    assert np.isclose(we[0] * e[0], 100.0 * fr.e / 2)     # weighted target = w_e * E / N
    assert np.isclose(we[0] * cfgs[0].natoms, 100.0)      # one-body column = w_e
    assert np.isclose(m * wf[0] ** 2, 4.0)                # m force copies at weight^2 / m


@pytest.mark.skipif(not os.path.isdir(TA_JSON), reason="MDP's Ta training set is not present")
def test_reads_the_reference_ta_training_set():
    sizes = {}
    for folder in sorted(os.listdir(TA_JSON)):
        frames = dataset.read_json_folder(os.path.join(TA_JSON, folder))
        for fr in frames:
            assert fr.e is not None and fr.f.shape == (fr.natoms, 3)
            cfg, m = dataset.replicate(fr, 4.67637)
            assert np.all(dataset.cell_widths(cfg.box) > 4.67637)
        sizes[folder] = len(frames)
    assert len(sizes) == 12 and sum(sizes.values()) == 363


def write_extxyz(path, frames):
    """Frames in extended-XYZ form (readEXTXYZ.jl)."""
    with open(path, "w") as fh:
        for fr in frames:
            fh.write(f"{fr.natoms}\n")
            lat = " ".join(f"{v:.17g}" for v in fr.lattice.ravel())
            st = " ".join(f"{v:.17g}" for v in fr.stress.ravel())
            fh.write(f'Lattice="{lat}" Properties=species:S:1:pos:R:3:forces:R:3 energy={fr.e:.17g} '
                     f'stress="{st}" pbc="T T T"\n')
            for i in range(fr.natoms):
                row = " ".join(f"{v:.17g}" for v in np.concatenate([fr.x[i], fr.f[i]]))
                fh.write(f"Ta {row}\n")


def test_extxyz_reader_matches_json_reader(tmp_path):
    rng = np.random.default_rng(7)
    frames = [dataset.Frame(natoms=n, lattice=np.diag(rng.uniform(5, 9, 3)) + rng.normal(0, 0.3, (3, 3)),
                            x=rng.uniform(0, 5, (n, 3)), e=float(rng.normal(-20, 3)), f=rng.normal(size=(n, 3)),
                            stress=rng.normal(size=(3, 3))) for n in (3, 1, 4)]
    write_json(tmp_path / "t.json", frames)
    write_extxyz(tmp_path / "t.xyz", frames)
    a = dataset.read_folder(str(tmp_path), extension="json")
    b = dataset.read_folder(str(tmp_path), extension="xyz")
    assert len(a) == len(b) == 3
    for fa, fb in zip(a, b):
        assert fa.natoms == fb.natoms and fa.e == fb.e
        for k in ("lattice", "x", "f", "stress", "types"):
            np.testing.assert_array_equal(getattr(fa, k), getattr(fb, k))


def test_fitsnap_folder_table_and_loading(tmp_path):
    from mdp_b200 import fitsnap
    assert len(fitsnap.TA_FOLDERS) == 12
    for k, (name, *_) in enumerate(fitsnap.TA_FOLDERS):
        (tmp_path / name).mkdir()
        write_json(tmp_path / name / "x.json", [bcc2(seed=k)])
    groups = fitsnap.load_groups(str(tmp_path))
    assert [g.name for g in groups] == [f[0] for f in fitsnap.TA_FOLDERS]
    assert groups[3].ws == 1e-4 and groups[7].we == 467.0
    assert all(len(g.frames) == 1 for g in groups)


def test_stress_rows_use_the_reference_component_order():
    """bv arrives as xx, yy, zz, xy, xz, yz; the rows are xx, yy, zz, yz, xz, xy
    (snapcpp.jl:662 with emldescriptors.jl's stress index [1, 5, 9, 6, 3, 2])."""
    bv = np.arange(12.0).reshape(2, 6)                  # (k, 6)
    cell = np.diag([2.0, 3.0, 4.0])
    R = dataset.stress_rows(bv, cell, 1)
    s = dataset.EV_PER_A3_IN_BAR / 24.0
    np.testing.assert_allclose(R[:, 0], 0.0)
    np.testing.assert_allclose(R[:, 1:], s * bv.T[[0, 1, 2, 5, 4, 3]])
    assert dataset.VOIGT[3] == (1, 2) and dataset.VOIGT[5] == (0, 1)


def test_non_periodic_frames_are_refused(tmp_path):
    fr = bcc2(seed=1)
    fr.e, fr.f, fr.stress = -20.0, np.zeros((2, 3)), np.zeros((3, 3))
    write_extxyz(tmp_path / "a.xyz", [fr])
    text = (tmp_path / "a.xyz").read_text().replace('pbc="T T T"', 'pbc="T T F"')
    (tmp_path / "a.xyz").write_text(text)
    got = dataset.read_extxyz(str(tmp_path / "a.xyz"))
    assert got[0].pbc == (True, True, False)
    with pytest.raises(ValueError, match="periodic"):
        dataset.batch_of([dataset.Group("slab", got)], 4.67637)


def test_missing_energy_or_forces_get_zero_weight():
    a, b = bcc2(seed=1), bcc2(seed=2)
    a.e = -20.0                                         # a: energy only; b: forces only
    b.f = np.ones((2, 3))
    cfgs, e, f, we, wf, copies, gid = dataset.batch_of([dataset.Group("g", [a, b], we=3.0, wf=2.0)], 4.67637)
    assert we[0] > 0 and wf[0] == 0.0
    assert we[1] == 0.0 and wf[1] > 0

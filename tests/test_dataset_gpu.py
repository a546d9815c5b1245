"""GPU: the real-data linear fit (mdp_b200.dataset.fit_groups) end to end.

Training files in MDP's JSON format are written for two groups of frames --
narrow sheared 2-atom BCC cells (replicated to cover the cutoff) and sheared
16-54 atom supercells -- with energies and forces of a known linear SNAP
model from the oracle.  Reading them back and fitting on the GPU must
recover the model: the fitted energies, forces and stresses match the
targets and the coefficients match the known ones."""
import numpy as np
import pytest

from mdp_b200 import configs, dataset, fit
from oracle import oracle
from test_dataset_cpu import bcc2, write_json

pytestmark = pytest.mark.gpu


def _targets(fr, p):
    """Energy, forces and stress (bar) of the known model on the frame."""
    cfg, m = dataset.replicate(fr, p.rcut)
    xa, al, nl, nn = oracle.neighbor_list(cfg.x, cfg.box, p.rcut, 1.0, 96)
    e, f, v = oracle.snap_force(xa, al, nl, nn, p)
    fr.e, fr.f = float(e.sum() / m), f[:fr.natoms].copy()
    w = v.sum(axis=1) * dataset.EV_PER_A3_IN_BAR / abs(np.linalg.det(cfg.box))
    fr.stress = np.zeros((3, 3))
    for k, (i, j) in enumerate(((0, 0), (1, 1), (2, 2), (0, 1), (0, 2), (1, 2))):   # the oracle's virial order
        fr.stress[i, j] = fr.stress[j, i] = w[k]
    return fr


def _frames(p):
    rng = np.random.default_rng(11)
    narrow = [_targets(bcc2(a=3.316 * (1 + rng.uniform(-0.04, 0.04)), tilt=tuple(rng.uniform(-0.1, 0.1, 3)),
                            jitter=0.08, seed=s), p) for s in range(6)]
    bulk = []
    for s, (kind, n) in enumerate([("bcc", 16), ("fcc", 32), ("a15", 64), ("bcc", 54), ("fcc", 32), ("bcc", 16)]):
        cfg = fit.make_config(kind, n, rng.uniform(-0.04, 0.04), rng.uniform(0.05, 0.25), rng)
        L = np.asarray(cfg.box)
        t = rng.uniform(-0.1, 0.1, 3)
        H = np.array([[L[0], 0, 0], [t[0] * L[0], L[1], 0], [t[1] * L[0], t[2] * L[1], L[2]]])
        bulk.append(_targets(dataset.Frame(natoms=cfg.natoms, lattice=H, x=(cfg.x / L) @ H), p))
    return narrow, bulk


def test_fit_recovers_known_model_from_json(tmp_path):
    p = configs.snap_params(6, seed=21)
    narrow, bulk = _frames(p)
    (tmp_path / "Narrow").mkdir()
    (tmp_path / "Bulk").mkdir()
    for i, fr in enumerate(narrow):
        write_json(tmp_path / "Narrow" / f"N_{i}.json", [fr])
    write_json(tmp_path / "Bulk" / "B.json", bulk)
    groups = [dataset.Group("Narrow", dataset.read_json_folder(str(tmp_path / "Narrow")), we=100.0, wf=1.0,
                            ws=1e-5),
              dataset.Group("Bulk", dataset.read_json_folder(str(tmp_path / "Bulk")), we=1.0, wf=1.0, ws=1e-4)]
    out = dataset.fit_groups(groups, p)
    assert out["replicated"] == 6
    smax = max(np.abs(fr.stress).max() for fr in narrow + bulk)
    for err in out["errors"]:
        assert err["energy_rmse"] < 1e-6, err        # eV/atom
        assert err["force_rmse"] < 1e-6, err         # eV/A
        assert err["stress_rmse"] < 1e-6 * smax, err  # bar
    beta = out["beta"]
    assert abs(beta[0] - p.coeff[0]) < 1e-6 * abs(p.coeff[0])
    assert np.max(np.abs(beta[1:] - p.coeff[1:])) < 1e-4 * np.max(np.abs(p.coeff[1:]))


def test_fitsnap_cli_on_a_folder_tree(tmp_path):
    """fitsnap.jl's twelve folders and weights through the command-line entry."""
    from mdp_b200 import fitsnap
    p = configs.snap_params(6, seed=21)
    narrow, bulk = _frames(p)
    for (name, *_), fr in zip(fitsnap.TA_FOLDERS, narrow + bulk):
        (tmp_path / name).mkdir()
        write_json(tmp_path / name / "a.json", [fr])
    res = fitsnap.main(["--data", str(tmp_path), "--no-zbl"])
    assert len(res["errors"]) == 12 and res["configs"] == 12
    assert len(res["coefficients"]) == 1 + p.ncoeff and np.all(np.isfinite(res["coefficients"]))
    for err in res["errors"]:                            # the data come from one linear model
        assert err["force_rmse"] < 1e-4, err


def test_zbl_reference_matches_oracle():
    """mdp_fit_zbl on a sheared cell and a replicated narrow cell against the
    oracle's full-list ZBL tally (oracle/zbl.py)."""
    from oracle import zbl
    p = configs.snap_params(6, seed=21)
    narrow, bulk = _frames(p)
    cfgs = [dataset.replicate(fr, 4.8)[0] for fr in (narrow[0], bulk[1], bulk[2])]
    e, f, w = dataset.zbl_reference(cfgs, p, (4.0, 4.8, 73.0))
    a0 = 0
    for c, cfg in enumerate(cfgs):
        xa, al, nl, nn = oracle.neighbor_list(cfg.x, cfg.box, 4.8, 0.5, 160)
        ez, fz, vz = zbl.zbl_tally(xa, nl, nn, 4.8)
        n = cfg.natoms
        assert abs(e[c] - ez.sum()) <= 1e-10 * abs(ez).sum()
        np.testing.assert_allclose(f[a0:a0 + n], fz, rtol=0, atol=1e-10 * np.abs(fz).max())
        np.testing.assert_allclose(w[c], vz.sum(axis=1), rtol=0, atol=1e-10 * np.abs(vz).sum())
        a0 += n


def test_fit_with_zbl_recovers_snap_part():
    """Targets = known linear SNAP + ZBL: fitting with the ZBL reference
    subtracted recovers the SNAP coefficients."""
    from oracle import zbl
    p = configs.snap_params(6, seed=21)
    narrow, bulk = _frames(p)
    for fr in narrow + bulk:
        cfg, m = dataset.replicate(fr, 4.8 + 0.5)
        xa, al, nl, nn = oracle.neighbor_list(cfg.x, cfg.box, 4.8, 0.5, 160)
        ez, fz, vz = zbl.zbl_tally(xa, nl, nn, 4.8)
        fr.e += ez.sum() / m
        fr.f = fr.f + fz[:fr.natoms]
        w = vz.sum(axis=1) * dataset.EV_PER_A3_IN_BAR / abs(np.linalg.det(cfg.box))
        for k, (i, j) in enumerate(((0, 0), (1, 1), (2, 2), (0, 1), (0, 2), (1, 2))):
            fr.stress[i, j] += w[k]
            if i != j:
                fr.stress[j, i] += w[k]
    groups = [dataset.Group("Narrow", narrow, we=100.0, wf=1.0, ws=1e-5),
              dataset.Group("Bulk", bulk, we=1.0, wf=1.0, ws=1e-4)]
    out = dataset.fit_groups(groups, p, zbl=(4.0, 4.8, 73.0))
    smax = max(np.abs(fr.stress).max() for fr in narrow + bulk)
    for err in out["errors"]:
        assert err["energy_rmse"] < 1e-6, err
        assert err["force_rmse"] < 1e-6, err
        assert err["stress_rmse"] < 1e-6 * smax, err
    beta = out["beta"]
    assert abs(beta[0] - p.coeff[0]) < 1e-6 * abs(p.coeff[0])
    assert np.max(np.abs(beta[1:] - p.coeff[1:])) < 1e-4 * np.max(np.abs(p.coeff[1:]))


def test_frames_missing_energies_or_forces_add_only_their_rows():
    """A group mixing energy-only, force-only and complete frames: the GPU
    fit's coefficients equal a NumPy least-squares solve over exactly the rows
    that are present (descriptors from the reference's ComputeSnap chain),
    with random targets so that every row matters."""
    from oracle import refpy
    p = configs.snap_params(6, seed=5)
    rng = np.random.default_rng(17)
    frames = []
    for s, (kind, n) in enumerate([("bcc", 54), ("fcc", 32), ("a15", 64), ("bcc", 16), ("fcc", 108), ("bcc", 54),
                                   ("a15", 64), ("fcc", 32)]):
        cfg = fit.make_config(kind, n, rng.uniform(-0.04, 0.04), rng.uniform(0.05, 0.25), rng)
        fr = dataset.Frame(natoms=cfg.natoms, lattice=np.diag(np.asarray(cfg.box, dtype=np.float64)), x=cfg.x)
        has_e, has_f = (s % 3 != 1), (s % 3 != 0)
        fr.e = float(rng.normal() * cfg.natoms) if has_e else None
        fr.f = rng.normal(size=(cfg.natoms, 3)) if has_f else None
        frames.append(fr)
    we, wf = 3.0, 0.7
    out = dataset.fit_groups([dataset.Group("Mixed", frames, we=we, wf=wf, ws=0.0)], p)
    rows, ys = [], []
    for fr in frames:
        cfg, m = dataset.replicate(fr, p.rcut)
        assert m == 1
        xa, al, nl, nn = refpy.neighbor_list(cfg.x, cfg.box, p.rcut, 0.0, 128, neighcell=0)
        bi, bd, _, _ = refpy.snap_descriptors(xa, al, nl, nn, p)
        if fr.e is not None:
            rows.append(we / fr.natoms * np.concatenate([[fr.natoms], bi]))
            ys.append(we / fr.natoms * fr.e)
        if fr.f is not None:
            F = np.zeros((3 * fr.natoms, 1 + p.ncoeff))
            F[:, 1:] = bd.reshape(p.ncoeff, -1).T
            rows.extend(wf * F)
            ys.extend(wf * fr.f.ravel())
    beta = np.linalg.lstsq(np.array(rows), np.array(ys), rcond=None)[0]
    assert np.abs(out["beta"] - beta).max() < 1e-6 * np.abs(beta).max()
    err = out["errors"][0]
    assert err["frames"] == len(frames) and "energy_rmse" in err and "force_rmse" in err

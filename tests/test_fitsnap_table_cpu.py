"""CPU: the real-data Ta fit reproduces the errors MDP publishes for it.

fitting/snap/Ta/fitsnap.jl ends with the per-folder energy, force and stress
MAE / RMSE / RSQ that its run printed.  This test repeats that fit on the same
363 frames with this repository's host-side fit logic (mdp_b200.dataset: the
JSON reader, the reference's cell orientation, cell replication for narrow
cells, energy-per-atom and stress-per-volume rows, the folder weights,
validate2's unweighted errors) and takes the per-configuration descriptors from
the reference's own C++ ComputeSnap chain and the ZBL reference potential from
the oracle (test infrastructure, oracle/).  The published table is read from
fitsnap.jl itself.

Read as fitsnap.jl reads them (transposelattice = true: cell vectors are the
columns of each file's Lattice array), the fit reproduces every published
RMSE to within 0.1 % -- except the force errors of the three Volume folders.
Those frames are perfect cubic crystals (A15, BCC, FCC cells with diagonal
lattices) whose DFT forces in the files are exactly zero; their SNAP and ZBL
forces vanish by symmetry, so the fit's force error there is zero, while the
table reports 6.25, 6.07 and 2.89 eV/A.  The table's RSQ for those folders is
finite, so the reference's force targets (DFT forces minus its ZBL forces)
were not zero: its Julia ZBL evaluation returned nonzero per-atom forces on
these cells, although its ZBL energies and virials agree with ours (the
Volume energy and stress errors match to 5 digits).  That is asserted here.

Read with the cell vectors as rows -- where the 2-atom BCC frames' second
atom sits exactly at the body centre -- the Elastic folders' force errors drop
from 0.079 / 0.065 to about 1e-4 eV/A: the published values come from the
distortion the transposition introduces.
"""
import os

import numpy as np
import pytest

from mdp_b200 import configs, dataset, fitsnap
from oracle.refroot import reference_root

_REF = reference_root()
TA = os.path.join(_REF, "fitting", "snap", "Ta") if _REF else ""

pytestmark = pytest.mark.skipif(not _REF or not os.path.isdir(os.path.join(TA, "JSON")),
                                reason="MDP's Ta training set is not present")


def published_table():
    """{'Energy' | 'Force' | 'Stress': {folder: (MAE, RMSE, RSQ)}} from the comment block of fitsnap.jl."""
    txt = open(os.path.join(TA, "fitsnap.jl")).read()
    out = {}
    for kind in ("Energy", "Force", "Stress"):
        blk = txt[txt.index(f"# {kind} Errors"):]
        rows = {}
        for line in blk.splitlines()[2:]:
            if line.startswith("# ---"):
                break
            parts = [p.strip() for p in line.lstrip("#").split("|")]
            rows[parts[0]] = tuple(float(v) for v in parts[1:4])
        out[kind] = rows
    return out


def close(ours, published, rtol):
    """Relative agreement; the table prints some values in a fixed-width column
    that drops the exponent (1.07923030094437 for 1,079,230), so a published
    value that is off by a power of ten is compared by its mantissa."""
    if published == 0.0:
        return abs(ours) < 1e-12
    r = ours / published
    k = round(np.log10(r)) if r > 0 else 0
    return abs(r / 10.0 ** k - 1.0) < rtol


def fit_errors(transpose_lattice):
    """The fit of fitsnap.jl (2J=6, ZBL subtracted, energy-force-stress loss,
    lsq) on all 12 folders; per-folder unweighted RMSE of energy per atom,
    force components and Voigt stresses."""
    from oracle import refpy, zbl
    if not refpy.available():
        pytest.fail("oracle/_ref/libmdp_ref_harness.so missing (build with make -C oracle ref)")
    p = configs.snap_params(6, seed=0, rcutfac=4.67637, radelem=0.5, rfac0=0.99363, rmin0=0.0, switchflag=1,
                            bzeroflag=0, bnormflag=0, wselfallflag=0)
    inner, outer, z = fitsnap.TA_ZBL
    groups = fitsnap.load_groups(os.path.join(TA, "JSON"), transpose_lattice=transpose_lattice)
    nc = 1 + p.ncoeff
    A = np.zeros((nc, nc))
    b = np.zeros(nc)
    rows = []
    for grp in groups:
        for fr in grp.frames:
            cfg, m = dataset.replicate(fr, max(p.rcut, outer))
            n, n0 = cfg.natoms, fr.natoms
            xa, al, nl, nn = refpy.neighbor_list(cfg.x, cfg.box, p.rcut, 0.0, 256, neighcell=0)
            bi, bd, bv, _ = refpy.snap_descriptors(xa, al, nl, nn, p)
            xz, _, nlz, nnz = refpy.neighbor_list(cfg.x, cfg.box, outer, 0.0, 384, neighcell=0)
            ez, fz, vz = zbl.zbl_tally(xz, nlz, nnz, outer, inner=inner, outer=outer, z=z)
            er = np.concatenate([[n], bi])
            ey = m * fr.e - ez.sum()
            F = np.zeros((3 * n, nc))
            F[:, 1:] = bd.reshape(p.ncoeff, 3 * n).T
            fy = np.tile(fr.f, (m, 1)).ravel() - fz[:n].ravel()
            S = dataset.stress_rows(bv, cfg.box, m)
            sref = dataset.EV_PER_A3_IN_BAR / abs(np.linalg.det(cfg.box)) * vz.sum(axis=1)[list(dataset.BV_TO_VOIGT)]
            sy = np.array([fr.stress[i, j] for i, j in dataset.VOIGT]) - sref
            we, wf = grp.we / n, grp.wf / np.sqrt(m)
            A += we * we * np.outer(er, er) + wf * wf * F.T @ F + grp.ws * grp.ws * S.T @ S
            b += we * we * er * ey + wf * wf * F.T @ fy + grp.ws * grp.ws * S.T @ sy
            rows.append((grp.name, n, er, ey, F[:3 * n0], fy[:3 * n0], S, sy))
    beta = np.linalg.solve(A, b)
    rmse = lambda v: float(np.sqrt(np.mean(np.square(np.concatenate(v)))))
    out = {}
    for grp in groups:
        mine = [r for r in rows if r[0] == grp.name]
        out[grp.name] = (rmse([[(er @ beta - ey) / n] for _, n, er, ey, *_ in mine]),
                         rmse([F @ beta - fy for *_, F, fy, S, sy in mine]),
                         rmse([S @ beta - sy for *_, S, sy in mine]))
    return out


def test_fit_reproduces_published_errors():
    tab = published_table()
    ours = fit_errors(transpose_lattice=True)
    volume = ("Volume_A15", "Volume_BCC", "Volume_FCC")
    for name, (e, f, s) in ours.items():
        assert close(e, tab["Energy"][name][1], 1e-3), (name, e, tab["Energy"][name][1])
        assert close(s, tab["Stress"][name][1], 1e-3), (name, s, tab["Stress"][name][1])
        if name in volume:
            # perfect cubic cells, zero DFT forces: the fit predicts zero forces;
            # the table's finite RSQ shows its targets were not zero
            assert f < 1e-8, (name, f)
            assert tab["Force"][name][1] > 1.0 and np.isfinite(tab["Force"][name][2])
        else:
            assert close(f, tab["Force"][name][1], 1e-3), (name, f, tab["Force"][name][1])


def test_row_reading_removes_the_elastic_force_errors():
    """With the cell vectors read as rows, the strained 2- and 4-atom cells
    keep their symmetry and the model's forces there match the (near-zero)
    DFT forces."""
    tab = published_table()
    ours = fit_errors(transpose_lattice=False)
    for name in ("Elastic_BCC", "Elastic_FCC"):
        assert ours[name][1] < 1e-3 < 0.05 < tab["Force"][name][1], (name, ours[name][1])

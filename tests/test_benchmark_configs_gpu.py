"""GPU parity on the benchmark's own configurations, against MDP's CPU code.

C2 -- 20x20x20 BCC Ta cells = 16,000 atoms, 600 K, jitter 0.05 A, SNAP 2J=8
with seeded coefficients, 1,000 NVE steps of 1 fs:
  * ghost atoms and the full neighbour rows equal the reference's (its O(N^2)
    builder, cpuNeighborList3D.cpp; run here from oracle/_ref) as sorted index
    sets, and equal the row hashes stored in the fixture;
  * per-atom energy, forces and virial within 1e-10 of the reference's
    cpuSnap4.cpp chain (infinity norm relative to the largest value);
  * the 1,000-step trajectory against the reference's own trajectory
    (tests/golden/c2_bcc16000_2j8.npz, made by make_golden.py --c2): thermo
    rows every step, positions and velocities of every 8th atom at steps 100
    and 1,000 (positions within 1e-10 at step 1,000), the same number of
    neighbour-list builds, and the same energy drift per atom per ps (both
    printed).
C3 -- the 2,000,000-atom workload of the benchmark (100x100x100 cells, 300 K,
the same seeds as bench.py), one FP64 force evaluation against the reference's
CPU chain on this host's cores (about a minute):
  * neighbour rows (cell form) identical as sorted sets, through row hashes;
  * energy, forces and virial within 1e-10;
  * the FP32 form's force error against the reference (RMSE < 1e-4 eV/A).
"""
import os

import numpy as np
import pytest

from conftest import load_golden, row_hashes
from mdp_b200 import configs

pytestmark = pytest.mark.gpu

TOL_FP64 = 1e-10


def rel_inf(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def _ref():
    from oracle import refpy
    if not refpy.available():
        pytest.fail("oracle/_ref/libmdp_ref_harness.so missing (build with make -C oracle ref)")
    return refpy


def _threads():
    return max(1, os.cpu_count() or 1)


def _c2():
    g = load_golden("c2_bcc16000_2j8")
    p = configs.snap_params(int(g["twojmax"]), seed=int(g["coeff_seed"]))
    assert np.array_equal(p.coeff, g["coeff"])
    cfg = configs.ta_config(tuple(int(c) for c in g["cells"]), temp=float(g["temp"]), jitter=float(g["jitter"]),
                            seed=int(g["seed"]))
    # the fixture pins the input generator
    assert np.allclose([cfg.x.sum(), (cfg.x ** 2).sum()], g["x_check"], rtol=1e-13, atol=0)
    assert np.allclose([cfg.v.sum(), (cfg.v ** 2).sum()], g["v_check"], rtol=1e-12, atol=1e-12)
    return g, p, cfg


def test_c2_neighbors_and_forces_match_reference(cuda_lib):
    from mdp_b200.snap import snap_compute
    refpy = _ref()
    g, p, cfg = _c2()
    skin, nm = float(g["skin"]), int(g["neighmax"])
    out = snap_compute(p, cfg.x, cfg.box, skin, nm, want_neighbors=True)
    xa, al, nl, nn = refpy.neighbor_list(cfg.x, cfg.box, p.rcut, skin, nm, neighcell=0)
    assert out["anum"] - cfg.natoms == int(g["ghosts"]) == xa.shape[0] - cfg.natoms
    assert np.array_equal(out["xall"], xa), "ghost coordinates differ from the reference"
    assert np.array_equal(out["alist"], al), "ghost numbering differs from the reference"
    assert np.array_equal(out["neighnum"], nn)
    h = row_hashes(out["neighlist"], out["neighnum"])
    assert np.array_equal(h, row_hashes(nl, nn)), "neighbour rows differ from the reference"
    assert np.array_equal(h, g["row_hash"]), "neighbour rows differ from the fixture"
    e, f, v = refpy.snap_force(xa, al, nl, nn, p, nblocks=8 * _threads(), nthreads=_threads())
    assert np.allclose([e.sum(), (e ** 2).sum()], g["e_check"], rtol=1e-12, atol=0)
    assert rel_inf(out["eatom"], e) < TOL_FP64
    assert rel_inf(out["fatom"], f) < TOL_FP64
    assert rel_inf(out["vatom"], v) < TOL_FP64


# Tolerances of the 1,000-step comparison (relative infinity norms).  At these
# coefficients the run stays a stable crystal, and on the B200 the trajectory
# separated from the reference's by 2e-16 (positions) and 8e-14 (velocities)
# at step 100 and by 4.5e-15 and 2.8e-12 at step 1,000; the thermo rows agreed
# to 1.5e-15.  The bounds leave two orders of magnitude.
TRAJ_TOL = {100: (1e-12, 1e-11), 1000: (1e-10, 1e-9)}   # step: (positions, velocities)
THERMO_TOL = 1e-12           # thermo rows, relative to the largest |value| per column, all 1,000 steps
TE_TOL = 1e-10               # total energy per atom, eV/atom


def test_c2_trajectory_matches_reference(cuda_lib):
    from mdp_b200.snap import SnapMD
    g, p, cfg = _c2()
    md = SnapMD(p, cfg.box, cfg.natoms, float(g["md_dt"]), skin=float(g["skin"]), neighmax=int(g["neighmax"]))
    md.set_state(cfg.x, cfg.v)
    md.setup()
    atoms = g["md_atoms"]
    ref = g["md_thermo"]
    th100, _ = md.run(100, thermo_every=1)
    x100, v100, _, _ = md.state()
    th900, _ = md.run(int(g["md_steps"]) - 100, thermo_every=1)
    x1k, v1k, _, _ = md.state()
    rebuilds = md.counters()["rebuilds"]
    md.close()
    th = np.vstack([th100, th900])
    assert th.shape[0] == ref.shape[0] - 1
    assert np.array_equal(th[:, 0], ref[1:, 0])
    dth = np.abs(th[:, 1:] - ref[1:, 1:]).max(axis=0) / np.abs(ref[1:, 1:]).max(axis=0)
    sep = {100: (rel_inf(x100[atoms], g["md_x_100"]), rel_inf(v100[atoms], g["md_v_100"])),
           1000: (rel_inf(x1k[atoms], g["md_x_1000"]), rel_inf(v1k[atoms], g["md_v_1000"]))}
    ps = float(g["md_steps"]) * float(g["md_dt"])
    drift = (th[-1, 3] - th[0, 3]) / ps
    drift_ref = (ref[-1, 3] - ref[1, 3]) / ps
    print(f"C2 separation from the reference: step 100 x {sep[100][0]:.2e} v {sep[100][1]:.2e}; "
          f"step 1000 x {sep[1000][0]:.2e} v {sep[1000][1]:.2e}; thermo {dth.max():.2e}; "
          f"TE/atom drift {drift:.3e} eV/ps (reference {drift_ref:.3e}); list builds {rebuilds} "
          f"(reference {int(g['md_rebuilds'])})")
    assert dth.max() < THERMO_TOL
    assert rebuilds == int(g["md_rebuilds"])
    for st, (tx, tv) in TRAJ_TOL.items():
        assert sep[st][0] < tx and sep[st][1] < tv, (st, sep[st])
    assert np.abs(th[:, 3] - ref[1:, 3]).max() < TE_TOL
    assert abs(drift - drift_ref) < TE_TOL / ps


C3_CELLS = (100, 100, 100)


def test_c3_full_size_force_matches_reference(cuda_lib):
    """One FP64 evaluation of the 2,000,000-atom benchmark configuration (the
    bench's seeds) against the reference's CPU chain; FP32 error against it."""
    from mdp_b200.snap import snap_compute
    refpy = _ref()
    p = configs.snap_params(8, seed=2024)
    cfg = configs.ta_config(C3_CELLS, temp=300.0, jitter=0.05, seed=2024)
    skin, nm = 1.0, 64
    out = snap_compute(p, cfg.x, cfg.box, skin, nm, want_neighbors=True)
    xa, al, nl, nn = refpy.neighbor_list(cfg.x, cfg.box, p.rcut, skin, nm, neighcell=1)
    assert nn.max() < nm
    assert out["anum"] == xa.shape[0]
    assert np.array_equal(out["xall"], xa), "ghost coordinates differ from the reference"
    assert np.array_equal(out["alist"], al), "ghost numbering differs from the reference"
    assert np.array_equal(out["neighnum"], nn)
    assert np.array_equal(row_hashes(out["neighlist"], out["neighnum"]), row_hashes(nl, nn)), \
        "neighbour rows differ from the reference"
    del out["neighlist"], out["xall"]
    e, f, v = refpy.snap_force(xa, al, nl, nn, p, nblocks=8 * _threads(), nthreads=_threads())
    del xa, al, nl
    assert rel_inf(out["eatom"], e) < TOL_FP64
    assert rel_inf(out["fatom"], f) < TOL_FP64
    assert rel_inf(out["vatom"], v) < TOL_FP64
    o32 = snap_compute(p, cfg.x, cfg.box, skin, nm, precision="fp32")
    df = o32["fatom"] - f
    rmse, mx = float(np.sqrt(np.mean(df ** 2))), float(np.abs(df).max())
    print(f"C3 FP32 vs reference: force RMSE {rmse:.2e} eV/A, max {mx:.2e} eV/A; "
          f"energy max {np.abs(o32['eatom'] - e).max():.2e} eV")
    assert rmse < 1e-4 and mx < 1e-3

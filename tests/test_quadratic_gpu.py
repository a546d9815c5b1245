"""GPU: quadratic SNAP (quadraticflag = 1) in the force path and the MD engine.

The reference evaluates the quadratic terms in its ComputePairSnap chain
(snappotential.cpp:236-410): per-atom coefficients beta + Q B_i
(cpuComputeBeta2) and energies beta0 + beta . B_i + B_i^T Q B_i / 2
(cpuSnapTallyEnergyFull, cpuSnap.cpp:1713-1770).  The fixtures
tests/golden/quad_*.npz hold that chain's energies, forces and virials
(make_golden.py --quad, oracle/_ref build); the GPU path -- U, per-atom B,
the quadratic coefficients, Y with per-atom coefficients, dE/dr and the
tally -- matches them within 1e-10, and NVE with the quadratic model
conserves energy.
"""
import glob
import os

import numpy as np
import pytest

from conftest import GOLDEN, load_golden
from mdp_b200 import configs

pytestmark = pytest.mark.gpu

TOL = 1e-10
NAMES = sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN, "quad_*.npz")))


def rel_inf(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def params(g):
    bnorm, bzero, switch = (int(v) for v in g["flags"])
    p = configs.snap_params(int(g["twojmax"]), seed=int(g["coeff_seed"]), quadraticflag=1, bnormflag=bnorm,
                            bzeroflag=bzero, switchflag=switch)
    assert np.array_equal(p.coeff, g["coeff"])
    return p


@pytest.mark.parametrize("name", NAMES)
def test_quadratic_forces_match_reference(cuda_lib, name):
    from mdp_b200.snap import snap_compute
    g = load_golden(name)
    p = params(g)
    out = snap_compute(p, g["x"], g["box"], float(g["skin"]), int(g["neighmax"]))
    assert rel_inf(out["eatom"], g["eatom"]) < TOL
    assert rel_inf(out["fatom"], g["fatom"]) < TOL
    assert rel_inf(out["vatom"], g["vatom"]) < TOL


def test_quadratic_is_fp64_only(cuda_lib):
    from mdp_b200 import _lib
    from mdp_b200.snap import snap_compute
    g = load_golden(NAMES[0])
    with pytest.raises(_lib.MdpError, match="FP64"):
        snap_compute(params(g), g["x"], g["box"], float(g["skin"]), int(g["neighmax"]), precision="fp32")


def test_quadratic_md_conserves_energy(cuda_lib):
    from mdp_b200.snap import SnapMD
    p = configs.snap_params(8, seed=2022, quadraticflag=1)
    cfg = configs.ta_config((6, 6, 6), temp=300.0, jitter=0.05, seed=5)
    md = SnapMD(p, cfg.box, cfg.natoms, 0.0005)
    md.set_state(cfg.x, cfg.v)
    md.setup()
    th, _ = md.run(200, thermo_every=20)
    md.close()
    te = th[:, 3]
    assert np.all(np.isfinite(te))
    assert np.abs(te - te[0]).max() < 1e-4, te

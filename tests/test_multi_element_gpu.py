"""GPU: several element types (nelements > 1, chemflag 0 and 1) in the FP64
force path, against the reference's ComputePairSnap3 chain.

The fixtures tests/golden/chem_*.npz (make_golden.py --chem, reference
build) hold random type assignments on Ta-like BCC cells with per-element
radii, weights and coefficient tables: two elements at 2J = 6 and 8, three
elements at 2J = 4 with bnorm / bzero, wselfallflag, and chemflag = 0.  The
GPU path -- pairs grouped per element block, U of the element blocks,
element-triple energies, Y per block, dE/dr with per-pair cutoffs -- matches
energies, forces and virials within 1e-10 (relative to the largest entry).
"""
import ctypes as C
import glob
import os

import numpy as np
import pytest

from conftest import GOLDEN, load_golden
from mdp_b200 import configs

pytestmark = pytest.mark.gpu

TOL = 1e-10
NAMES = sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN, "chem_*.npz")))


def rel_inf(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def params(g):
    bnorm, bzero, switch, wsa = (int(v) for v in g["flags"])
    p = configs.snap_params_elements(int(g["twojmax"]), g["radelems"], g["wjelems"], chemflag=int(g["chemflag"]),
                                     seed=int(g["coeff_seed"]), bnormflag=bnorm, bzeroflag=bzero,
                                     switchflag=switch, wselfallflag=wsa)
    assert np.array_equal(p.coeff, g["coeff"])
    return p


@pytest.mark.parametrize("name", NAMES)
def test_multi_element_forces_match_reference(cuda_lib, name):
    from mdp_b200.snap import snap_compute
    g = load_golden(name)
    out = snap_compute(params(g), g["x"], g["box"], float(g["skin"]), int(g["neighmax"]), types=g["types"])
    de, df, dv = (rel_inf(out["eatom"], g["eatom"]), rel_inf(out["fatom"], g["fatom"]),
                  rel_inf(out["vatom"], g["vatom"]))
    print(f"{name}: energy {de:.1e} forces {df:.1e} virial {dv:.1e}")
    assert de < TOL and df < TOL and dv < TOL


def test_device_entry_on_reference_neighbour_list(cuda_lib):
    """mdp_snap_compute_device_typed on the reference's own ghosts, owner list
    and neighbour rows (device arrays)."""
    import torch
    from mdp_b200 import _lib
    g = load_golden("chem_bcc128_2j6")
    p = params(g)
    sp, keep = _lib.snap_params_c(p)
    L = _lib.lib()
    n, nm = g["neighlist"].shape
    anum = g["xall"].shape[0]
    t = lambda a, dt: torch.from_numpy(np.ascontiguousarray(a, dtype=dt).copy()).cuda()
    x = t(g["xall"], np.float64); ty = t(g["types"], np.int32); al = t(g["alist"], np.int32)
    nl = t(g["neighlist"], np.int32); nn = t(g["neighnum"], np.int32)
    e = torch.zeros(n, dtype=torch.float64, device="cuda"); f = torch.zeros(3 * n, dtype=torch.float64, device="cuda")
    v = torch.zeros(6 * n, dtype=torch.float64, device="cuda")
    rc = L.mdp_snap_compute_device_typed(C.byref(sp), 0, x.data_ptr(), ty.data_ptr(), al.data_ptr(), nl.data_ptr(),
                                         nn.data_ptr(), n, anum, nm, e.data_ptr(), f.data_ptr(), v.data_ptr(), None)
    _lib.check(rc, "mdp_snap_compute_device_typed")
    torch.cuda.synchronize()
    assert rel_inf(e.cpu().numpy(), g["eatom"]) < TOL
    assert rel_inf(f.cpu().numpy().reshape(n, 3), g["fatom"]) < TOL
    assert rel_inf(v.cpu().numpy().reshape(6, n), g["vatom"]) < TOL


def test_refusals(cuda_lib):
    from mdp_b200 import _lib
    from mdp_b200.snap import snap_compute
    g = load_golden("chem_bcc54_2j4_3el_flags")
    p = params(g)
    args = (p, g["x"], g["box"], float(g["skin"]), int(g["neighmax"]))
    with pytest.raises(_lib.MdpError, match="types"):
        snap_compute(*args)
    with pytest.raises(_lib.MdpError, match="FP64"):
        snap_compute(*args, precision="fp32", types=g["types"])
    bad = g["types"].copy(); bad[3] = 4
    with pytest.raises(_lib.MdpError, match="type 4"):
        snap_compute(*args, types=bad)


def test_two_element_md_conserves_energy(cuda_lib):
    """NVE with two element types (chemflag = 0, whose forces are the exact
    gradient of its energy)."""
    from mdp_b200.snap import SnapMD
    p = configs.snap_params_elements(8, (0.5, 0.45), (1.0, 0.8), chemflag=0, seed=2022)
    cfg = configs.ta_config((6, 6, 6), temp=300.0, jitter=0.05, seed=5)
    types = np.random.default_rng(9).integers(1, 3, cfg.natoms).astype(np.int32)
    md = SnapMD(p, cfg.box, cfg.natoms, 0.0005)
    md.set_types(types)
    md.set_state(cfg.x, cfg.v)
    md.setup()
    th, _ = md.run(200, thermo_every=20)
    md.close()
    te = th[:, 3]
    assert np.all(np.isfinite(te))
    assert np.abs(te - te[0]).max() < 1e-4, te

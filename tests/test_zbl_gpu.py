"""GPU: the ZBL pair term of MDP's snapTA06A example added to SNAP by the MD
engine (mdp_md_set_zbl), against the reference: golden SNAP forces and
energies plus the ZBL term tallied as MDP's full-list pair driver tallies it,
with the pair potential of MDP's generated code (restated in oracle/zbl.py and
pinned to that code in tests/test_oracle.py).  Also energy conservation of
SNAP + ZBL MD and the cutoff check."""
import numpy as np
import pytest

from conftest import golden_params, load_golden
from mdp_b200 import configs

pytestmark = pytest.mark.gpu


def rel_inf(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


@pytest.mark.parametrize("name", ["bcc250_2j8", "bcc250_2j8_hot", "bcc54_2j8_flags"])
def test_snap_plus_zbl_matches_reference(cuda_lib, name):
    from mdp_b200.snap import SnapMD
    from oracle import zbl
    g = load_golden(name)
    p = golden_params(g)
    n = g["x"].shape[0]
    md = SnapMD(p, g["box"], n, 0.001, skin=float(g["skin"]), neighmax=int(g["neighmax"]))
    md.set_zbl(4.0, 4.8, 73.0)
    md.set_state(np.ascontiguousarray(g["x"]), np.zeros((n, 3)))
    md.setup()
    _, _, f, e = md.state()
    md.close()
    ez, fz, _ = zbl.zbl_tally(g["xall"], g["neighlist"], g["neighnum"], 4.8)
    assert np.abs(fz).max() > 0.1          # the term is not negligible here
    assert rel_inf(f, g["fatom"] + fz) < 1e-10
    assert rel_inf(e, g["eatom"] + ez) < 1e-10


def test_snap_plus_zbl_md_conserves_energy(cuda_lib):
    from mdp_b200.snap import SnapMD
    p = configs.snap_params(8, seed=21)
    cfg = configs.ta_config((8, 8, 8), temp=600, jitter=0.05, seed=21)
    md = SnapMD(p, cfg.box, cfg.natoms, 0.001)
    md.set_zbl()
    md.set_state(cfg.x, cfg.v)
    md.setup()
    th, _ = md.run(200, thermo_every=50)
    md.close()
    te = th[:, 3]
    assert np.abs(te - te[0]).max() < 2e-4   # eV/atom over 0.2 ps


def test_zbl_cutoff_beyond_neighbour_reach_is_an_error(cuda_lib):
    from mdp_b200 import _lib
    from mdp_b200.snap import SnapMD
    p = configs.snap_params(8, seed=21)
    cfg = configs.ta_config((8, 8, 8), temp=300, jitter=0.05, seed=21)
    md = SnapMD(p, cfg.box, cfg.natoms, 0.001, skin=0.1)
    with pytest.raises(_lib.MdpError, match="ZBL cutoff"):
        md.set_zbl(4.0, 4.8, 73.0)
    md.close()

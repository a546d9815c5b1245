"""GPU: size-independent properties at the full benchmark size (2,000,000-atom
BCC Ta, 2J=8), where the oracle would take hours: Newton's third law of the
pair tally, forces as energy gradients (central differences of the total
energy), the FP32 form's force error, and NVE energy conservation."""
import numpy as np
import pytest

from mdp_b200 import configs

pytestmark = pytest.mark.gpu

CELLS = (100, 100, 100)


@pytest.fixture(scope="module")
def full():
    from mdp_b200.snap import snap_compute
    p = configs.snap_params(8, seed=2024)
    cfg = configs.ta_config(CELLS, temp=300.0, jitter=0.05, seed=2024)
    out = snap_compute(p, cfg.x, cfg.box, 1.0, 64, precision="fp64")
    return p, cfg, out


def test_forces_sum_to_zero(cuda_lib, full):
    _, cfg, out = full
    f = out["fatom"]
    assert cfg.natoms == 2_000_000
    assert np.isfinite(f).all() and np.isfinite(out["eatom"]).all()
    # every pair adds +dE to its atom and -dE to its neighbour's owner
    assert np.abs(f.sum(axis=0)).max() < 1e-8


def test_forces_are_energy_gradients(cuda_lib, full):
    from mdp_b200.snap import snap_compute
    p, cfg, out = full
    h = 1e-5
    rng = np.random.default_rng(7)
    for k in rng.choice(cfg.natoms, 3, replace=False):
        for d in range(3):
            xs = []
            for sgn in (1.0, -1.0):
                x = cfg.x.copy()
                x[k, d] = np.mod(x[k, d] + sgn * h, cfg.box[d])
                xs.append(snap_compute(p, x, cfg.box, 1.0, 64, precision="fp64")["eatom"])
            # per-atom differences first: only atoms near k change
            fd = -(xs[0] - xs[1]).sum() / (2 * h)
            assert abs(fd - out["fatom"][k, d]) < 1e-6 * max(1.0, abs(out["fatom"][k, d])), (k, d)


def test_fp32_force_error_full_size(cuda_lib, full):
    from mdp_b200.snap import snap_compute
    p, cfg, out = full
    f32 = snap_compute(p, cfg.x, cfg.box, 1.0, 64, precision="fp32")["fatom"]
    err = f32 - out["fatom"]
    assert np.sqrt(np.mean(err ** 2)) < 1e-4          # eV/A, the FP32 form's tolerance
    assert np.abs(err).max() < 1e-3


def test_nve_energy_conservation_full_size(cuda_lib):
    from mdp_b200.snap import SnapMD
    p = configs.snap_params(8, seed=2024)
    cfg = configs.ta_config(CELLS, temp=300.0, jitter=0.05, seed=2024)
    md = SnapMD(p, cfg.box, cfg.natoms, 0.001, skin=1.0, neighmax=64)
    md.set_state(cfg.x, cfg.v)
    md.setup()
    th, _ = md.run(20, thermo_every=10)
    md.close()
    te = th[:, 3]
    assert np.isfinite(te).all()
    assert np.abs(te - te[0]).max() < 1e-5      # eV/atom over 20 fs

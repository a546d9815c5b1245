"""GPU parity tests: the CUDA SNAP path, called through the C ABI, against
the golden fixtures (reference CPU results) and against the oracle."""
import numpy as np
import pytest

from conftest import golden_names, golden_params, load_golden
from mdp_b200 import configs

pytestmark = pytest.mark.gpu

# Appendix A.7 style norms: relative to the largest magnitude in the reference
TOL_FP64 = 1e-10


def rel_inf(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def sorted_rows(nl, nn):
    return [tuple(sorted(nl[i, : nn[i]].tolist())) for i in range(len(nn))]


@pytest.mark.parametrize("name", golden_names())
def test_neighbors_bit_exact(cuda_lib, name):
    from mdp_b200.snap import snap_compute
    g = load_golden(name)
    p = golden_params(g)
    out = snap_compute(p, g["x"], g["box"], float(g["skin"]), int(g["neighmax"]), want_neighbors=True)
    assert out["anum"] == g["xall"].shape[0]
    assert np.array_equal(out["xall"], g["xall"]), "ghost coordinates differ from the reference"
    assert np.array_equal(out["alist"], g["alist"]), "ghost numbering differs from the reference"
    assert sorted_rows(out["neighlist"], out["neighnum"]) == sorted_rows(g["neighlist"], g["neighnum"])


@pytest.mark.parametrize("name", golden_names())
def test_fp64_matches_reference(cuda_lib, name):
    from mdp_b200.snap import snap_compute
    g = load_golden(name)
    p = golden_params(g)
    out = snap_compute(p, g["x"], g["box"], float(g["skin"]), int(g["neighmax"]))
    assert rel_inf(out["eatom"], g["eatom"]) < TOL_FP64
    assert rel_inf(out["fatom"], g["fatom"]) < TOL_FP64
    assert rel_inf(out["vatom"], g["vatom"]) < TOL_FP64


@pytest.mark.parametrize("name", ["bcc250_2j8", "bcc128_2j6", "bcc250_2j8_hot"])
def test_fp32_force_error(cuda_lib, name):
    from mdp_b200.snap import snap_compute
    g = load_golden(name)
    p = golden_params(g)
    out = snap_compute(p, g["x"], g["box"], float(g["skin"]), int(g["neighmax"]), precision="fp32")
    rmse = np.sqrt(np.mean((out["fatom"] - g["fatom"]) ** 2))
    assert rmse < 1e-4, rmse
    assert np.abs(out["eatom"] - g["eatom"]).max() < 1e-4


def test_fp64_matches_oracle_2000_atoms(cuda_lib):
    from mdp_b200.snap import snap_compute
    from oracle import oracle
    p = configs.snap_params(8, seed=77)
    cfg = configs.ta_config((10, 10, 10), temp=600, jitter=0.05, seed=7)
    xa, al, nl, nn = oracle.neighbor_list(cfg.x, cfg.box, p.rcut, 1.0, 80)
    e, f, v = oracle.snap_force(xa, al, nl, nn, p)
    out = snap_compute(p, cfg.x, cfg.box, 1.0, 80, want_neighbors=True)
    assert sorted_rows(out["neighlist"], out["neighnum"]) == sorted_rows(nl, nn)
    assert rel_inf(out["eatom"], e) < TOL_FP64
    assert rel_inf(out["fatom"], f) < TOL_FP64
    assert rel_inf(out["vatom"], v) < TOL_FP64


def test_md_trajectory_matches_reference(cuda_lib):
    from mdp_b200.snap import SnapMD
    g = load_golden("bcc128_2j6")
    p = golden_params(g)
    md = SnapMD(p, g["box"], g["x"].shape[0], float(g["md_dt"]), skin=float(g["skin"]), neighmax=int(g["neighmax"]))
    md.set_state(g["x"], g["v"])
    md.setup()
    th, _ = md.run(int(g["md_steps"]), thermo_every=1)
    x, v, f, e = md.state()
    ref = g["md_thermo"]
    assert np.abs(th[:, 1:] - ref[1:, 1:]).max() / np.abs(ref[1:, 1:]).max() < 1e-9
    assert rel_inf(x, g["md_x"]) < 1e-10
    assert rel_inf(v, g["md_v"]) < 1e-8
    assert rel_inf(e, g["md_e"]) < 1e-10
    assert md.counters()["rebuilds"] >= 1
    md.close()


def test_md_energy_conservation_2j8(cuda_lib):
    from mdp_b200.snap import SnapMD
    p = configs.snap_params(8, seed=21)
    cfg = configs.ta_config((8, 8, 8), temp=600, jitter=0.05, seed=21)
    md = SnapMD(p, cfg.box, cfg.natoms, 0.001)
    md.set_state(cfg.x, cfg.v)
    md.setup()
    th, _ = md.run(200, thermo_every=50)
    te = th[:, 3]
    assert np.abs(te - te[0]).max() < 2e-4, te   # eV/atom over 0.2 ps
    md.close()


def test_md_setup_on_reused_memory_matches_one_shot(cuda_lib):
    """The MD engine's first evaluation, on buffers freshly grown while the
    device memory still holds other data, equals the one-shot path on the same
    positions for every atom (250,000 atoms at 1,000 K, neighmax 96).  A zero
    fill that was not ordered with the engine's stream once corrupted a few
    atoms of exactly this evaluation."""
    import torch
    from mdp_b200.snap import SnapMD, snap_compute
    p = configs.snap_params(8, seed=2024)
    cfg = configs.ta_config((50, 50, 50), temp=1000.0, jitter=0.05 * np.sqrt(1000.0 / 300.0), seed=2025)
    junk = torch.full((1 << 30,), float("nan"), dtype=torch.float64, device="cuda")   # 8 GB of NaN bytes
    del junk
    torch.cuda.synchronize()
    torch.cuda.empty_cache()
    md = SnapMD(p, cfg.box, cfg.natoms, 0.001, skin=1.0, neighmax=96)
    md.set_state(cfg.x, cfg.v)
    md.setup()
    _, _, f, e = md.state()
    md.close()
    ref = snap_compute(p, cfg.x, cfg.box, 1.0, 96)
    assert np.isfinite(f).all() and np.isfinite(e).all()
    assert rel_inf(f, ref["fatom"]) < TOL_FP64
    assert rel_inf(e, ref["eatom"]) < TOL_FP64


def test_neighbor_overflow_is_an_error(cuda_lib):
    from mdp_b200 import _lib
    from mdp_b200.snap import snap_compute
    g = load_golden("bcc54_2j8_flags")
    p = golden_params(g)
    with pytest.raises(_lib.MdpError, match="neighmax"):
        snap_compute(p, g["x"], g["box"], 1.0, 16)
    # the library stays usable after the error
    out = snap_compute(p, g["x"], g["box"], float(g["skin"]), int(g["neighmax"]))
    assert rel_inf(out["fatom"], g["fatom"]) < TOL_FP64


def test_device_entry_point(cuda_lib):
    """mdp_snap_compute_device on device arrays in the reference's layouts."""
    import ctypes as C
    import torch
    from mdp_b200 import _lib
    g = load_golden("bcc250_2j8")
    p = golden_params(g)
    sp, keep = _lib.snap_params_c(p)
    dev = torch.device("cuda:0")
    x = torch.tensor(g["xall"], dtype=torch.float64, device=dev).contiguous()
    al = torch.tensor(g["alist"], dtype=torch.int32, device=dev)
    nl = torch.tensor(g["neighlist"], dtype=torch.int32, device=dev).contiguous()
    nn = torch.tensor(g["neighnum"], dtype=torch.int32, device=dev)
    n, nm = g["neighlist"].shape
    e = torch.zeros(n, dtype=torch.float64, device=dev)
    f = torch.zeros(n, 3, dtype=torch.float64, device=dev)
    v = torch.zeros(6, n, dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream().cuda_stream
    rc = cuda_lib.mdp_snap_compute_device(C.byref(sp), 0, x.data_ptr(), al.data_ptr(), nl.data_ptr(), nn.data_ptr(),
                                          n, x.shape[0], nm, e.data_ptr(), f.data_ptr(), v.data_ptr(), stream)
    _lib.check(rc)
    torch.cuda.synchronize()
    assert rel_inf(e.cpu().numpy(), g["eatom"]) < TOL_FP64
    assert rel_inf(f.cpu().numpy(), g["fatom"]) < TOL_FP64
    assert rel_inf(v.cpu().numpy(), g["vatom"]) < TOL_FP64

"""GPU: force constraints, set-velocity integration and the velocity-rescaling
thermostats of the backend dispatch (mdpgpucore.h:303-349, here
mdp_b200/csrc/abi_fix.cu) against MDP's own CPU functions (cpuFixes.cpp,
cpuVelocityIntegration.cpp), compiled from the reference tree behind
oracle/ref_harness.cpp, on identical inputs.

Tolerances: 1e-13 relative to the largest entry for the plain arithmetic
(rounded in the reference's order, so mostly bit-identical), 1e-12 where the
group sums differ in order (ave force, thermostat temperatures) or where CUDA's
exp / pow meet the host's (LJ 10-4-3 and Morse walls).  Two documented
departures from the CPU code are checked against their formula instead: the
line / plane force projects the z component on fparam[2], as the reference's
own GPU kernels do (cpuFixes.cpp uses fparam[1]).
"""
import ctypes as C

import numpy as np
import pytest

from oracle import refpy
from test_gpucore_md import dev, ptr, sync
from test_gpucore_md import _release_tensors  # noqa: F401  (autouse fixture)

pytestmark = pytest.mark.gpu

P = C.c_void_p
FIX_KINDS = {"set_force": 0, "line_force": 1, "plane_force": 2, "ave_force": 3, "wall_reflect": 4,
             "wall_harmonic": 5, "wall_lj93": 6, "wall_lj126": 7, "wall_lj1043": 8, "wall_morse": 9}


def rel(a, b):
    return np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(b).max(), 1e-300)


def hp(a):
    return C.c_void_p(a.ctypes.data)


def ref():
    R = refpy.lib()
    R.ref_fix.argtypes = [C.c_int] + [P] * 11 + [C.c_int] * 5
    R.ref_set_velocity.argtypes = [C.c_int] + [P] * 5 + [C.c_double, C.c_double] + [P] * 3 + [C.c_int] * 2
    R.ref_velocity_rescaling.argtypes = [P] * 5 + [C.c_double] + [P] * 4 + [C.c_int] * 4
    R.ref_velocity_rescaling.restype = C.c_double
    return R


def ours(S="f64"):
    from mdp_b200 import _lib
    L = _lib.lib()
    real = C.c_double if S == "f64" else C.c_float
    for k in FIX_KINDS:
        getattr(L, f"mdp_gpu_fix_{k}_{S}").argtypes = [P] * 8 + [C.c_int] * 4
    getattr(L, f"mdp_gpu_fix_add_force_{S}").argtypes = [P] * 10 + [C.c_int] * 5
    getattr(L, f"mdp_gpu_fix_drag_force_{S}").argtypes = [P] * 10 + [C.c_int] * 5
    getattr(L, f"mdp_gpu_set_velocity_initial_integrate_{S}").argtypes = [P] * 5 + [real, real] + [P] * 3 + \
        [C.c_int] * 2
    getattr(L, f"mdp_gpu_set_velocity_final_integrate_{S}").argtypes = [P] * 4 + [real] + [P] * 3 + [C.c_int] * 2
    fn = getattr(L, f"mdp_gpu_velocity_rescaling_thermostat_{S}")
    fn.argtypes = [P] * 7 + [real] + [P] * 4 + [C.c_int] * 4
    fn.restype = real
    return L


def system(seed, n=4000, dim=3, box=20.0):
    rng = np.random.default_rng(seed)
    x = rng.uniform(0.0, box, size=(n, dim))
    v = rng.normal(size=(n, dim)) * 3.0
    f = rng.normal(size=(n, dim)) * 5.0
    eatom = rng.normal(size=n)
    vatom = rng.normal(size=(n, 6))
    ilist = rng.permutation(n).astype(np.int32)[: n - 137]
    return rng, dict(x=x, v=v, f=f, eatom=eatom, vatom=vatom), ilist


WALL_PARAMS = {
    "wall_harmonic": [2.5, 3.0, 1.7],
    "wall_lj93": [2.5, 3.0, 0.013, 1.3, 0.9, 0.7, 1.1],
    "wall_lj126": [2.5, 3.0, 0.021, 2.2, 1.4, 0.6, 0.8],
    "wall_lj1043": [2.5, 3.0, 0.017, 1.1, 0.9, 0.4, 0.3, 2.1, 1.6, 0.25],
    "wall_morse": [2.5, 3.0, 0.05, 1.3, 1.7, 2.9],
}


def run_fix(kind, arrays, fparam, iparam, ilist, eflag, vflag, dim):
    """(reference host result, ours) for one of the common-signature fixes."""
    R, L = ref(), ours()
    a = {k: np.ascontiguousarray(v.copy()) for k, v in arrays.items()}
    fp = np.ascontiguousarray(fparam, dtype=np.float64); ip = np.ascontiguousarray(iparam, dtype=np.int32)
    R.ref_fix(FIX_KINDS[kind], hp(a["x"]), hp(a["v"]), hp(a["f"]), hp(a["eatom"]), hp(a["vatom"]), hp(fp), hp(ip),
              hp(ilist), None, None, None, 0, eflag, vflag, dim, len(ilist))
    d = {k: dev(v) for k, v in arrays.items()}
    getattr(L, f"mdp_gpu_fix_{kind}_f64")(ptr(d["x"]), ptr(d["v"]), ptr(d["f"]), ptr(d["eatom"]), ptr(d["vatom"]),
                                          ptr(dev(fp)), ptr(dev(ip)), ptr(dev(ilist)), eflag, vflag, dim, len(ilist))
    sync()
    return a, {k: t.cpu().numpy() for k, t in d.items()}


@pytest.mark.parametrize("dim", [3, 2])
def test_set_and_ave_force(cuda_lib, dim):
    """In two dimensions cpuFixAveForce still tests iparam[2] and, when it is
    set, writes f[i*dim+2] -- the next atom's x (cpuFixes.cpp:292).  The
    entry point sets components d < dim only; the test passes iparam[2] = 0,
    where the two agree."""
    _, arrays, ilist = system(1, dim=dim)
    for kind, fp, ip, tol in (("set_force", [0.3, -1.2, 2.5][:dim], [1, 0, 1][:dim], 0.0),
                              ("ave_force", [0.3, -1.2, 2.5][:dim], [1, 1, 0] if dim == 2 else [1, 1, 0], 1e-12)):
        a, b = run_fix(kind, arrays, fp, ip, ilist, 1, 1, dim)
        assert rel(b["f"], a["f"]) <= tol, kind
        assert np.array_equal(b["x"], a["x"]) and np.array_equal(b["eatom"], a["eatom"])


@pytest.mark.parametrize("dim", [3, 2])
def test_line_and_plane_force(cuda_lib, dim):
    _, arrays, ilist = system(2, dim=dim)
    p = np.array([0.48, -0.6, 0.64][:dim])
    for kind in ("line_force", "plane_force"):
        a, b = run_fix(kind, arrays, p, [0, 0, 0], ilist, 0, 0, dim)
        f0 = arrays["f"][ilist]
        dot = f0[:, 0] * p[0] + f0[:, 1] * p[1]
        if dim == 3:
            dot = dot + f0[:, 2] * p[2]
        assert rel(b["f"][:, :2], a["f"][:, :2]) < 1e-15, kind          # x, y as the CPU code
        if dim == 3:                                                    # z on fparam[2] (gpuFixes.cu)
            want = dot * p[2] if kind == "line_force" else f0[:, 2] - dot * p[2]
            assert rel(b["f"][ilist, 2], want) < 1e-15, kind


@pytest.mark.parametrize("side", range(6))
@pytest.mark.parametrize("kind", sorted(WALL_PARAMS) + ["wall_reflect"])
def test_walls(cuda_lib, kind, side):
    rng, arrays, ilist = system(3 + side, box=6.0)
    fp = WALL_PARAMS.get(kind, [2.5])
    if kind == "wall_reflect":
        fp = [3.0]
    for eflag, vflag in ((1, 1), (1, 0), (0, 1)):
        a, b = run_fix(kind, arrays, fp, [side], ilist, eflag, vflag, 3)
        tol = 1e-12 if kind in ("wall_lj1043", "wall_morse") else 1e-13
        for k in ("x", "v", "f", "eatom", "vatom"):
            assert rel(b[k], a[k]) < tol, (kind, side, k)
        assert not np.array_equal(a["f"], arrays["f"]) or kind == "wall_reflect"


@pytest.mark.parametrize("triclinic", [0, 1])
@pytest.mark.parametrize("dim", [3, 2])
def test_add_and_drag_force(cuda_lib, triclinic, dim):
    R, L = ref(), ours()
    rng, arrays, ilist = system(9, dim=dim)
    n = arrays["x"].shape[0]
    box = np.array([20.0, 18.0, 16.0, 1.5, -2.0, 0.75])   # h: lengths, then yz, xz, xy tilts
    image = rng.integers(-3, 4, size=(n, dim)).astype(np.int32)
    pbc = np.array([1, 1, 1], dtype=np.int32)
    fp_add = np.array([0.3, -1.2, 2.5][:dim] + [0.0] * (3 - dim))
    fp_drag = np.array([0.8, 0.5, 3.0, 55.0, -41.0])     # far from the box: several image shifts
    for kind, fp, ip, idx in ((10, fp_add, [1, 1, 1], image), (11, fp_drag, [1, 1, 0], pbc)):
        a = {k: v.copy() for k, v in arrays.items()}
        R.ref_fix(kind, hp(a["x"]), hp(a["v"]), hp(a["f"]), hp(a["eatom"]), hp(a["vatom"]), hp(fp),
                  hp(np.array(ip, np.int32)), hp(ilist), hp(box), hp(image), hp(pbc), triclinic, 1, 1, dim, len(ilist))
        d = {k: dev(v) for k, v in arrays.items()}
        fn = L.mdp_gpu_fix_add_force_f64 if kind == 10 else L.mdp_gpu_fix_drag_force_f64
        fn(ptr(d["x"]), ptr(d["v"]), ptr(d["f"]), ptr(d["eatom"]), ptr(d["vatom"]), ptr(dev(fp)), ptr(dev(box)),
           ptr(dev(np.array(ip, np.int32))), ptr(dev(ilist)), ptr(dev(idx)), triclinic, 1, 1, dim, len(ilist))
        sync()
        for k in ("f", "eatom", "vatom"):
            assert rel(d[k].cpu().numpy(), a[k]) < 1e-13, (kind, k)


@pytest.mark.parametrize("dim", [3, 2])
def test_set_velocity_integration(cuda_lib, dim):
    R, L = ref(), ours()
    rng, arrays, ilist = system(11, dim=dim)
    n = arrays["x"].shape[0]
    mass = np.array([0.0, 180.88, 92.9]); typ = rng.integers(1, 3, n).astype(np.int32)
    fp = np.array([0.5, -0.25, 1.0][:dim]); ip = np.array([1, 0, 1][:dim], np.int32)
    dtf, dtv = 0.5 * 0.001 / 1.0364269e-4, 0.001
    x, v = arrays["x"].copy(), arrays["v"].copy()
    dx, dv, df = dev(x), dev(v), dev(arrays["f"])
    for stage in (0, 1, 0, 1):
        R.ref_set_velocity(stage, hp(x), hp(v), hp(arrays["f"]), hp(mass), hp(fp), dtf, dtv, hp(typ), hp(ilist),
                           hp(ip), dim, len(ilist))
        if stage == 0:
            L.mdp_gpu_set_velocity_initial_integrate_f64(ptr(dx), ptr(dv), ptr(df), ptr(dev(mass)), ptr(dev(fp)),
                                                         dtf, dtv, ptr(dev(typ)), ptr(dev(ilist)), ptr(dev(ip)), dim,
                                                         len(ilist))
        else:
            L.mdp_gpu_set_velocity_final_integrate_f64(ptr(dx), ptr(dv), ptr(df), ptr(dev(mass)), dtf, ptr(dev(typ)),
                                                       ptr(dev(ilist)), ptr(dev(ip)), dim, len(ilist))
        sync()
        assert np.array_equal(dx.cpu().numpy(), x) and np.array_equal(dv.cpu().numpy(), v), stage


# tdof values reaching every branch of the CSVR noise sum: nn = tdof - 1 of 0,
# 1, even below / above 12 (gamma deviate by product / by rejection), odd
@pytest.mark.parametrize("mode,tdof", [(0, None), (1, None), (2, 1.0), (2, 2.0), (2, 7.0), (2, 30.0), (2, 14.0),
                                       (2, None)])
def test_velocity_rescaling_thermostats(cuda_lib, mode, tdof):
    R, L = ref(), ours()
    rng, arrays, ilist = system(13)
    n = arrays["x"].shape[0]
    mass = np.array([0.0, 180.88, 92.9]); typ = rng.integers(1, 3, n).astype(np.int32)
    dt = 0.001
    dtarray = np.array([dt, 0.5 * dt / 1.0364269e-4, dt, 0.0, 100.0, 0.0])
    td = 3.0 * len(ilist) - 3.0 if tdof is None else tdof
    # t_start, t_stop, t_freq, t_target, t_current, tdof, boltz, drag, mvv2e, t_window, fraction
    tarray = np.array([300.0, 600.0, 10.0, 0.0, 0.0, td, 8.617343e-5, 0.0, 1.0364269e-4, 5.0, 0.7])
    v_ref = arrays["v"].copy()
    st_ref = dict(d=dtarray.copy(), t=tarray.copy(), seed=np.array([12345], np.int32), save=np.zeros(1, np.int32),
                  second=np.zeros(1))
    st = {k: a.copy() for k, a in st_ref.items()}
    dv, ke, tmp = dev(arrays["v"]), dev(np.zeros(n)), dev(np.zeros(4))
    dm, dty, dil = dev(mass), dev(typ), dev(ilist)
    e_ref = e = 0.0
    for step in range(6):
        st_ref["d"][5] = st["d"][5] = 10.0 * step
        e_ref = R.ref_velocity_rescaling(hp(v_ref), hp(mass), hp(st_ref["d"]), hp(st_ref["t"]), hp(st_ref["second"]),
                                         e_ref, hp(typ), hp(ilist), hp(st_ref["seed"]), hp(st_ref["save"]), 0, mode,
                                         3, len(ilist))
        e = L.mdp_gpu_velocity_rescaling_thermostat_f64(ptr(dv), ptr(dm), hp(st["d"]), hp(st["t"]), ptr(ke),
                                                        ptr(tmp), hp(st["second"]), e, ptr(dty), ptr(dil),
                                                        hp(st["seed"]), hp(st["save"]), 0, mode, 3, len(ilist))
        sync()
        assert abs(e - e_ref) <= 1e-12 * max(1.0, abs(e_ref)), (step, e, e_ref)
        assert rel(st["t"], st_ref["t"]) < 1e-12
        assert st["seed"][0] == st_ref["seed"][0] and st["save"][0] == st_ref["save"][0]
        assert abs(st["second"][0] - st_ref["second"][0]) < 1e-12
        assert rel(dv.cpu().numpy(), v_ref) < 1e-12, step


def test_float_entries_follow_the_double_path(cuda_lib):
    """The _f32 fixes of PREC_FLOAT builds: walls and set force in float
    against the double reference, within float rounding (the LJ 9-3 wall
    differences its 1/delta^10 and 1/delta^4 terms, which float resolves to
    about 1e-3 of the largest force)."""
    R, L32 = ref(), ours("f32")
    _, arrays, ilist = system(21, box=6.0)
    for kind, fp, ip in (("wall_lj93", WALL_PARAMS["wall_lj93"], [1]), ("set_force", [0.3, -1.2, 2.5], [1, 0, 1]),
                         ("wall_harmonic", WALL_PARAMS["wall_harmonic"], [4])):
        a = {k: v.copy() for k, v in arrays.items()}
        fpd = np.array(fp); ipd = np.array(ip, np.int32)
        R.ref_fix(FIX_KINDS[kind], hp(a["x"]), hp(a["v"]), hp(a["f"]), hp(a["eatom"]), hp(a["vatom"]), hp(fpd),
                  hp(ipd), hp(ilist), None, None, None, 0, 1, 1, 3, len(ilist))
        d = {k: dev(v, np.float32) for k, v in arrays.items()}
        getattr(L32, f"mdp_gpu_fix_{kind}_f32")(ptr(d["x"]), ptr(d["v"]), ptr(d["f"]), ptr(d["eatom"]),
                                                ptr(d["vatom"]), ptr(dev(fpd, np.float32)), ptr(dev(ipd)),
                                                ptr(dev(ilist)), 1, 1, 3, len(ilist))
        sync()
        tol = 2e-3 if kind == "wall_lj93" else 1e-5
        for k in ("f", "eatom", "vatom"):
            assert rel(d[k].cpu().numpy().astype(np.float64), a[k]) < tol, (kind, k)

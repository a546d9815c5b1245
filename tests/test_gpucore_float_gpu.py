"""GPU: the PREC_FLOAT (dstype = float) instantiations of the mdpcore.h
boundary.

* ComputePairSnap3's stage sequence through the reference's own wrappers in a
  float build of the driver (tests/cpp/gpucore_driver.cpp compiled with
  -DPREC_FLOAT, so mdpcore.h calls the gpu*<float> templates): per-atom
  energy, forces and virial against the golden double results of the
  reference's CPU build, within the error that rounding the inputs to float
  brings (positions to about 1e-7 relative).
* The MD-loop entry points in float: velocity Verlet bit-identical to a
  float32 restatement of the reference's update; ghosts and neighbour rows of
  the float path equal to the double path run on the same float positions;
  kinetic energy and column sums against float32 / float64 NumPy.
"""
import ctypes as C
import os

import numpy as np
import pytest

import julia_abi
from conftest import golden_params, load_golden
from test_gpucore_md import box_inputs, dev, ptr, sync
from test_gpucore_md import _release_tensors  # noqa: F401  (autouse fixture)
from oracle import refpy

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
DRIVER32 = os.path.join(HERE, "cpp", "_build", "libgpucore_driver_f32.so")
REF_LIB = os.path.join(os.path.dirname(HERE), "oracle", "_ref", "libcpuSnap_ref.so")
P = C.c_void_p

F = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
I = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")


def rel_inf(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


@pytest.mark.parametrize("name", ["bcc250_2j8", "bcc128_2j6", "bcc54_2j8_flags"])
def test_compute_pair_snap3_float_build(cuda_lib, name):
    if not os.path.exists(DRIVER32):
        pytest.fail("tests/cpp/_build/libgpucore_driver_f32.so missing (make -C tests/cpp REFROOT=<MDP tree>)")
    L = C.CDLL(DRIVER32)
    L.gpucore_pair_snap3.restype = C.c_int
    L.gpucore_pair_snap3.argtypes = ([F, F, F, F, I, I, I, I] + [C.c_int] * 3 + [F, C.c_int] +
                                     [F, C.c_int, F, C.c_int, I, C.c_int, I, I, C.c_int, I, I, C.c_int, I, C.c_int,
                                      F, F, C.c_int, I, F, F] + [C.c_float] * 4 + [C.c_int] * 6 + [C.c_char_p])
    g = load_golden(name)
    p = golden_params(g)
    t = julia_abi.tables(julia_abi.bind(REF_LIB), p.twojmax)
    f32 = lambda a: np.ascontiguousarray(a, dtype=np.float32).ravel()
    n, nm = g["neighlist"].shape
    anum = g["xall"].shape[0]
    jd = p.twojmax + 1
    e = np.zeros(n, np.float32); f = np.zeros(3 * n, np.float32); v = np.zeros(6 * n, np.float32)
    msg = C.create_string_buffer(512)
    rc = p.rcut
    code = L.gpucore_pair_snap3(
        e, f, v, f32(g["xall"]), np.ones(anum, np.int32), np.ascontiguousarray(g["alist"], np.int32),
        np.ascontiguousarray(g["neighlist"], np.int32).ravel(), np.ascontiguousarray(g["neighnum"], np.int32),
        n, anum, nm, f32([0.0, 0.0, 0.0, rc * rc]), 1, f32(t["rootpq"]), t["rootpq"].size, f32(t["cg"]), t["ncg"],
        t["idxz"], t["nz"], t["idxz_block"], t["idxb"], t["nb"], t["idxb_block"], t["idxu_block"], t["nu"],
        t["idxcg_block"], jd ** 3, f32([1.0 if p.bnormflag else j + 1.0 for j in range(jd)]), f32(p.coeff),
        p.coeff.size, np.zeros(2, np.int32), f32([0.0, p.radelem]), f32([0.0, p.wjelem]), p.rmin0, p.rfac0,
        p.rcutfac, 1.0, p.twojmax, p.switchflag, p.bzeroflag, p.bnormflag, p.wselfallflag, 2, msg)
    assert code == 0, msg.value
    de, dfo, dv = (rel_inf(e.astype(np.float64), g["eatom"]), rel_inf(f.reshape(n, 3).astype(np.float64), g["fatom"]),
                   rel_inf(v.reshape(6, n).astype(np.float64), g["vatom"]))
    print(f"{name} float build vs double reference: energy {de:.1e}, forces {dfo:.1e}, virial {dv:.1e}")
    assert de < 1e-6 and dfo < 1e-4 and dv < 1e-4


def lib():
    from mdp_b200 import _lib
    L = _lib.lib()
    L.mdp_gpu_atom_list3d_f32.argtypes = [P] * 10 + [C.c_int] * 3
    L.mdp_gpu_atom_list3d_f64.argtypes = [P] * 10 + [C.c_int] * 3
    L.mdp_gpu_full_neighbor_list3d_f32.argtypes = [P] * 4 + [C.c_int] * 4
    L.mdp_gpu_full_neighbor_list3d_f64.argtypes = [P] * 4 + [C.c_int] * 4
    L.mdp_gpu_array_get_value_at_index_int.argtypes = [P, C.c_int]
    L.mdp_gpu_array_get_value_at_index_int.restype = C.c_int
    for fn in (L.mdp_gpu_initial_integrate_f32, L.mdp_gpu_final_integrate_f32):
        fn.argtypes = [P] * 12 + [C.c_float, P, P] + [C.c_int] * 7
    L.mdp_gpu_compute_ke_atom_f32.argtypes = [P, P, P, C.c_float, P, P, C.c_int, C.c_int]
    L.mdp_gpu_array_sum_every_column_f32.argtypes = [P, P, C.c_int, C.c_int]
    return L


def test_float_ghosts_and_neighbors_equal_double_path(cuda_lib):
    L = lib()
    g = load_golden("bcc250_2j8")
    p = golden_params(g)
    x0 = np.ascontiguousarray(g["x"], dtype=np.float32).astype(np.float64)   # the float positions, exactly
    inum = x0.shape[0]
    rc = p.rcut + float(g["skin"])
    nm = int(g["neighmax"])
    bs, _, _ = box_inputs(g["box"], rc)
    pnum = int(bs["pnum"])
    cap = inum * 8 + 4096
    out = {}
    for prec, dt in (("f64", np.float64), ("f32", np.float32)):
        x = np.zeros((cap, 3), dt); x[:inum] = x0
        dx = dev(x)
        alist = dev(np.zeros(cap, np.int32)); inside = dev(np.zeros(inum * pnum, np.int32))
        gsum = dev(np.zeros(inum + 1, np.int32)); gnum = dev(np.zeros(inum + 1, np.int32))
        sums = dev(np.zeros(inum + 8, np.int32))
        getattr(L, f"mdp_gpu_atom_list3d_{prec}")(ptr(alist), ptr(inside), ptr(gsum), ptr(gnum), ptr(sums), ptr(sums),
                                                  ptr(dx), ptr(dev(bs["pimages"], dt)), ptr(dev(bs["rbvertices"], dt)),
                                                  ptr(dev(bs["s2rmap"], dt)), inum, pnum, 3)
        anum = inum + L.mdp_gpu_array_get_value_at_index_int(ptr(gsum), inum)
        nl = dev(np.full(inum * nm, -1, np.int32)); nn = dev(np.zeros(inum, np.int32))
        getattr(L, f"mdp_gpu_full_neighbor_list3d_{prec}")(ptr(nl), ptr(nn), ptr(dx), ptr(dev([rc * rc], dt)), anum,
                                                           inum, nm, 3)
        sync()
        out[prec] = (dx.cpu().numpy()[:anum].astype(np.float64), alist.cpu().numpy()[:anum], nn.cpu().numpy(),
                     nl.cpu().numpy().reshape(inum, nm))
    (x64, a64, n64, l64), (x32, a32, n32, l32) = out["f64"], out["f32"]
    assert np.array_equal(a32, a64)
    assert np.abs(x32 - x64).max() < 1e-5
    assert np.array_equal(n32, n64)
    for i in range(inum):
        assert np.array_equal(l32[i, : n32[i]], l64[i, : n64[i]])


def test_float_verlet_ke_and_column_sums(cuda_lib):
    L = lib()
    rng = np.random.default_rng(5)
    n, dim = 3000, 3
    x = rng.normal(size=(n, dim)).astype(np.float32)
    v = (rng.normal(size=(n, dim)) * 3).astype(np.float32)
    f = (rng.normal(size=(n, dim)) * 40).astype(np.float32)
    mass = np.array([0.0, 180.88, 92.9], np.float32)
    typ = rng.integers(1, 3, n).astype(np.int32)
    ilist = rng.permutation(n).astype(np.int32)[: n - 50]
    dtarray = np.array([0.0, 0.5 * 0.001 / 1.0364269e-4, 0.001], np.float32)
    dx, dv, df, dm, dt, di = dev(x), dev(v), dev(f), dev(mass), dev(typ), dev(ilist)
    z = dev(np.zeros(4, np.float32))
    args = [ptr(dx), ptr(dv), ptr(df), ptr(dm), dtarray.ctypes.data_as(C.c_void_p)] + [ptr(z)] * 7 + \
        [4.0, ptr(dt), ptr(di), 0, 0, 1, 1, 0, dim, len(ilist)]
    L.mdp_gpu_initial_integrate_f32(*args)
    sync()
    xw, vw = x.copy(), v.copy()
    for i in ilist:     # cpuVelocityIntegration.cpp:307-339 in float
        dtfm = np.float32(dtarray[1] / mass[typ[i]])
        vw[i] = vw[i] + dtfm * f[i]
        xw[i] = xw[i] + dtarray[2] * vw[i]
    assert np.array_equal(dv.cpu().numpy(), vw) and np.array_equal(dx.cpu().numpy(), xw)
    ke = dev(np.zeros(len(ilist), np.float32))
    L.mdp_gpu_compute_ke_atom_f32(ptr(ke), ptr(dm), ptr(dv), np.float32(1.0364269e-4), ptr(dt), ptr(di), dim,
                                  len(ilist))
    sync()
    want = np.float32(0.5) * np.float32(1.0364269e-4) * mass[typ[ilist]] * (vw[ilist] ** 2).sum(axis=1)
    assert np.abs(ke.cpu().numpy() - want).max() <= 1e-6 * np.abs(want).max()
    a = rng.normal(size=(7, 5000)).astype(np.float32)
    b = dev(np.zeros(7, np.float32))
    L.mdp_gpu_array_sum_every_column_f32(ptr(b), ptr(dev(a)), 7, 5000)
    sync()
    assert np.abs(b.cpu().numpy() - a.astype(np.float64).sum(axis=1)).max() < 1e-3

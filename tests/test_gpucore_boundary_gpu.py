"""GPU: the mdpcore.h boundary (MDP's C++ backend dispatch, backend == 2).

tests/cpp/gpucore_driver.cpp is compiled against the reference's own
mdpcommon.h, mdpgpucore.h and mdpcore.h with this library's
include/mdp_b200_gpucore.h templates in between, and linked to
libmdp_b200.so.  It runs ComputePairSnap3's stage sequence
(src/C++/Descriptors/snappotential.cpp:634-760) through the reference's inline
wrappers -- NeighborPairList, Cumsum, IntArrayGetValueAtIndex, NeighborPairs,
SnapComputeUi, AddWself2Ui, SnapComputeEi, SnapComputeYi, SnapComputeFi -- on
device arrays, in one block and in three atom blocks (ilist offsets, per-block
atom types).  Per-atom energy, forces and the SoA virial vatom[6][inum] are
compared with the golden ComputePairSnap3 results of the reference's CPU build.
"""
import ctypes as C
import os

import numpy as np
import pytest

import julia_abi
from conftest import golden_params, load_golden

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
DRIVER = os.path.join(HERE, "cpp", "_build", "libgpucore_driver.so")
REF_LIB = os.path.join(os.path.dirname(HERE), "oracle", "_ref", "libcpuSnap_ref.so")
TOL = 1e-10

D = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
I = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")


def rel_inf(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


@pytest.fixture(scope="module")
def driver(cuda_lib):
    if not os.path.exists(DRIVER):
        pytest.fail("tests/cpp/_build/libgpucore_driver.so missing (make -C tests/cpp REFROOT=<MDP tree>)")
    L = C.CDLL(DRIVER)
    L.gpucore_pair_snap3.restype = C.c_int
    L.gpucore_pair_snap3.argtypes = ([D, D, D, D, I, I, I, I] + [C.c_int] * 3 + [D, C.c_int] +
                                     [D, C.c_int, D, C.c_int, I, C.c_int, I, I, C.c_int, I, I, C.c_int, I, C.c_int,
                                      D, D, C.c_int, I, D, D] + [C.c_double] * 4 + [C.c_int] * 6 + [C.c_char_p])
    L.gpucore_pair_snap3_elements.restype = C.c_int
    L.gpucore_pair_snap3_elements.argtypes = L.gpucore_pair_snap3.argtypes[:-1] + [C.c_int, C.c_char_p]
    return L


@pytest.mark.parametrize("name", ["bcc250_2j8", "bcc128_2j6", "bcc54_2j8_flags", "bcc128_2j4"])
@pytest.mark.parametrize("nblocks", [1, 3])
def test_compute_pair_snap3_through_mdpcore_wrappers(driver, name, nblocks):
    if not os.path.exists(REF_LIB):
        pytest.fail("oracle/_ref/libcpuSnap_ref.so missing (build with make -C oracle ref)")
    g = load_golden(name)
    p = golden_params(g)
    t = julia_abi.tables(julia_abi.bind(REF_LIB), p.twojmax)   # cpuInitSna of the reference library
    xall = np.ascontiguousarray(g["xall"], dtype=np.float64)
    n, nm = g["neighlist"].shape
    anum = xall.shape[0]
    jd = p.twojmax + 1
    bzero = np.array([1.0 if p.bnormflag else j + 1.0 for j in range(jd)])   # InitSnap's bzero (www = 1)
    rc = p.rcut
    e = np.zeros(n); f = np.zeros(3 * n); v = np.zeros(6 * n)
    msg = C.create_string_buffer(512)
    rcode = driver.gpucore_pair_snap3(
        e, f, v, xall.ravel(), np.ones(anum, dtype=np.int32), np.ascontiguousarray(g["alist"], dtype=np.int32),
        np.ascontiguousarray(g["neighlist"], dtype=np.int32).ravel(), np.ascontiguousarray(g["neighnum"], np.int32),
        n, anum, nm, np.array([0.0, 0.0, 0.0, rc * rc]), 1,
        t["rootpq"], t["rootpq"].size, t["cg"], t["ncg"], t["idxz"], t["nz"], t["idxz_block"], t["idxb"], t["nb"],
        t["idxb_block"], t["idxu_block"], t["nu"], t["idxcg_block"], jd ** 3, bzero,
        np.ascontiguousarray(p.coeff, dtype=np.float64), p.coeff.size, np.zeros(2, dtype=np.int32),
        np.array([0.0, p.radelem]), np.array([0.0, p.wjelem]), p.rmin0, p.rfac0, p.rcutfac, 1.0, p.twojmax,
        p.switchflag, p.bzeroflag, p.bnormflag, p.wselfallflag, nblocks, msg)
    assert rcode == 0, msg.value
    assert rel_inf(e, g["eatom"]) < TOL
    assert rel_inf(f.reshape(n, 3), g["fatom"]) < TOL
    assert rel_inf(v.reshape(6, n), g["vatom"]) < TOL


CHEM = ["chem_bcc128_2j6", "chem_bcc250_2j8", "chem_bcc54_2j4_3el_flags", "chem_bcc54_2j6_wselfall",
        "chem_bcc128_2j8_chemflag0"]


@pytest.mark.parametrize("name", CHEM)
def test_compute_pair_snap3_several_elements(driver, name):
    """ComputePairSnap3 with InitSnap's multi-element set-up through the same
    wrappers: typed pair list with type-pair cutoffs, U / Y element blocks
    (chemflag), per-atom coefficient sets map[type]; against the reference's
    CPU chain (the tests/golden/chem_*.npz fixtures).  One atom block: with
    several blocks the reference's SnapComputeEi reads the types of the first
    block's atoms (it is passed atomtype without the block offset)."""
    from mdp_b200 import configs
    if not os.path.exists(REF_LIB):
        pytest.fail("oracle/_ref/libcpuSnap_ref.so missing (build with make -C oracle ref)")
    g = load_golden(name)
    bnorm, bzero_f, switch, wsa = (int(v) for v in g["flags"])
    p = configs.snap_params_elements(int(g["twojmax"]), g["radelems"], g["wjelems"], chemflag=int(g["chemflag"]),
                                     seed=int(g["coeff_seed"]), bnormflag=bnorm, bzeroflag=bzero_f,
                                     switchflag=switch, wselfallflag=wsa)
    t = julia_abi.tables(julia_abi.bind(REF_LIB), p.twojmax)
    xall = np.ascontiguousarray(g["xall"], dtype=np.float64)
    n, nm = g["neighlist"].shape
    anum = xall.shape[0]
    jd = p.twojmax + 1
    ne = p.nelements
    bzero = np.array([1.0 if p.bnormflag else j + 1.0 for j in range(jd)])
    rcutsq = np.zeros((ne + 1) ** 2)
    for a in range(ne):
        for b in range(ne):
            rcutsq[b + 1 + (a + 1) * (ne + 1)] = ((p.radelems[a] + p.radelems[b]) * p.rcutfac) ** 2
    alist = np.ascontiguousarray(g["alist"], dtype=np.int32)
    atype = np.ascontiguousarray(g["types"][alist], dtype=np.int32)
    e = np.zeros(n); f = np.zeros(3 * n); v = np.zeros(6 * n)
    msg = C.create_string_buffer(512)
    rcode = driver.gpucore_pair_snap3_elements(
        e, f, v, xall.ravel(), atype, alist, np.ascontiguousarray(g["neighlist"], dtype=np.int32).ravel(),
        np.ascontiguousarray(g["neighnum"], np.int32), n, anum, nm, rcutsq, ne,
        t["rootpq"], t["rootpq"].size, t["cg"], t["ncg"], t["idxz"], t["nz"], t["idxz_block"], t["idxb"], t["nb"],
        t["idxb_block"], t["idxu_block"], t["nu"], t["idxcg_block"], jd ** 3, bzero,
        np.ascontiguousarray(p.coeff, dtype=np.float64), p.ncoeffall,
        np.concatenate([[0], np.arange(ne)]).astype(np.int32), np.concatenate([[0.0], p.radelems]),
        np.concatenate([[0.0], p.wjelems]), p.rmin0, p.rfac0, p.rcutfac, 1.0, p.twojmax,
        p.switchflag, p.bzeroflag, p.bnormflag, p.wselfallflag, 1, p.chemflag, msg)
    assert rcode == 0, msg.value
    assert rel_inf(e, g["eatom"]) < TOL
    assert rel_inf(f.reshape(n, 3), g["fatom"]) < TOL
    assert rel_inf(v.reshape(6, n), g["vatom"]) < TOL

"""Test infrastructure: ctypes bindings to the reference's own CPU code.

`oracle/_ref/libmdp_ref_harness.so` is MDP's C++ core (src/C++/Core/cpuCore.cpp)
compiled from the reference tree behind `oracle/ref_harness.cpp`;
`oracle/_ref/libcpuSnap_ref.so` is MDP's Julia C-ABI SNAP library
(src/Julia/Potential/cpuSnap.cpp).  Both are built by `make -C oracle ref`.
Only tests, golden-fixture generation, smoke() and bench.py's CPU baseline use
this module; the product path never does.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")

_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_ip = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")


def available() -> bool:
    return os.path.exists(os.path.join(REF_DIR, "libmdp_ref_harness.so"))


_lib = None


def lib():
    global _lib
    if _lib is None:
        _lib = C.CDLL(os.path.join(REF_DIR, "libmdp_ref_harness.so"))
        _lib.ref_box_setup.restype = C.c_int
        _lib.ref_box_setup.argtypes = [_dp, _dp, _dp, _dp, _ip, _dp, _dp, _dp, _ip, _dp, _dp, _dp]
        _lib.ref_neighbor_list.restype = C.c_long
        _lib.ref_neighbor_list.argtypes = [_dp, _ip, _ip, _ip, _dp, _dp, _dp, _ip, _dp, _dp, _dp,
                                           C.c_double, C.c_int, C.c_int, C.c_int, C.c_int, C.c_long]
        _lib.ref_snap_force.restype = None
        _lib.ref_snap_force.argtypes = [_dp, _dp, _dp, _dp, _ip, _ip, _ip, _ip, C.c_int, C.c_int,
                                        C.c_int, C.c_int, _dp, C.c_double, C.c_double, C.c_double,
                                        C.c_double, C.c_double, C.c_int, C.c_int, C.c_int, C.c_int,
                                        C.c_int, C.c_int]
        _lib.ref_snap_descriptors.argtypes = [_dp, _dp, _dp, _dp, _dp, _ip, _ip, _ip, _ip, C.c_int, C.c_int,
                                              C.c_int, C.c_double, C.c_double, C.c_double, C.c_double,
                                              C.c_double, C.c_int, C.c_int, C.c_int, C.c_int]
        _lib.ref_snap_descriptors.restype = None
        _lib.ref_snap_force_pairsnap.restype = None
        _lib.ref_snap_force_pairsnap.argtypes = [_dp, _dp, _dp, _dp, _ip, _ip, _ip, _ip, C.c_int, C.c_int,
                                                 C.c_int, C.c_int, _dp, C.c_double, C.c_double, C.c_double,
                                                 C.c_double, C.c_double, C.c_int, C.c_int, C.c_int, C.c_int,
                                                 C.c_int]
        _lib.ref_snap_force_me.restype = None
        _lib.ref_snap_force_me.argtypes = [_dp, _dp, _dp, _dp, _ip, _ip, _ip, _ip, C.c_int, C.c_int, C.c_int,
                                           C.c_int, C.c_int, C.c_int, _dp, C.c_double, C.c_double, C.c_double,
                                           _dp, _dp, C.c_int, C.c_int, C.c_int, C.c_int]
        _lib.ref_nve_initial.argtypes = [_dp, _dp, _dp, _dp, C.c_double, C.c_double, _ip, _ip, C.c_int]
        _lib.ref_nve_final.argtypes = [_dp, _dp, _dp, _dp, C.c_double, _ip, _ip, C.c_int]
        _lib.ref_omp_max_threads.restype = C.c_int
    return _lib


def box_setup(box, rcut_skin):
    B = np.asarray(box, dtype=np.float64)
    if B.shape == (3,):
        B = np.diag(B)
    a, b, c = (np.ascontiguousarray(B[k]) for k in range(3))   # cell vectors as rows
    off = np.full(3, float(rcut_skin))
    pbc = np.ones(3, dtype=np.int32)
    s2r = np.zeros(9); rbv = np.zeros(24); pim = np.zeros(81)
    cellnum = np.zeros(3, dtype=np.int32)
    eta1 = np.zeros(4096); eta2 = np.zeros(4096); eta3 = np.zeros(4096)
    pnum = lib().ref_box_setup(a, b, c, off, pbc, s2r, rbv, pim, cellnum, eta1, eta2, eta3)
    return dict(s2rmap=s2r, rbvertices=rbv, pimages=pim, pnum=pnum, cellnum=cellnum,
                eta1=eta1, eta2=eta2, eta3=eta3)


def neighbor_list(x_local, box, rcut, skin, neighmax=64, neighcell=1):
    """Ghost atoms + full neighbour list exactly as MDP builds them.
    Returns (x_all (anum,3), alist (anum,), neighlist (inum,neighmax), neighnum (inum,))."""
    inum = x_local.shape[0]
    bs = box_setup(box, rcut + skin)
    anummax = inum * 8 + 4096
    x = np.zeros(anummax * 3)
    x[: 3 * inum] = x_local.ravel()
    alist = np.zeros(anummax, dtype=np.int32)
    nl = np.zeros(inum * neighmax, dtype=np.int32)
    nn = np.zeros(inum, dtype=np.int32)
    gnum = lib().ref_neighbor_list(x, alist, nl, nn, bs["pimages"], bs["rbvertices"], bs["s2rmap"],
                                   bs["cellnum"], bs["eta1"], bs["eta2"], bs["eta3"],
                                   (rcut + skin) ** 2, inum, bs["pnum"], neighmax, neighcell, anummax)
    if gnum < 0:
        raise RuntimeError("ghost capacity exceeded")
    anum = inum + int(gnum)
    return x[: 3 * anum].reshape(anum, 3).copy(), alist[:anum].copy(), nl.reshape(inum, neighmax), nn


def snap_force(x_all, alist, neighlist, neighnum, params, nblocks=1, nthreads=1):
    """Per-atom energy, forces (N,3) and virial (6,N SoA) from the reference's
    ComputePairSnap3 chain (cpuSnap4.cpp)."""
    inum, neighmax = neighlist.shape
    e = np.zeros(inum); f = np.zeros(3 * inum); v = np.zeros(6 * inum)
    atype = np.ones(x_all.shape[0], dtype=np.int32)
    lib().ref_snap_force(e, f, v, np.ascontiguousarray(x_all).ravel(), atype,
                         np.ascontiguousarray(alist, dtype=np.int32),
                         np.ascontiguousarray(neighlist, dtype=np.int32).ravel(),
                         np.ascontiguousarray(neighnum, dtype=np.int32),
                         inum, neighmax, params.twojmax, params.ncoeffall,
                         np.ascontiguousarray(params.coeff, dtype=np.float64),
                         params.rcutfac, params.rfac0, params.rmin0, params.radelem, params.wjelem,
                         params.switchflag, params.bzeroflag, params.bnormflag, params.wselfallflag,
                         nblocks, nthreads)
    return e, f.reshape(inum, 3), v.reshape(6, inum)


def snap_force_pairsnap(x_all, alist, neighlist, neighnum, params):
    """Per-atom energy, forces (N,3) and virial (6,N) from the reference's
    ComputePairSnap chain (snappotential.cpp:236-410), the one that evaluates
    the quadratic SNAP terms (quadraticflag)."""
    inum, neighmax = neighlist.shape
    e = np.zeros(inum); f = np.zeros(3 * inum); v = np.zeros(6 * inum)
    atype = np.ones(x_all.shape[0], dtype=np.int32)
    lib().ref_snap_force_pairsnap(e, f, v, np.ascontiguousarray(x_all).ravel(), atype,
                                  np.ascontiguousarray(alist, dtype=np.int32),
                                  np.ascontiguousarray(neighlist, dtype=np.int32).ravel(),
                                  np.ascontiguousarray(neighnum, dtype=np.int32),
                                  inum, neighmax, params.twojmax, params.ncoeffall,
                                  np.ascontiguousarray(params.coeff, dtype=np.float64),
                                  params.rcutfac, params.rfac0, params.rmin0, params.radelem, params.wjelem,
                                  params.switchflag, params.bzeroflag, params.bnormflag, params.wselfallflag,
                                  params.quadraticflag)
    return e, f.reshape(inum, 3), v.reshape(6, inum)


def snap_force_me(x_all, alist, neighlist, neighnum, atomtype, params):
    """Per-atom energy, forces (N,3) and virial (6,N) of a multi-element model
    (types 1..nelements in atomtype, one per local atom) from the reference's
    ComputePairSnap3 chain with InitSnap's per-element set-up."""
    inum, neighmax = neighlist.shape
    e = np.zeros(inum); f = np.zeros(3 * inum); v = np.zeros(6 * inum)
    lib().ref_snap_force_me(e, f, v, np.ascontiguousarray(x_all).ravel(),
                            np.ascontiguousarray(atomtype, dtype=np.int32),
                            np.ascontiguousarray(alist, dtype=np.int32),
                            np.ascontiguousarray(neighlist, dtype=np.int32).ravel(),
                            np.ascontiguousarray(neighnum, dtype=np.int32), inum, neighmax, params.twojmax,
                            params.nelements, params.chemflag, params.ncoeffall,
                            np.ascontiguousarray(params.coeff, dtype=np.float64),
                            params.rcutfac, params.rfac0, params.rmin0,
                            np.ascontiguousarray(params.radelems, dtype=np.float64),
                            np.ascontiguousarray(params.wjelems, dtype=np.float64),
                            params.switchflag, params.bzeroflag, params.bnormflag, params.wselfallflag)
    return e, f.reshape(inum, 3), v.reshape(6, inum)


def snap_descriptors(x_all, alist, neighlist, neighnum, params):
    """Per-configuration descriptors from the reference's ComputeSnap chain
    (snappotential.cpp:762-910, cpuSnap2.cpp): bi (ncoeff,), bd (ncoeff, inum, 3)
    with bd[k, i, c] = d(sum_a B_ak)/dx_ic, bv (ncoeff, 6) and per-atom B (ncoeff, inum)."""
    inum, neighmax = neighlist.shape
    nc = params.ncoeff
    bi = np.zeros(nc); bd = np.zeros(3 * inum * nc); bv = np.zeros(6 * nc); bl = np.zeros(inum * nc)
    atype = np.ones(x_all.shape[0], dtype=np.int32)
    lib().ref_snap_descriptors(bi, bd, bv, bl, np.ascontiguousarray(x_all).ravel(), atype,
                               np.ascontiguousarray(alist, dtype=np.int32),
                               np.ascontiguousarray(neighlist, dtype=np.int32).ravel(),
                               np.ascontiguousarray(neighnum, dtype=np.int32), inum, neighmax, params.twojmax,
                               params.rcutfac, params.rfac0, params.rmin0, params.radelem, params.wjelem,
                               params.switchflag, params.bzeroflag, params.bnormflag, params.wselfallflag)
    return bi, bd.reshape(nc, inum, 3), bv.reshape(nc, 6), bl.reshape(nc, inum)

"""Test infrastructure: ctypes bindings to the project's C restatement
(`oracle/snap_oracle.c` -> `oracle/libsnap_oracle.so`, built by `make -C oracle`).

Used only as the checker by tests, smoke() and bench.py's CPU-baseline leg.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "libsnap_oracle.so")

_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_ip = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_lib = None


def build():
    subprocess.check_call(["make", "-s", "-C", HERE, "all"])


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        _lib = C.CDLL(LIB)
        _lib.orc_table_sizes.argtypes = [C.c_int, _ip]
        _lib.orc_tables_copy.argtypes = [C.c_int, _dp, _dp, _ip, _ip, _ip]
        _lib.orc_neighbor_list.restype = C.c_long
        _lib.orc_neighbor_list.argtypes = [_dp, _ip, _ip, _ip, _dp, _dp, _dp, C.c_double, C.c_int,
                                           C.c_int, C.c_long]
        _lib.orc_snap_force.argtypes = [_dp, _dp, _dp, _dp, _ip, _ip, _ip, C.c_int, C.c_int, C.c_int,
                                        _dp, C.c_double, C.c_double, C.c_double, C.c_double,
                                        C.c_double, C.c_int, C.c_int, C.c_int,
                                        C.c_void_p, C.c_void_p, C.c_void_p]
        _lib.orc_nve_initial.argtypes = [_dp, _dp, _dp, C.c_double, C.c_double, C.c_int]
        _lib.orc_nve_final.argtypes = [_dp, _dp, C.c_double, C.c_int]
    return _lib


def table_sizes(twojmax):
    out = np.zeros(4, dtype=np.int32)
    lib().orc_table_sizes(twojmax, out)
    return dict(idxcg=int(out[0]), idxu=int(out[1]), idxb=int(out[2]), idxz=int(out[3]))


def tables(twojmax):
    s = table_sizes(twojmax)
    cg = np.zeros(s["idxcg"]); rootpq = np.zeros((twojmax + 2) ** 2)
    idxz = np.zeros(10 * s["idxz"], dtype=np.int32); idxb = np.zeros(3 * s["idxb"], dtype=np.int32)
    idxu_block = np.zeros(twojmax + 1, dtype=np.int32)
    lib().orc_tables_copy(twojmax, cg, rootpq, idxz, idxb, idxu_block)
    return dict(cg=cg, rootpq=rootpq, idxz=idxz.reshape(-1, 10), idxb=idxb.reshape(-1, 3),
                idxu_block=idxu_block, n_cg=s["idxcg"], n_u=s["idxu"], n_b=s["idxb"], n_z=s["idxz"])


def neighbor_list(x_local, box, rcut, skin, neighmax=64):
    inum = x_local.shape[0]
    anummax = inum * 8 + 4096
    x = np.zeros(anummax * 3)
    x[: 3 * inum] = np.ascontiguousarray(x_local).ravel()
    alist = np.zeros(anummax, dtype=np.int32)
    nl = np.zeros(inum * neighmax, dtype=np.int32)
    nn = np.zeros(inum, dtype=np.int32)
    B = np.asarray(box, dtype=np.float64)
    if B.shape == (3,):
        B = np.diag(B)
    a, b, c = (np.ascontiguousarray(B[k]) for k in range(3))   # cell vectors as rows
    anum = lib().orc_neighbor_list(x, alist, nl, nn, a, b, c, rcut + skin, inum, neighmax, anummax)
    if anum == -1:
        raise RuntimeError("ghost capacity exceeded")
    if anum == -2:
        raise RuntimeError("neighbour list truncated at neighmax")
    return x[: 3 * anum].reshape(anum, 3).copy(), alist[:anum].copy(), nl.reshape(inum, neighmax), nn


def snap_force(x_all, alist, neighlist, neighnum, params, want_uy=False):
    """Returns eatom (N,), fatom (N,3), vatom (6,N) [, U (N,2,idxu), Y (N,2,idxu), B (N,ncoeff)]."""
    inum, neighmax = neighlist.shape
    s = table_sizes(params.twojmax)
    e = np.zeros(inum); f = np.zeros(3 * inum); v = np.zeros(6 * inum)
    U = Y = B = None
    ptr = [None, None, None]
    if want_uy:
        U = np.zeros((inum, 2, s["idxu"])); Y = np.zeros((inum, 2, s["idxu"])); B = np.zeros((inum, s["idxb"]))
        ptr = [U.ctypes.data, Y.ctypes.data, B.ctypes.data]
    lib().orc_snap_force(e, f, v, np.ascontiguousarray(x_all).ravel(),
                         np.ascontiguousarray(alist, dtype=np.int32),
                         np.ascontiguousarray(neighlist, dtype=np.int32).ravel(),
                         np.ascontiguousarray(neighnum, dtype=np.int32), inum, neighmax,
                         params.twojmax, np.ascontiguousarray(params.coeff, dtype=np.float64),
                         params.rcutfac, params.rfac0, params.rmin0, params.radelem, params.wjelem,
                         params.switchflag, params.bzeroflag, params.bnormflag, *ptr)
    out = (e, f.reshape(inum, 3), v.reshape(6, inum))
    if want_uy:
        out = out + (U, Y, B)
    return out

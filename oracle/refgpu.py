"""Baseline infrastructure: MDP's own GPU SNAP kernels (src/C++/Core/gpuSnap4.cu,
compiled unchanged for sm_100a into oracle/_ref/libmdp_ref_gpusnap.so by
`make -C oracle ref`) timed on this GPU, as a speed bar for the repository's
kernels.  They are never the oracle (their dE/dr drops the switching
derivative, gpuSnap4.cu:1116).  Only bench.py's baseline leg uses this.

The reference launchers index with 32-bit ints; ref_gpu_snap_check refuses a
size at which any of their index products would overflow before anything is
launched (at 2J=8, idxz_max * inum alone limits a run to about 900,000 atoms).
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_ref", "libmdp_ref_gpusnap.so")
SNAP_LIB = os.path.join(HERE, "_ref", "libcpuSnap_ref.so")


def available() -> bool:
    return os.path.exists(LIB) and os.path.exists(SNAP_LIB)


def _tables(tj):
    """Index tables, rootpq and CG list in the reference's layouts (its own cpuInitSna)."""
    D = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
    I = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
    L = C.CDLL(SNAP_LIB)
    L.cpuInitSna.argtypes = [D, D, D, I, I, I, I, I, I, I, C.c_int]
    for f in ("idxbcount", "idxcgcount", "idxucount", "idxzcount"):
        getattr(L, f).argtypes = [C.c_int]
    nb, ncg, nu, nz = L.idxbcount(tj), L.idxcgcount(tj), L.idxucount(tj), L.idxzcount(tj)
    jd = tj + 1
    t = dict(rootpq=np.zeros((jd + 1) ** 2), cg=np.zeros(ncg), fac=np.ones(168), idx_max=np.zeros(5, np.int32),
             idxz=np.zeros(10 * nz, np.int32), idxz_block=np.zeros(jd ** 3, np.int32),
             idxb=np.zeros(3 * nb, np.int32), idxb_block=np.zeros(jd ** 3, np.int32),
             idxu_block=np.zeros(jd, np.int32), idxcg_block=np.zeros(jd ** 3, np.int32))
    for k in range(1, 168):
        t["fac"][k] = t["fac"][k - 1] * k
    L.cpuInitSna(t["rootpq"], t["cg"], t["fac"], t["idx_max"], t["idxz"], t["idxz_block"], t["idxb"],
                 t["idxb_block"], t["idxu_block"], t["idxcg_block"], tj)
    t.update(nb=nb, nu=nu, nz=nz)
    return t


def pairs_of(xall, alist, neighlist, neighnum, rcut):
    """ComputePairSnap3's pair arrays (NeighborPairList + NeighborPairs,
    cpuSnap.cpp:1883-1933) for one atom block holding every atom: pairs with
    1e-20 < r^2 < rcut^2 in row order; rij = x_j - x_i, ai = aii = i, aj = owner."""
    n, nm = neighlist.shape
    cols = np.arange(nm)[None, :]
    valid = cols < neighnum[:, None]
    j = np.where(valid, neighlist, 0)
    d = xall[j] - xall[:n][:, None, :]
    r2 = (d * d).sum(-1)
    keep = valid & (r2 < rcut * rcut) & (r2 > 1e-20)
    ii, kk = np.nonzero(keep)
    rij = np.ascontiguousarray(d[ii, kk])
    return rij, ii.astype(np.int32), alist[j[ii, kk]].astype(np.int32)


def stage_times(params, x, box, skin=1.0, neighmax=64, repeats=3, device=0):
    """Median milliseconds of the reference's Ui(+wself), Ei, Yi and Fi GPU
    stages on the configuration, and its pair count; None when the size does
    not fit the reference's 32-bit indexing."""
    import torch
    from oracle import refpy
    tj = params.twojmax
    t = _tables(tj)
    xa, al, nl, nn = refpy.neighbor_list(x, box, params.rcut, skin, neighmax, neighcell=1)
    rij, ai, aj = pairs_of(xa, al, nl, nn, params.rcut)
    n, ij = x.shape[0], rij.shape[0]
    L = C.CDLL(LIB)
    L.ref_gpu_snap_check.argtypes = [C.c_int] * 6
    if L.ref_gpu_snap_check(tj, t["nu"], t["nb"], t["nz"], n, ij) != 0:
        return None
    dev = torch.device("cuda", device)
    f64 = lambda a: torch.tensor(np.ascontiguousarray(a, dtype=np.float64).ravel(), device=dev)
    i32 = lambda a: torch.tensor(np.ascontiguousarray(a, dtype=np.int32).ravel(), device=dev)
    z = lambda k: torch.zeros(k, dtype=torch.float64, device=dev)
    bufs = dict(Ur=z(t["nu"] * n), Ui=z(t["nu"] * n), Yr=z(t["nu"] * n), Yi=z(t["nu"] * n), e=z(n), f=z(3 * n),
                v=z(6 * n), rootpq=f64(t["rootpq"]), rij=f64(rij), wj=f64([0.0, params.wjelem]),
                rad=f64([0.0, params.radelem]), cg=f64(t["cg"]),
                bzero=f64([1.0 if params.bnormflag else j + 1.0 for j in range(tj + 1)]), coeff=f64(params.coeff),
                idxu_block=i32(t["idxu_block"]), idxz=i32(t["idxz"]), idxb=i32(t["idxb"]),
                idxb_block=i32(t["idxb_block"]), idxcg_block=i32(t["idxcg_block"]), map=i32([0, 0]),
                type=i32(np.ones(n)), ilist=i32(np.arange(n)), ai=i32(ai), aj=i32(aj), ti=i32(np.ones(ij)))
    P = C.c_void_p
    L.ref_gpu_snap_stages.argtypes = [P] * 27 + [C.c_double] * 3 + [C.c_int] * 11 + [P]
    L.ref_gpu_snap_stages.restype = C.c_int
    b = bufs
    args = [b["Ur"], b["Ui"], b["Yr"], b["Yi"], b["e"], b["f"], b["v"], b["rootpq"], b["rij"], b["wj"], b["rad"],
            b["cg"], b["bzero"], b["coeff"], b["idxu_block"], b["idxz"], b["idxb"], b["idxb_block"],
            b["idxcg_block"], b["map"], b["type"], b["ilist"], b["ai"], b["ai"], b["aj"], b["ti"], b["ti"]]
    ms = (C.c_float * 4)()
    runs = []
    torch.cuda.synchronize()
    for _ in range(repeats + 1):
        rc = L.ref_gpu_snap_stages(*[a.data_ptr() for a in args], params.rmin0, params.rfac0, params.rcutfac, tj,
                                   t["nu"], t["nb"], t["nz"], params.ncoeffall, params.bnormflag, params.bzeroflag,
                                   params.switchflag, params.wselfallflag, n, ij, ms)
        if rc != 0:
            raise RuntimeError(f"reference GPU stages returned {rc}")
        runs.append(list(ms))
    med = np.median(np.array(runs[1:]), axis=0)
    return dict(zip(("ui", "ei", "yi", "fi"), (float(v) for v in med)), pairs=int(ij), atoms=int(n))

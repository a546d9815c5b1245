"""Drives a cpuSnap.h-style library through the call sequence of MDP's
snappotential (src/Julia/Potential/snapcpp.jl:323-426): pair list, pairs, Ui,
wself, Ei, Yi, Fi, plus Bi.  Used to run the reference library and ours on
identical inputs."""
import ctypes as C

import numpy as np

D = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
I = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")


def bind(path):
    L = C.CDLL(path)
    L.cpuInitSna.argtypes = [D, D, D, I, I, I, I, I, I, I, C.c_int]
    L.cpuNeighPairList.argtypes = [I, I, D, D, I, I, I, I, I, C.c_int, C.c_int, C.c_int]
    L.cpuNeighPairs.argtypes = [D, D, I, I, I, I, I, I, I, I, I, I, C.c_int, C.c_int]
    L.cpuSnapComputeUi.argtypes = [D, D, D, D, D, D, C.c_double, C.c_double, C.c_double, I, I, I, I] + [C.c_int] * 6
    L.cpuAddWself2Ui.argtypes = [D, D, C.c_double, I, I, I] + [C.c_int] * 6
    L.cpuSnapComputeEi.argtypes = [D, D, D, D, D, D, I, I, I, I, I, I] + [C.c_int] * 10
    L.cpuSnapComputeBi.argtypes = [D, D, D, D, D, I, I, I, I] + [C.c_int] * 9
    L.cpuSnapComputeYi.argtypes = [D, D, D, D, D, D, I, I, I, I, I, I] + [C.c_int] * 9
    L.cpuSnapComputeFi.argtypes = [D, D, D, D, D, D, D, D, C.c_double, C.c_double, C.c_double, I, I, I, I, I, I] + \
        [C.c_int] * 7
    for f in ("idxbcount", "idxcgcount", "idxucount", "idxzcount"):
        getattr(L, f).argtypes = [C.c_int]
    # descriptor chain (cpuSnap.h:48-84)
    L.cpuComputeSij.argtypes = [D] * 8 + [D, D, D, D, C.c_double, C.c_double, C.c_double, I, I, I] + [C.c_int] * 4
    L.cpuComputeUij.argtypes = [D] * 4 + [D, D, D, D, C.c_double, C.c_double, C.c_double, I, I, I] + [C.c_int] * 4
    L.cpuZeroUarraytot2.argtypes = [D, D, C.c_double, I, I, I, I] + [C.c_int] * 6
    L.cpuAddUarraytot.argtypes = [D, D, D, D, I, I, I] + [C.c_int] * 4
    L.cpuComputeZi2.argtypes = [D, D, D, D, D, I, I, I] + [C.c_int] * 6
    L.cpuComputeBi2.argtypes = [D, D, D, D, D, D, I, I, I, I, I, I] + [C.c_int] * 9
    L.cpuComputeDbidrj.argtypes = [D, D, D, D, D, I, I, I, I, I, I] + [C.c_int] * 9
    L.cpuSnapTallyBispectrum.argtypes = [D, D, I, I] + [C.c_int] * 5
    L.cpuSnapTallyBispectrumDeriv.argtypes = [D, D, D, I, I, I, I] + [C.c_int] * 6
    L.cpuSnapTallyBispectrumVirial.argtypes = [D, D, D, D, I, I] + [C.c_int] * 6
    return L


def tables(L, tj):
    nb, ncg, nu, nz = L.idxbcount(tj), L.idxcgcount(tj), L.idxucount(tj), L.idxzcount(tj)
    jd = tj + 1
    fac = np.ones(168)
    for k in range(1, 168):
        fac[k] = fac[k - 1] * k
    t = dict(rootpq=np.zeros((jd + 1) ** 2), cg=np.zeros(ncg), fac=fac,
             idx_max=np.zeros(5, dtype=np.int32), idxz=np.zeros(10 * nz, dtype=np.int32),
             idxz_block=np.zeros(jd ** 3, dtype=np.int32), idxb=np.zeros(3 * nb, dtype=np.int32),
             idxb_block=np.zeros(jd ** 3, dtype=np.int32), idxu_block=np.zeros(jd, dtype=np.int32),
             idxcg_block=np.zeros(jd ** 3, dtype=np.int32), nb=nb, nu=nu, nz=nz, ncg=ncg)
    L.cpuInitSna(t["rootpq"], t["cg"], t["fac"], t["idx_max"], t["idxz"], t["idxz_block"], t["idxb"],
                 t["idxb_block"], t["idxu_block"], t["idxcg_block"], tj)
    return t


def _pairs(L, g, p):
    """Pair list and pair arrays of golden fixture g (cpuNeighPairList, cpuNeighPairs)."""
    x = np.ascontiguousarray(g["xall"]).ravel()
    n = g["x"].shape[0]
    nl, nn = g["neighlist"], g["neighnum"]
    csr = np.zeros(n + 1, dtype=np.int32); csr[1:] = np.cumsum(nn)
    flat = np.concatenate([nl[i, : nn[i]] for i in range(n)]).astype(np.int32)
    ilist = np.arange(n, dtype=np.int32)
    anum = g["xall"].shape[0]
    atype = np.ones(anum, dtype=np.int32)
    alist = np.ascontiguousarray(g["alist"], dtype=np.int32)
    rc = p.rcut
    rcutsq = np.array([0.0, 0.0, 0.0, rc * rc])
    pairnum = np.zeros(n, dtype=np.int32)
    pairlist = np.zeros(flat.size + 1, dtype=np.int32)
    L.cpuNeighPairList(pairnum, pairlist, x, rcutsq, ilist, flat, csr, atype, alist, n, 3, 1)
    pns = np.zeros(n + 1, dtype=np.int32); pns[1:] = np.cumsum(pairnum)
    ij = int(pns[-1])
    rij = np.zeros(3 * ij); aii = np.zeros(ij, dtype=np.int32); ai = np.zeros(ij, dtype=np.int32)
    aj = np.zeros(ij, dtype=np.int32); ti = np.zeros(ij, dtype=np.int32); tjv = np.zeros(ij, dtype=np.int32)
    L.cpuNeighPairs(rij, x, aii, ai, aj, ti, tjv, pairlist, pns, ilist, atype, alist, n, 3)
    radelem = np.array([0.0, p.radelem]); wjelem = np.array([0.0, p.wjelem]); mp = np.zeros(2, dtype=np.int32)
    return dict(n=n, ij=ij, ilist=ilist, atype=atype, pairnum=pairnum, pairlist=pairlist, rij=rij, aii=aii, ai=ai,
                aj=aj, ti=ti, tjv=tjv, radelem=radelem, wjelem=wjelem, mp=mp)


def snap_sequence(L, g, p):
    """Returns every stage's output for the configuration in golden fixture g."""
    tj = p.twojmax
    t = tables(L, tj)
    q = _pairs(L, g, p)
    n, ij, ilist, atype, pairnum, pairlist = q["n"], q["ij"], q["ilist"], q["atype"], q["pairnum"], q["pairlist"]
    rij, aii, ai, aj, ti, tjv = q["rij"], q["aii"], q["ai"], q["aj"], q["ti"], q["tjv"]
    radelem, wjelem, mp = q["radelem"], q["wjelem"], q["mp"]
    nu = t["nu"]
    ur = np.zeros(n * nu); ui = np.zeros(n * nu)
    L.cpuSnapComputeUi(ur, ui, t["rootpq"], rij, wjelem, radelem, p.rmin0, p.rfac0, p.rcutfac, mp, ai, ti, tjv,
                       tj, nu, n, ij, p.switchflag, 0)
    u_pairs = (ur.copy(), ui.copy())
    L.cpuAddWself2Ui(ur, ui, 1.0, t["idxu_block"], atype, mp, p.wselfallflag, 0, nu, 1, tj, n)
    bzero = np.array([1.0 if p.bnormflag else j + 1.0 for j in range(tj + 1)])
    coeff = np.ascontiguousarray(p.coeff)
    e = np.zeros(n)
    L.cpuSnapComputeEi(e, ur, ui, t["cg"], bzero, coeff, ilist, mp, atype, t["idxb"], t["idxcg_block"],
                       t["idxu_block"], tj, t["nb"], nu, 1, coeff.size, p.bnormflag, p.bzeroflag, p.wselfallflag, 0, n)
    b = np.zeros(n * t["nb"])
    L.cpuSnapComputeBi(b, ur, ui, t["cg"], bzero, t["idxb"], t["idxcg_block"], t["idxu_block"], t["idxz_block"],
                       tj, t["nb"], nu, t["nz"], 1, p.bnormflag, p.bzeroflag, p.wselfallflag, n)
    yr = np.zeros(n * nu); yi = np.zeros(n * nu)
    L.cpuSnapComputeYi(yr, yi, ur, ui, t["cg"], coeff, mp, atype, t["idxz"], t["idxb_block"], t["idxu_block"],
                       t["idxcg_block"], tj, t["nb"], nu, t["nz"], 1, coeff.size, p.bnormflag, 0, n)
    f = np.zeros(3 * n); v = np.zeros(6 * n)
    L.cpuSnapComputeFi(f, v, yr, yi, t["rootpq"], rij, wjelem, radelem, p.rmin0, p.rfac0, p.rcutfac, mp, ai, ai, aj,
                       ti, tjv, tj, nu, n, n, ij, p.switchflag, 0)
    return dict(tables=t, pairnum=pairnum, pairlist=pairlist[:ij], rij=rij, aii=aii, ai=ai, aj=aj, u_pairs=u_pairs,
                u=(ur, ui), eatom=e, blist=b, y=(yr, yi), fatom=f, vatom=v)


def descriptor_sequence(L, g, p, quadratic=0):
    """snapdescriptors' calls after the pair list (src/Julia/Potential/snapcpp.jl:539-665):
    per-pair U and dU (cpuComputeUij, and cpuComputeSij on the same pairs), U
    totals, Z, B, dB/dr and the three tallies.  Returns every stage's output."""
    tj = p.twojmax
    t = tables(L, tj)
    q = _pairs(L, g, p)
    n, ij, ilist, atype = q["n"], q["ij"], q["ilist"], q["atype"]
    rij, ai, aj, ti, tjv, mp = q["rij"], q["ai"], q["aj"], q["ti"], q["tjv"], q["mp"]
    nu, nz, nb = t["nu"], t["nz"], t["nb"]
    geo = (t["rootpq"], rij, q["wjelem"], q["radelem"], p.rmin0, p.rfac0, p.rcutfac, t["idxu_block"], ti, tjv, tj, nu,
           ij, p.switchflag)
    ur = np.zeros(nu * ij); ui = np.zeros(nu * ij); dur = np.zeros(3 * nu * ij); dui = np.zeros(3 * nu * ij)
    L.cpuComputeUij(ur, ui, dur, dui, *geo)
    s8 = [np.zeros(nu * ij) for _ in range(8)]
    L.cpuComputeSij(*s8, *geo)
    utr = np.zeros(n * nu); uti = np.zeros(n * nu)
    L.cpuZeroUarraytot2(utr, uti, 1.0, t["idxu_block"], atype, mp, ai, p.wselfallflag, 0, nu, 1, tj, n)
    L.cpuAddUarraytot(utr, uti, ur, ui, mp, ai, tjv, nu, n, ij, 0)
    zr = np.zeros(nz * n); zi = np.zeros(nz * n)
    L.cpuComputeZi2(zr, zi, utr, uti, t["cg"], t["idxz"], t["idxu_block"], t["idxcg_block"], tj, nu, nz, 1,
                    p.bnormflag, n)
    bzero = np.array([1.0 if p.bnormflag else j + 1.0 for j in range(tj + 1)])
    bl = np.zeros(nb * n)
    L.cpuComputeBi2(bl, zr, zi, utr, uti, bzero, ilist, atype, mp, t["idxb"], t["idxu_block"], t["idxz_block"], tj,
                    nb, nu, nz, 1, p.bzeroflag, p.wselfallflag, 0, n)
    dbl = np.zeros(nb * 3 * ij)
    L.cpuComputeDbidrj(dbl, zr, zi, dur, dui, t["idxb"], t["idxu_block"], t["idxz_block"], mp, ai, tjv, tj, nb, nu,
                       nz, 1, p.bnormflag, 0, n, ij)
    nper = nb + (nb * (nb + 1) // 2 if quadratic else 0)
    bi = np.zeros(nper)
    L.cpuSnapTallyBispectrum(bi, bl, ilist, atype, n, nb, nper, 1, quadratic)
    bd = np.zeros(nper * 3 * n)
    L.cpuSnapTallyBispectrumDeriv(bd, bl, dbl, ai, ai, aj, ti, n, ij, nb, nper, 1, quadratic)
    bv = np.zeros(6 * nper)
    L.cpuSnapTallyBispectrumVirial(bv, bl, dbl, rij, ai, ti, n, ij, nb, nper, 1, quadratic)
    return dict(ulist=(ur, ui), dulist=(dur, dui), sij=tuple(s8), utot=(utr, uti), zlist=(zr, zi), blist=bl,
                dblist=dbl, bi=bi, bd=bd, bv=bv)


def snap_sequence_elements(L, g, p):
    """The same call sequence for a multi-element fixture (tests/golden/chem_*.npz):
    types 1..nelements (owners' types through alist for ghosts), map[t] = t - 1,
    type-pair cutoffs (radelem_i + radelem_j) rcutfac, element blocks of U and
    Y when chemflag is set.  Returns every stage's output."""
    tj = p.twojmax
    t = tables(L, tj)
    ne = p.nelements
    chem = int(p.chemflag)
    nelem = ne if chem else 1
    x = np.ascontiguousarray(g["xall"]).ravel()
    n = g["x"].shape[0]
    nl, nn = g["neighlist"], g["neighnum"]
    csr = np.zeros(n + 1, dtype=np.int32); csr[1:] = np.cumsum(nn)
    flat = np.concatenate([nl[i, : nn[i]] for i in range(n)]).astype(np.int32)
    ilist = np.arange(n, dtype=np.int32)
    alist = np.ascontiguousarray(g["alist"], dtype=np.int32)
    atype = np.ascontiguousarray(g["types"][alist], dtype=np.int32)
    rad = np.concatenate([[0.0], p.radelems]); wj = np.concatenate([[0.0], p.wjelems])
    mp = np.concatenate([[0], np.arange(ne)]).astype(np.int32)
    rcutsq = np.zeros((ne + 1) ** 2)
    for a in range(ne):
        for b in range(ne):
            rcutsq[b + 1 + (a + 1) * (ne + 1)] = ((p.radelems[a] + p.radelems[b]) * p.rcutfac) ** 2
    pairnum = np.zeros(n, dtype=np.int32)
    pairlist = np.zeros(flat.size + 1, dtype=np.int32)
    L.cpuNeighPairList(pairnum, pairlist, x, rcutsq, ilist, flat, csr, atype, alist, n, 3, ne)
    pns = np.zeros(n + 1, dtype=np.int32); pns[1:] = np.cumsum(pairnum)
    ij = int(pns[-1])
    rij = np.zeros(3 * ij); aii = np.zeros(ij, dtype=np.int32); ai = np.zeros(ij, dtype=np.int32)
    aj = np.zeros(ij, dtype=np.int32); ti = np.zeros(ij, dtype=np.int32); tjv = np.zeros(ij, dtype=np.int32)
    L.cpuNeighPairs(rij, x, aii, ai, aj, ti, tjv, pairlist, pns, ilist, atype, alist, n, 3)
    nu = t["nu"]
    ur = np.zeros(n * nu * nelem); ui = np.zeros(n * nu * nelem)
    L.cpuSnapComputeUi(ur, ui, t["rootpq"], rij, wj, rad, p.rmin0, p.rfac0, p.rcutfac, mp, aii, ti, tjv,
                       tj, nu, n, ij, p.switchflag, chem)
    u_pairs = (ur.copy(), ui.copy())
    ltype = np.ascontiguousarray(atype[:n])
    L.cpuAddWself2Ui(ur, ui, 1.0, t["idxu_block"], ltype, mp, p.wselfallflag, chem, nu, nelem, tj, n)
    bzero = np.array([1.0 if p.bnormflag else j + 1.0 for j in range(tj + 1)])
    coeff = np.ascontiguousarray(p.coeff)
    e = np.zeros(n)
    L.cpuSnapComputeEi(e, ur, ui, t["cg"], bzero, coeff, ilist, mp, ltype, t["idxb"], t["idxcg_block"],
                       t["idxu_block"], tj, t["nb"], nu, nelem, p.ncoeffall, p.bnormflag, p.bzeroflag,
                       p.wselfallflag, chem, n)
    b = np.zeros(n * t["nb"] * nelem ** 3)
    L.cpuSnapComputeBi(b, ur, ui, t["cg"], bzero, t["idxb"], t["idxcg_block"], t["idxu_block"], t["idxz_block"],
                       tj, t["nb"], nu, t["nz"], nelem, p.bnormflag, p.bzeroflag, p.wselfallflag, n)
    yr = np.zeros(n * nu * nelem); yi = np.zeros(n * nu * nelem)
    L.cpuSnapComputeYi(yr, yi, ur, ui, t["cg"], coeff, mp, ltype, t["idxz"], t["idxb_block"], t["idxu_block"],
                       t["idxcg_block"], tj, t["nb"], nu, t["nz"], nelem, p.ncoeffall, p.bnormflag, chem, n)
    f = np.zeros(3 * n); v = np.zeros(6 * n)
    L.cpuSnapComputeFi(f, v, yr, yi, t["rootpq"], rij, wj, rad, p.rmin0, p.rfac0, p.rcutfac, mp, aii, ai, aj,
                       ti, tjv, tj, nu, n, n, ij, p.switchflag, chem)
    return dict(pairnum=pairnum, pairlist=pairlist[:ij], rij=rij, u_pairs=u_pairs, u=(ur, ui), eatom=e, blist=b,
                y=(yr, yi), fatom=f, vatom=v)

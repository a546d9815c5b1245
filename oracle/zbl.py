"""Test infrastructure (oracle): the ZBL pair potential of MDP's snapTA06A
example restated in numpy, as simulating/snap/ZBLpotential.jl defines it:

    u(r) = E_zbl(r) + s(r),  E_zbl = Z^2 qqr2e / r * sum_k c_k exp(-d_k r / a),
    1/a = 2 Z^0.23 / 0.4685,
    s(r) = sw5 + A(t) t^3 (sw3 + sw4 t),  t = r - r_inner,
    A(t) = 1/2 + 1/2 tanh(100 t),

with sw3, sw4, sw5 from E_zbl and its first two derivatives at r_outer
(ZBLpotential.jl:66-99).  It is checked against MDP's generated code for the
same potential (src/C++/Potentials/cpuPairaGradient.cpp, compiled behind
oracle/ref_harness.cpp)."""
import numpy as np

C = np.array([0.02817, 0.28022, 0.50986, 0.18175])
D = np.array([0.20162, 0.40290, 0.94229, 3.19980])
A0, PZBL, QQR2E = 0.46850, 0.23, 14.399645


def zbl_terms(r, z):
    """E_zbl and its first two derivatives (ZBLpotential.jl:14-63)."""
    r = np.asarray(r, dtype=np.float64)[..., None]
    ainv = 2.0 * z ** PZBL / A0
    da = D * ainv
    ex = np.exp(-da * r)
    s = (C * ex).sum(-1)
    sp = (-C * da * ex).sum(-1)
    spp = (C * da * da * ex).sum(-1)
    r = r[..., 0]
    zze = z * z * QQR2E
    return zze * s / r, zze * (sp - s / r) / r, zze * (spp - 2.0 * sp / r + 2.0 * s / r / r) / r


def switch_coeffs(inner, outer, z):
    tc = outer - inner
    fc, fcp, fcpp = zbl_terms(outer, z)
    swa = (-3.0 * fcp + tc * fcpp) / (tc * tc)
    swb = (2.0 * fcp - tc * fcpp) / (tc * tc * tc)
    swc = -fc + 0.5 * tc * fcp - tc * tc / 12.0 * fcpp
    return swa / 3.0, swb / 4.0, swc


def zbl_pair(xij, inner=4.0, outer=4.8, z=73.0):
    """u and du/dx_ij for pair vectors xij (n, 3)."""
    xij = np.asarray(xij, dtype=np.float64)
    r = np.sqrt((xij * xij).sum(-1))
    e, ep, _ = zbl_terms(r, z)
    sw3, sw4, sw5 = switch_coeffs(inner, outer, z)
    t = r - inner
    th = np.tanh(100.0 * t)
    a, da = 0.5 + 0.5 * th, 50.0 * (1.0 - th * th)
    poly = sw3 + sw4 * t
    u = e + sw5 + a * t ** 3 * poly
    dudr = ep + da * t ** 3 * poly + a * (3.0 * t * t * poly + t ** 3 * sw4)
    return u, (dudr / r)[:, None] * xij


def zbl_tally(xall, neighlist, neighnum, rcut, **kw):
    """Per-atom energy, force and virial (6, n) of MDP's full-list pair driver
    (cpuPotentials.cpp:1587-1650, cpuEnergyForceTally.cpp:216-227,
    cpuVirialTally.cpp:34-58): e_i += u/2, f_i += du/dx_ij,
    v_i -= x_ij (x) du/dx_ij / 2, over pairs with |x_ij|^2 <= rcut^2."""
    n = neighlist.shape[0]
    e = np.zeros(n); f = np.zeros((n, 3)); v = np.zeros((6, n))
    for i in range(n):
        js = neighlist[i, : neighnum[i]]
        d = xall[js] - xall[i]
        keep = (d * d).sum(-1) <= rcut * rcut
        d = d[keep]
        if len(d) == 0:
            continue
        u, ux = zbl_pair(d, **kw)
        e[i] = 0.5 * u.sum()
        f[i] = ux.sum(0)
        for k, (a, b) in enumerate(((0, 0), (1, 1), (2, 2), (0, 1), (0, 2), (1, 2))):
            v[k, i] = -0.5 * (d[:, a] * ux[:, b]).sum()
    return e, f, v

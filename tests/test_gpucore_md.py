"""GPU: the MD-loop entry points behind mdpcore.h's backend-2 dispatch
(include/mdp_b200_gpucore.h) on device arrays, against MDP's own CPU code
(the compiled reference core behind oracle/ref_harness.cpp) or against
restatements of it: prefix sums, ghost atoms, cell lists, full neighbour
lists, velocity Verlet, periodic wrapping, kinetic energy, column sums, and
the per-atom-beta form of Yi."""
import ctypes as C

import numpy as np
import pytest

from conftest import golden_params, load_golden
from oracle import refpy

pytestmark = pytest.mark.gpu

P = C.c_void_p


def lib():
    from mdp_b200 import _lib
    L = _lib.lib()
    L.mdp_gpu_cumsum.argtypes = [P, P, P, P, C.c_int]
    L.mdp_gpu_atom_list3d_f64.argtypes = [P] * 10 + [C.c_int] * 3
    L.mdp_gpu_cell_list3d_f64.argtypes = [P] * 7 + [C.c_int] * 3
    L.mdp_gpu_cell2atom_list.argtypes = [P] * 5 + [C.c_int] * 2
    L.mdp_gpu_full_neighbor_list3d_cells_f64.argtypes = [P] * 9 + [C.c_int] * 3
    L.mdp_gpu_full_neighbor_list3d_f64.argtypes = [P] * 4 + [C.c_int] * 4
    for f in (L.mdp_gpu_initial_integrate_f64, L.mdp_gpu_final_integrate_f64):
        f.argtypes = [P] * 12 + [C.c_double, P, P] + [C.c_int] * 7
    L.mdp_gpu_pbc_f64.argtypes = [P] * 11 + [C.c_int] * 4
    L.mdp_gpu_compute_ke_atom_f64.argtypes = [P, P, P, C.c_double, P, P, C.c_int, C.c_int]
    L.mdp_gpu_array_sum_every_column_f64.argtypes = [P, P, C.c_int, C.c_int]
    L.mdp_gpu_array_get_value_at_index_int.argtypes = [P, C.c_int]
    L.mdp_gpu_array_get_value_at_index_int.restype = C.c_int
    L.mdp_gpu_snap_compute_yi_beta_f64.argtypes = [P] * 10 + [C.c_int] * 7
    L.mdp_gpu_snap_compute_yi_f64.argtypes = [P] * 12 + [C.c_int] * 8
    return L


def dev(a, dtype=None):
    import torch
    a = np.ascontiguousarray(a if dtype is None else np.asarray(a, dtype=dtype))
    return torch.from_numpy(a.copy()).cuda()


_KEEP = []


@pytest.fixture(autouse=True)
def _release_tensors():
    yield
    _KEEP.clear()


def ptr(t):
    # the tensor stays referenced until the test ends, so a temporary passed
    # inline cannot be freed and its block handed to the next argument
    _KEEP.append(t)
    return C.c_void_p(t.data_ptr())


def sync():
    import torch
    torch.cuda.synchronize()


@pytest.mark.parametrize("length", [1, 2, 7, 4096, 4097, 70001])
def test_cumsum(cuda_lib, length):
    L = lib()
    rng = np.random.default_rng(length)
    a = rng.integers(0, 50, length).astype(np.int32)
    d_in, d_out, d_sums = dev(a), dev(np.full(length, -7, np.int32)), dev(np.zeros(length + 8, np.int32))
    L.mdp_gpu_cumsum(ptr(d_out), ptr(d_in), ptr(d_sums), ptr(d_sums), length)
    sync()
    want = np.zeros(length, np.int64)
    want[1:] = np.cumsum(a[:-1])
    assert np.array_equal(d_out.cpu().numpy(), want)
    assert L.mdp_gpu_array_get_value_at_index_int(ptr(d_out), length - 1) == int(want[-1])


def box_inputs(box, rc):
    bs = refpy.box_setup(box, rc)
    smax = bs["rbvertices"][18:21]
    nc = bs["cellnum"].copy()
    ne2 = max(1, int(np.round(1.0 / (smax[2] - 1.0))))
    cnum = int(nc[0] * nc[1] * (ne2 + 2))
    return bs, nc, cnum


@pytest.mark.parametrize("name", ["bcc250_2j8", "bcc128_2j6", "bcc250_2j8_hot"])
def test_neighbor_build_matches_reference(cuda_lib, name):
    """AtomList3D -> CellList3D -> Cell2AtomList -> FullNeighborList3D on the
    GPU entry points equals MDP's CPU chain: ghosts and owners bit-identical,
    neighbour rows identical including their order."""
    L = lib()
    g = load_golden(name)
    p = golden_params(g)
    x0 = np.ascontiguousarray(g["x"])
    inum = x0.shape[0]
    rc = p.rcut + float(g["skin"])
    nm = int(g["neighmax"])
    bs, nc, cnum = box_inputs(g["box"], rc)
    pnum = int(bs["pnum"])
    xr, alr, nlr, nnr = refpy.neighbor_list(x0, g["box"], p.rcut, float(g["skin"]), nm, neighcell=1)
    anum = xr.shape[0]
    cap = inum * 8 + 4096
    x = np.zeros((cap, 3)); x[:inum] = x0
    dx = dev(x)
    alist = dev(np.zeros(cap, np.int32)); inside = dev(np.zeros(inum * pnum, np.int32))
    gsum = dev(np.zeros(inum + 1, np.int32)); gnum = dev(np.zeros(inum + 1, np.int32))
    sums = dev(np.zeros(inum + 8, np.int32))
    pim, wc, s2r = dev(bs["pimages"]), dev(bs["rbvertices"]), dev(bs["s2rmap"])
    L.mdp_gpu_atom_list3d_f64(ptr(alist), ptr(inside), ptr(gsum), ptr(gnum), ptr(sums), ptr(sums), ptr(dx), ptr(pim),
                              ptr(wc), ptr(s2r), inum, pnum, 3)
    g_tot = L.mdp_gpu_array_get_value_at_index_int(ptr(gsum), inum)
    assert inum + g_tot == anum
    assert np.array_equal(dx.cpu().numpy()[:anum], xr)
    assert np.array_equal(alist.cpu().numpy()[:anum], alr)
    clist = dev(np.zeros(anum, np.int32))
    e1, e2, e3, dnc = dev(bs["eta1"]), dev(bs["eta2"]), dev(bs["eta3"]), dev(nc.astype(np.int32))
    L.mdp_gpu_cell_list3d_f64(ptr(clist), ptr(dx), ptr(e1), ptr(e2), ptr(e3), ptr(s2r), ptr(dnc), inum, anum, 3)
    c2alist = dev(np.zeros(anum, np.int32)); c2anum = dev(np.zeros(anum, np.int32))
    c2anumsum = dev(np.zeros(cnum + 1, np.int32))
    L.mdp_gpu_cell2atom_list(ptr(c2alist), ptr(c2anumsum), ptr(c2anum), ptr(clist), ptr(sums), anum, cnum)
    sync()
    cl = clist.cpu().numpy()
    order = np.argsort(cl, kind="stable")
    assert np.array_equal(c2alist.cpu().numpy(), order)
    assert np.array_equal(c2anum.cpu().numpy(), cl[order])
    assert np.array_equal(c2anumsum.cpu().numpy(), np.concatenate([[0], np.cumsum(np.bincount(cl, minlength=cnum))]))
    nl = dev(np.full(inum * nm, -1, np.int32)); nn = dev(np.zeros(inum, np.int32))
    rcs = dev(np.array([rc * rc]))
    L.mdp_gpu_full_neighbor_list3d_cells_f64(ptr(nl), ptr(nn), ptr(dx), ptr(rcs), ptr(alist), ptr(clist),
                                             ptr(c2alist), ptr(c2anumsum), ptr(dnc), inum, nm, 3)
    sync()
    nn_h, nl_h = nn.cpu().numpy(), nl.cpu().numpy().reshape(inum, nm)
    assert np.array_equal(nn_h, nnr)
    for i in range(inum):
        assert np.array_equal(nl_h[i, : nn_h[i]], nlr[i, : nnr[i]])
    # all-pairs form against MDP's O(N^2) list
    _, _, nl0, nn0 = refpy.neighbor_list(x0, g["box"], p.rcut, float(g["skin"]), nm, neighcell=0)
    L.mdp_gpu_full_neighbor_list3d_f64(ptr(nl), ptr(nn), ptr(dx), ptr(rcs), anum, inum, nm, 3)
    sync()
    nn_h, nl_h = nn.cpu().numpy(), nl.cpu().numpy().reshape(inum, nm)
    assert np.array_equal(nn_h, nn0)
    for i in range(inum):
        assert np.array_equal(nl_h[i, : nn_h[i]], nl0[i, : nn0[i]])


@pytest.mark.parametrize("mode", [0, 1])
def test_velocity_verlet(cuda_lib, mode):
    L = lib()
    rng = np.random.default_rng(3 + mode)
    n, dim = 5000, 3
    x, v, f = rng.normal(size=(n, dim)), rng.normal(size=(n, dim)) * 3, rng.normal(size=(n, dim)) * 40
    mass = np.array([0.0, 180.88, 92.9]); typ = rng.integers(1, 3, n).astype(np.int32)
    ilist = rng.permutation(n).astype(np.int32)[: n - 100]
    dtarray = np.array([0.0, 0.5 * 0.001 / 1.0364269e-4, 0.001])
    vlim2 = 4.0
    dx, dv, df, dm, dt, di = dev(x), dev(v), dev(f), dev(mass), dev(typ), dev(ilist)
    z = dev(np.zeros(4))
    args = lambda: [ptr(dx), ptr(dv), ptr(df), ptr(dm), dtarray.ctypes.data_as(C.c_void_p)] + [ptr(z)] * 7 + \
        [vlim2, ptr(dt), ptr(di), 0, 0, 1, 1, mode, dim, len(ilist)]
    L.mdp_gpu_initial_integrate_f64(*args())
    sync()
    xw, vw = x.copy(), v.copy()
    for i in ilist:     # cpuVelocityIntegration.cpp:307-420
        dtfm = dtarray[1] / mass[typ[i]]
        vw[i] = vw[i] + dtfm * f[i]
        if mode == 1:
            vsq = vw[i, 0] * vw[i, 0] + vw[i, 1] * vw[i, 1] + vw[i, 2] * vw[i, 2]
            if vsq > vlim2:
                vw[i] *= np.sqrt(vlim2 / vsq)
        xw[i] = xw[i] + dtarray[2] * vw[i]
    assert np.array_equal(dv.cpu().numpy(), vw) and np.array_equal(dx.cpu().numpy(), xw)
    L.mdp_gpu_final_integrate_f64(*args())
    sync()
    for i in ilist:
        vw[i] = vw[i] + dtarray[1] / mass[typ[i]] * f[i]
        if mode == 1:
            vsq = vw[i, 0] * vw[i, 0] + vw[i, 1] * vw[i, 1] + vw[i, 2] * vw[i, 2]
            if vsq > vlim2:
                vw[i] *= np.sqrt(vlim2 / vsq)
    assert np.array_equal(dv.cpu().numpy(), vw) and np.array_equal(dx.cpu().numpy(), xw)
    # against MDP's own NVE code (mode 0)
    if mode == 0:
        xr, vr = x.copy().ravel(), v.copy().ravel()
        refpy.lib().ref_nve_initial(xr, vr, f.ravel().copy(), mass, dtarray[1], dtarray[2], typ, ilist, len(ilist))
        assert np.abs(xr.reshape(n, dim) - xw).max() <= 1e-12 * np.abs(xw).max()


@pytest.mark.parametrize("triclinic", [0, 1])
def test_pbc(cuda_lib, triclinic):
    L = lib()
    rng = np.random.default_rng(11 + triclinic)
    n = 4000
    lo, hi = np.array([-1.0, 0.5, 2.0]), np.array([9.0, 12.5, 7.0])
    h = np.array([10.0, 12.0, 5.0, 0.0, 0.0, 0.0])          # xx yy zz yz xz xy
    if triclinic:
        h[3:] = [0.4, -0.7, 1.1]
    hinv = np.zeros(6)
    hinv[0], hinv[1], hinv[2] = 1 / h[0], 1 / h[1], 1 / h[2]
    hinv[5] = -h[5] / (h[0] * h[1]); hinv[3] = -h[3] / (h[1] * h[2])
    hinv[4] = (h[3] * h[5] - h[1] * h[4]) / (h[0] * h[1] * h[2])
    lol, hil = np.zeros(3), np.ones(3)
    x = lo + rng.uniform(-0.3, 1.3, (n, 3)) * (hi - lo)
    v = rng.normal(size=(n, 3)); image = rng.integers(-2, 3, (n, 3)).astype(np.int32)
    rate = rng.normal(size=6) * 0.01
    pbc = np.array([1, 1, 0], np.int32)
    dx, dv, dim_ = dev(x), dev(v), dev(image)
    L.mdp_gpu_pbc_f64(ptr(dx), ptr(dv), ptr(dim_), ptr(dev(hi)), ptr(dev(lo)), ptr(dev(hil)), ptr(dev(lol)),
                      ptr(dev(h)), ptr(dev(hinv)), ptr(dev(rate)), ptr(dev(pbc)), 1, triclinic, 3, n)
    sync()
    xw, vw, iw = x.copy(), v.copy(), image.copy()
    shift = {0: [(0, 0)], 1: [(0, 5), (1, 1)], 2: [(0, 4), (1, 3), (2, 2)]}
    for i in range(n):      # cpuDomain.cpp:235-385
        c = xw[i].copy()
        if triclinic:
            d = xw[i] - lo
            c = np.array([hinv[0] * d[0] + hinv[5] * d[1] + hinv[4] * d[2], hinv[1] * d[1] + hinv[3] * d[2],
                          hinv[2] * d[2]])
        L_, lb, ub = (hil, lol, hil) if triclinic else (h, lo, hi)
        for k in range(3):
            if not pbc[k]:
                continue
            if c[k] < lb[k]:
                c[k] += L_[k]; iw[i, k] -= 1
                for a, r in shift[k]:
                    vw[i, a] += rate[r]
            if c[k] >= ub[k]:
                c[k] -= L_[k]; c[k] = max(c[k], lb[k]); iw[i, k] += 1
                for a, r in shift[k]:
                    vw[i, a] -= rate[r]
        if triclinic:
            c = np.array([h[0] * c[0] + h[5] * c[1] + lo[0] + h[4] * c[2], h[1] * c[1] + lo[1] + h[3] * c[2],
                          h[2] * c[2] + lo[2]])
        xw[i] = c
    assert np.array_equal(dim_.cpu().numpy(), iw)
    assert np.allclose(dv.cpu().numpy(), vw, rtol=0, atol=1e-14)
    tol = 1e-12 if triclinic else 0.0
    assert np.abs(dx.cpu().numpy() - xw).max() <= tol


def test_kinetic_energy_and_column_sums(cuda_lib):
    L = lib()
    rng = np.random.default_rng(5)
    n = 3000
    v = rng.normal(size=(n, 3)); mass = np.array([0.0, 180.88, 50.0]); typ = rng.integers(1, 3, n).astype(np.int32)
    ilist = rng.permutation(n).astype(np.int32)
    ke = dev(np.zeros(n))
    mvv2e = 1.0364269e-4
    L.mdp_gpu_compute_ke_atom_f64(ptr(ke), ptr(dev(mass)), ptr(dev(v)), mvv2e, ptr(dev(typ)), ptr(dev(ilist)), 3, n)
    sync()
    want = np.array([0.5 * mvv2e * mass[typ[i]] * (v[i, 0] * v[i, 0] + v[i, 1] * v[i, 1] + v[i, 2] * v[i, 2])
                     for i in ilist])
    assert np.array_equal(ke.cpu().numpy(), want)
    a = rng.normal(size=(6, 777))        # 6 columns of 777 rows, column-major
    b = dev(np.zeros(6))
    L.mdp_gpu_array_sum_every_column_f64(ptr(b), ptr(dev(a)), 6, 777)
    sync()
    assert np.allclose(b.cpu().numpy(), a.sum(axis=1), rtol=1e-14, atol=1e-12)


@pytest.mark.parametrize("name", ["bcc128_2j4", "bcc128_2j6", "bcc250_2j8", "bcc54_2j8_flags"])
def test_yi_per_atom_beta(cuda_lib, name):
    """The beta form of Yi equals the coeffelem form atom by atom: atoms given
    coefficient set A match the coeffelem Yi of A, atoms given B that of B."""
    import julia_abi
    from mdp_b200 import _lib
    L = lib()
    g = load_golden(name)
    p = golden_params(g)
    seq = julia_abi.snap_sequence(julia_abi.bind(_lib.LIB_PATH), g, p)
    t = seq["tables"]
    ur, ui = seq["u"]
    n = g["x"].shape[0]
    nu, nb, nz, tj = t["nu"], t["nb"], t["nz"], p.twojmax
    rng = np.random.default_rng(9)
    cA = np.concatenate([[0.0], rng.normal(0, 0.1, nb)]); cB = np.concatenate([[0.0], rng.normal(0, 0.1, nb)])
    pick = rng.integers(0, 2, n)
    beta = np.where(pick[None, :] == 0, cA[1:, None], cB[1:, None])          # [jjb][inum]
    dur, dui, dcg = dev(ur), dev(ui), dev(t["cg"])
    tabs = [dev(t["idxz"].ravel()), dev(t["idxb_block"]), dev(t["idxu_block"]), dev(t["idxcg_block"])]
    yr, yi = dev(np.zeros(nu * n)), dev(np.zeros(nu * n))
    L.mdp_gpu_snap_compute_yi_beta_f64(ptr(yr), ptr(yi), ptr(dur), ptr(dui), ptr(dcg), ptr(dev(beta)),
                                       *[ptr(x) for x in tabs], tj, nb, nu, nz, 1, p.bnormflag, n)
    sync()
    got = yr.cpu().numpy().reshape(nu, n), yi.cpu().numpy().reshape(nu, n)
    mp, ty = dev(np.zeros(2, np.int32)), dev(np.ones(n, np.int32))
    for which, c in ((0, cA), (1, cB)):
        wr, wi = dev(np.zeros(nu * n)), dev(np.zeros(nu * n))
        L.mdp_gpu_snap_compute_yi_f64(ptr(wr), ptr(wi), ptr(dur), ptr(dui), ptr(dcg), ptr(dev(c)), ptr(mp), ptr(ty),
                                      *[ptr(x) for x in tabs], tj, nb, nu, nz, 1, c.size, p.bnormflag, n)
        sync()
        want = wr.cpu().numpy().reshape(nu, n), wi.cpu().numpy().reshape(nu, n)
        cols = pick == which
        for k in (0, 1):
            scale = max(np.abs(want[k]).max(), 1e-300)
            assert np.abs(got[k][:, cols] - want[k][:, cols]).max() / scale < 1e-13


def test_nvt_matches_reference(cuda_lib):
    """Mode 2 (Nose-Hoover chain NVT) of the integrator entry points against
    MDP's own cpuNVTInitialIntegrate / cpuNVTFinalIntegrate: five steps with a
    ramped target temperature, a 3-link chain and two sub-steps, positions,
    velocities, chain state and temperatures compared after every half step."""
    L = lib()
    R = refpy.lib()
    R.ref_nvt_initial.argtypes = [P] * 12 + [C.c_int] * 4
    R.ref_nvt_final.argtypes = [P] * 12 + [C.c_int] * 4
    rng = np.random.default_rng(17)
    n = 3000
    x, v, f = rng.normal(size=(n, 3)) * 10, rng.normal(size=(n, 3)) * 4, rng.normal(size=(n, 3)) * 5
    mass = np.array([0.0, 180.88, 92.9]); typ = rng.integers(1, 3, n).astype(np.int32)
    ilist = rng.permutation(n).astype(np.int32)[: n - 50]
    dt = 0.001
    dtarray = np.array([dt, 0.5 * dt / 1.0364269e-4, dt, 0.0, 100.0, 0.0])
    tarray = np.array([300.0, 600.0, 10.0, 0.0, 0.0, 3.0 * len(ilist) - 3.0, 8.617343e-5, 0.2, 1.0364269e-4])
    mt, nc = 3, 2
    chains = [np.zeros(mt + 1) for _ in range(4)]        # eta_mass, eta, eta_dot, eta_dotdot
    ref = dict(x=x.copy(), v=v.copy(), d=dtarray.copy(), t=tarray.copy(), c=[a.copy() for a in chains])
    ours = dict(d=dtarray.copy(), t=tarray.copy(), c=[a.copy() for a in chains])
    dx, dv, df, dm, dt_, di = dev(x), dev(v), dev(f), dev(mass), dev(typ), dev(ilist)
    ke, tmp = dev(np.zeros(n)), dev(np.zeros(8))
    hp = lambda a: C.c_void_p(a.ctypes.data)

    def ours_half(fn):
        fn(ptr(dx), ptr(dv), ptr(df), ptr(dm), hp(ours["d"]), hp(ours["t"]), *[hp(a) for a in ours["c"]],
           ptr(ke), ptr(tmp), 0.0, ptr(dt_), ptr(di), 1, 0, mt, nc, 2, 3, len(ilist))
        sync()

    def ref_half(fn):
        fn(hp(ref["x"]), hp(ref["v"]), hp(f), hp(mass), hp(ref["d"]), hp(ref["t"]), *[hp(a) for a in ref["c"]],
           hp(typ), hp(ilist), 1, mt, nc, len(ilist))

    for step in range(1, 6):
        ours["d"][5] = ref["d"][5] = float(step)
        for mine, theirs in ((L.mdp_gpu_initial_integrate_f64, R.ref_nvt_initial),
                             (L.mdp_gpu_final_integrate_f64, R.ref_nvt_final)):
            ours_half(mine)
            ref_half(theirs)
            assert np.abs(dv.cpu().numpy() - ref["v"]).max() <= 1e-12 * np.abs(ref["v"]).max()
            assert np.abs(dx.cpu().numpy() - ref["x"]).max() <= 1e-12 * np.abs(ref["x"]).max()
            assert np.allclose(ours["t"], ref["t"], rtol=1e-12, atol=0)
            for a, b in zip(ours["c"], ref["c"]):
                assert np.allclose(a, b, rtol=1e-10, atol=1e-14)
    assert ref["c"][2][0] != 0.0          # the chain moved

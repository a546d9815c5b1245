"""Generate the committed golden fixtures from the reference's own CPU code.

Run in a container that has the reference tree (the reference is compiled by
`make -C oracle ref`, into oracle/_ref/):

    python tests/golden/make_golden.py

Each fixture holds a seeded synthetic Ta configuration and what MDP's CPU
implementation computes for it:
  * the ghost atoms (positions and owners) and the full neighbour list, built
    by cpuNeighborList3D.cpp in both its O(N^2) and cell forms;
  * per-atom energy, forces and virial from the cpuSnap4.cpp chain
    (ComputePairSnap3 order);
  * for the MD fixtures, a short NVE velocity-Verlet trajectory in the order of
    CIntegration::VelocityVerlet (Integration.cpp:17-139), with thermo rows.
The inputs are regenerated by the tests from the stored seeds and checked
against the stored copies, so the fixtures also pin the input generator.

The tri_* fixtures hold sheared (triclinic) cells with the reference's ghosts,
neighbour lists and per-atom energy, forces and virial (`--tri-only` stops
after them).

The fit_* fixtures hold single configurations of the batched-fitting workload
(BCC / FCC / A15 supercells) with the per-configuration descriptors of MDP's
ComputeSnap chain (snappotential.cpp:762-910, cpuSnap2.cpp): bi, bd, bv and the
per-atom bispectrum (`--fit-only` regenerates just these).
"""
from __future__ import annotations

import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

from mdp_b200 import configs  # noqa: E402
from oracle import refpy  # noqa: E402

# (name, cells, 2J, temp, jitter, seed, coeff seed, flag overrides, md steps, dt)
CASES = [
    ("bcc128_2j6", (4, 4, 4), 6, 300.0, 0.05, 11, 101, {}, 40, 0.0005),
    ("bcc250_2j8", (5, 5, 5), 8, 600.0, 0.05, 12, 102, {}, 20, 0.001),
    ("bcc128_2j4", (4, 4, 4), 4, 1000.0, 0.10, 13, 103, {}, 20, 0.001),
    ("bcc54_2j8_flags", (3, 3, 3), 8, 300.0, 0.08, 14, 104,
     {"bnormflag": 1, "bzeroflag": 1, "switchflag": 0}, 0, 0.001),
    ("bcc250_2j8_hot", (5, 5, 5), 8, 3000.0, 0.20, 15, 105, {}, 0, 0.001),
]
SKIN = 1.0
NEIGHMAX = 80


def thermo_row(step, e, v, vatom, box, mass):
    n = e.size
    tdof = (n - 1) * 3.0
    temp = configs.MVV2E / (tdof * configs.BOLTZ) * mass * np.sum(v * v)
    pe = e.sum() / n
    ke = 0.5 * tdof * configs.BOLTZ * temp / n
    vol = box[0] * box[1] * box[2]
    pres = (tdof * configs.BOLTZ * temp + vatom[0].sum() + vatom[1].sum() + vatom[2].sum()) / 3.0 / vol * configs.NKTV2P
    return [step, temp, pe, pe + ke, pres]


def ref_md(x0, v0, box, p, nsteps, dt, mass, neighmax=NEIGHMAX, nthreads=1, snap_steps=(), snap_atoms=None):
    """NVE in the reference's step order using the reference's own kernels.
    With snap_steps, also returns {step: (x, v)} of the atoms snap_atoms at those steps."""
    dtf = 0.5 * dt * configs.FTM2V
    ilist = np.arange(x0.shape[0], dtype=np.int32)
    typ = np.ones(x0.shape[0] + 1, dtype=np.int32)
    massarr = np.array([0.0, mass])
    x = x0.copy(); v = v0.copy()
    nb = dict(nblocks=8 * nthreads, nthreads=nthreads) if nthreads > 1 else {}
    snaps = {}
    xa, al, nl, nn = refpy.neighbor_list(x, box, p.rcut, SKIN, neighmax, neighcell=0)
    xhold = x.copy()
    e, f, va = refpy.snap_force(xa, al, nl, nn, p, **nb)
    rows = [thermo_row(0, e, v, va, box, mass)]
    rebuilds = 1
    n = x.shape[0]
    lib = refpy.lib()
    for step in range(1, nsteps + 1):
        xstart = x.copy()
        xf = np.ascontiguousarray(x).ravel(); vf = np.ascontiguousarray(v).ravel()
        lib.ref_nve_initial(xf, vf, np.ascontiguousarray(f).ravel(), massarr, dtf, dt, typ, ilist, n)
        x = xf.reshape(n, 3); v = vf.reshape(n, 3)
        if np.max(np.sum((x - xhold) ** 2, axis=1)) > 0.25 * SKIN * SKIN:
            x = np.where(x < 0.0, x + box, x)
            x = np.where(x >= box, np.maximum(x - box, 0.0), x)
            xa, al, nl, nn = refpy.neighbor_list(x, box, p.rcut, SKIN, neighmax, neighcell=0)
            if nn.max() >= neighmax:
                raise RuntimeError("neighmax too small for the reference trajectory")
            xhold = x.copy()
            rebuilds += 1
        else:
            xa = xa.copy()
            xa[:n] = x
            xa[n:] += (x - xstart)[al[n:]]
        e, f, va = refpy.snap_force(xa, al, nl, nn, p, **nb)
        vf = np.ascontiguousarray(v).ravel()
        lib.ref_nve_final(np.ascontiguousarray(x).ravel(), vf, np.ascontiguousarray(f).ravel(), massarr, dtf, typ,
                          ilist, n)
        v = vf.reshape(n, 3)
        rows.append(thermo_row(step, e, v, va, box, mass))
        if step in snap_steps:
            snaps[step] = (x[snap_atoms].copy(), v[snap_atoms].copy())
    if snap_steps:
        return np.array(rows), x, v, f, e, rebuilds, snaps
    return np.array(rows), x, v, f, e, rebuilds


# descriptor fixtures (ComputeSnap chain): (name, kind, target atoms, strain, sigma, seed, 2J, flag overrides)
FIT_CASES = [
    ("fit_bcc16_2j8", "bcc", 16, 0.03, 0.10, 31, 8, {}),
    ("fit_fcc32_2j8", "fcc", 32, -0.04, 0.20, 32, 8, {}),
    ("fit_a15_64_2j8", "a15", 64, 0.00, 0.05, 33, 8, {}),
    ("fit_bcc54_2j6_flags", "bcc", 54, 0.02, 0.30, 34, 6, {"bnormflag": 1, "bzeroflag": 1}),
]


# triclinic descriptor fixtures: as FIT_CASES plus the tilts (xy, xz, yz) as
# fractions of the edge lengths; the cell vectors are a = (Lx, 0, 0),
# b = (xy Lx, Ly, 0), c = (xz Lx, yz Ly, Lz) and the atoms keep their
# fractional coordinates
TRI_FIT_CASES = [
    ("fit_bcc54_tri_2j8", "bcc", 54, 0.02, 0.10, 35, 8, {}, (0.12, -0.08, 0.05)),
    ("fit_fcc108_tri_2j6", "fcc", 108, -0.03, 0.25, 36, 6, {"bnormflag": 1}, (-0.10, 0.06, 0.15)),
]


# sparse descriptor fixtures: (name, atoms, box edge, seed, 2J); one isolated atom, or atoms uniform in
# the box (many with no neighbour inside the cutoff)
SPARSE_FIT_CASES = [
    ("fit_isolated1_2j8", 1, 20.0, 41, 8),
    ("fit_gas40_2j8", 40, 32.0, 42, 8),
]


def sparse_config(n, edge, seed):
    from mdp_b200 import fit
    x = np.array([[3.0, 4.0, 5.0]]) if n == 1 else np.random.default_rng(seed).uniform(0.0, edge, (n, 3))
    return fit.FitConfig(x=x, box=np.array([edge, edge, edge]), kind="sparse")


def sheared(cfg, tilt):
    """The configuration in the sheared cell of the tilts (xy, xz, yz)."""
    from mdp_b200 import fit
    L = np.asarray(cfg.box, dtype=np.float64)
    H = np.array([[L[0], 0.0, 0.0], [tilt[0] * L[0], L[1], 0.0], [tilt[1] * L[0], tilt[2] * L[1], L[2]]])
    return fit.FitConfig(x=(cfg.x / L) @ H, box=H, kind=cfg.kind)


def fit_fixtures():
    """Per configuration: positions, box (edge lengths or cell vectors as rows)
    and the reference's bi, bd, bv, blist."""
    from mdp_b200 import fit
    cases = [c + ((0.0, 0.0, 0.0),) for c in FIT_CASES] + TRI_FIT_CASES
    for (name, kind, target, strain, sigma, seed, tj, flags, tilt) in cases:
        rng = np.random.default_rng(seed)
        cfg = fit.make_config(kind, target, strain, sigma, rng)
        if any(tilt):
            cfg = sheared(cfg, tilt)
        p = configs.snap_params(tj, seed=0, **flags)
        xa, al, nl, nn = refpy.neighbor_list(cfg.x, cfg.box, p.rcut, SKIN, NEIGHMAX, neighcell=0)
        bi, bd, bv, bl = refpy.snap_descriptors(xa, al, nl, nn, p)
        path = os.path.join(HERE, f"{name}.npz")
        np.savez_compressed(path, kind=kind, twojmax=tj, flags=np.array([p.bnormflag, p.bzeroflag, p.switchflag]),
                            x=cfg.x, box=cfg.box, bi=bi, bd=bd, bv=bv, blist=bl)
        print(name, cfg.natoms, "atoms", os.path.getsize(path), "bytes")
    for (name, n, edge, seed, tj) in SPARSE_FIT_CASES:
        cfg = sparse_config(n, edge, seed)
        p = configs.snap_params(tj, seed=0)
        xa, al, nl, nn = refpy.neighbor_list(cfg.x, cfg.box, p.rcut, SKIN, NEIGHMAX, neighcell=0)
        bi, bd, bv, bl = refpy.snap_descriptors(xa, al, nl, nn, p)
        path = os.path.join(HERE, f"{name}.npz")
        np.savez_compressed(path, kind=cfg.kind, twojmax=tj, flags=np.array([p.bnormflag, p.bzeroflag,
                                                                             p.switchflag]),
                            x=cfg.x, box=cfg.box, bi=bi, bd=bd, bv=bv, blist=bl)
        print(name, cfg.natoms, "atoms", os.path.getsize(path), "bytes")


# sheared-cell force fixtures: (name, cells, 2J, temp, jitter, seed, coeff seed, tilts (xy, xz, yz)); the
# atoms of the orthogonal lattice keep their fractional coordinates in the cell a = (Lx, 0, 0),
# b = (xy Lx, Ly, 0), c = (xz Lx, yz Ly, Lz)
TRI_CASES = [
    ("tri_bcc128_2j8", (4, 4, 4), 8, 300.0, 0.05, 16, 106, (0.10, -0.05, 0.08)),
    ("tri_bcc250_2j6", (5, 5, 5), 6, 1000.0, 0.10, 17, 107, (-0.15, 0.12, 0.0)),
]


def tri_config(cells, temp, jit, seed, tilt):
    """Positions and cell vectors (rows) of a sheared case."""
    cfg = configs.ta_config(cells, temp=temp, jitter=jit, seed=seed)
    L = np.asarray(cfg.box, dtype=np.float64)
    H = np.array([[L[0], 0.0, 0.0], [tilt[0] * L[0], L[1], 0.0], [tilt[1] * L[0], tilt[2] * L[1], L[2]]])
    s = cfg.x / L
    s -= np.floor(s)
    return s @ H, H


def tri_fixtures():
    """Sheared cells: the reference's ghosts, both neighbour-list forms and
    per-atom energy, forces and virial."""
    for (name, cells, tj, temp, jit, seed, cseed, tilt) in TRI_CASES:
        p = configs.snap_params(tj, seed=cseed)
        x, H = tri_config(cells, temp, jit, seed, tilt)
        xa0, al0, nl0, nn0 = refpy.neighbor_list(x, H, p.rcut, SKIN, NEIGHMAX, neighcell=0)
        xa1, al1, nl1, nn1 = refpy.neighbor_list(x, H, p.rcut, SKIN, NEIGHMAX, neighcell=1)
        e, f, va = refpy.snap_force(xa0, al0, nl0, nn0, p)
        path = os.path.join(HERE, f"{name}.npz")
        np.savez_compressed(path, cells=np.array(cells), twojmax=tj, temp=temp, jitter=jit, seed=seed,
                            coeff_seed=cseed, tilt=np.array(tilt), flags=np.array([p.bnormflag, p.bzeroflag,
                                                                                   p.switchflag]),
                            skin=SKIN, neighmax=NEIGHMAX, x=x, box=H, coeff=p.coeff, xall=xa0, alist=al0,
                            neighlist=nl0, neighnum=nn0, neighlist_cell=nl1, neighnum_cell=nn1,
                            xall_cell=xa1, alist_cell=al1, eatom=e, fatom=f, vatom=va)
        print(name, x.shape[0], "atoms", xa0.shape[0] - x.shape[0], "ghosts", os.path.getsize(path), "bytes")


# The 16,000-atom configuration of the benchmark's FP64-vs-reference check: 20x20x20 BCC Ta cells at
# 600 K, jitter 0.05 A, 2J=8 with seeded coefficients beta_k ~ N(0, 0.01), 1,000 NVE steps of 1 fs.
# Coefficients drawn at random need not hold a BCC crystal together: of the seeds 2017-2096, run for
# 1,000 steps at 600 K, most heat up or collapse (one reached 1.8 million K).  Seed 2022 keeps the
# temperature near 570 K and the potential energy flat, and rebuilds the neighbour list a dozen times.
C2 = dict(name="c2_bcc16000_2j8", cells=(20, 20, 20), twojmax=8, temp=600.0, jitter=0.05, seed=2016,
          coeff_seed=2022, dt=0.001, steps=1000, neighmax=80, snap_steps=(100, 1000), atom_stride=8)


def row_hashes(nl, nn):
    """One 64-bit hash per neighbour row, of its sorted index set (tests/conftest.py restates it)."""
    from conftest import row_hashes as rh
    return rh(nl, nn)


def c2_fixture(nthreads):
    """The reference's neighbour rows (as per-row hashes), ghosts, per-atom energy/force/virial sums
    and a 1,000-step NVE run (thermo every step; positions and velocities of every 8th atom at steps
    100 and 1,000) for the 16,000-atom configuration."""
    c = C2
    p = configs.snap_params(c["twojmax"], seed=c["coeff_seed"])
    cfg = configs.ta_config(c["cells"], temp=c["temp"], jitter=c["jitter"], seed=c["seed"])
    nm = c["neighmax"]
    xa, al, nl, nn = refpy.neighbor_list(cfg.x, cfg.box, p.rcut, SKIN, nm, neighcell=0)
    xa1, al1, nl1, nn1 = refpy.neighbor_list(cfg.x, cfg.box, p.rcut, SKIN, nm, neighcell=1)
    e, f, va = refpy.snap_force(xa, al, nl, nn, p, nblocks=8 * nthreads, nthreads=nthreads)
    atoms = np.arange(0, cfg.natoms, c["atom_stride"])
    th, x, v, ff, ee, nreb, snaps = ref_md(cfg.x, cfg.v, cfg.box, p, c["steps"], c["dt"], configs.TA_MASS,
                                           neighmax=nm, nthreads=nthreads, snap_steps=c["snap_steps"],
                                           snap_atoms=atoms)
    out = dict(cells=np.array(c["cells"]), twojmax=c["twojmax"], temp=c["temp"], jitter=c["jitter"],
               seed=c["seed"], coeff_seed=c["coeff_seed"], skin=SKIN, neighmax=nm, md_dt=c["dt"],
               md_steps=c["steps"], box=cfg.box, coeff=p.coeff,
               x_check=np.array([cfg.x.sum(), (cfg.x ** 2).sum()]), v_check=np.array([cfg.v.sum(), (cfg.v ** 2).sum()]),
               ghosts=xa.shape[0] - cfg.natoms, xall_check=np.array([xa.sum(), (xa ** 2).sum()]),
               alist_check=np.array([int(al.astype(np.int64).sum()), int((al.astype(np.int64) ** 2).sum())]),
               neighnum=nn.astype(np.int8), row_hash=row_hashes(nl, nn), cell_rows_equal=np.array(
                   [tuple(sorted(nl[i, :nn[i]])) == tuple(sorted(nl1[i, :nn1[i]])) for i in range(cfg.natoms)]).all(),
               e_check=np.array([e.sum(), (e ** 2).sum()]), f_check=np.array([f.sum(), (f ** 2).sum()]),
               v_virial_check=np.array([va.sum(), (va ** 2).sum()]),
               md_thermo=th, md_rebuilds=nreb, md_atoms=atoms)
    for st, (xs, vs) in snaps.items():
        out[f"md_x_{st}"] = xs
        out[f"md_v_{st}"] = vs
    path = os.path.join(HERE, f"{c['name']}.npz")
    np.savez_compressed(path, **out)
    print(c["name"], cfg.natoms, "atoms", nreb, "list builds", os.path.getsize(path), "bytes")


# quadratic SNAP fixtures (quadraticflag = 1; the reference evaluates the quadratic terms in its
# ComputePairSnap chain): (name, cells, 2J, temp, jitter, seed, coeff seed, flag overrides)
QUAD_CASES = [
    ("quad_bcc128_2j6", (4, 4, 4), 6, 600.0, 0.05, 18, 108, {}),
    ("quad_bcc250_2j8", (5, 5, 5), 8, 300.0, 0.08, 19, 109, {}),
    ("quad_bcc54_2j4_flags", (3, 3, 3), 4, 1000.0, 0.10, 20, 110, {"bnormflag": 1, "bzeroflag": 1}),
]


def quad_fixtures():
    """Quadratic SNAP: positions, the reference's neighbour list and its per-atom energy, forces and
    virial from the ComputePairSnap chain (cpuComputeBeta2 / cpuSnapTallyEnergyFull)."""
    for (name, cells, tj, temp, jit, seed, cseed, flags) in QUAD_CASES:
        p = configs.snap_params(tj, seed=cseed, quadraticflag=1, **flags)
        cfg = configs.ta_config(cells, temp=temp, jitter=jit, seed=seed)
        xa, al, nl, nn = refpy.neighbor_list(cfg.x, cfg.box, p.rcut, SKIN, NEIGHMAX, neighcell=0)
        e, f, va = refpy.snap_force_pairsnap(xa, al, nl, nn, p)
        path = os.path.join(HERE, f"{name}.npz")
        np.savez_compressed(path, cells=np.array(cells), twojmax=tj, temp=temp, jitter=jit, seed=seed,
                            coeff_seed=cseed, flags=np.array([p.bnormflag, p.bzeroflag, p.switchflag]),
                            quadraticflag=1, skin=SKIN, neighmax=NEIGHMAX, x=cfg.x, box=cfg.box, coeff=p.coeff,
                            xall=xa, alist=al, neighlist=nl, neighnum=nn, eatom=e, fatom=f, vatom=va)
        print(name, cfg.natoms, "atoms", os.path.getsize(path), "bytes")


# several element types: (name, cells, 2J, T, jitter, seed, coeff seed, radelems, wjelems, chemflag, flags)
CHEM_CASES = [
    ("chem_bcc128_2j6", (4, 4, 4), 6, 600.0, 0.05, 21, 111, (0.5, 0.45), (1.0, 0.8), 1, {}),
    ("chem_bcc250_2j8", (5, 5, 5), 8, 300.0, 0.06, 22, 112, (0.5, 0.47), (1.0, 0.9), 1, {}),
    ("chem_bcc54_2j4_3el_flags", (3, 3, 3), 4, 1000.0, 0.10, 23, 113, (0.5, 0.44, 0.48), (1.0, 0.7, 1.2), 1,
     {"bnormflag": 1, "bzeroflag": 1}),
    ("chem_bcc54_2j6_wselfall", (3, 3, 3), 6, 800.0, 0.08, 24, 114, (0.5, 0.46), (0.9, 1.1), 1,
     {"bzeroflag": 1, "wselfallflag": 1}),
    ("chem_bcc128_2j8_chemflag0", (4, 4, 4), 8, 600.0, 0.05, 25, 115, (0.5, 0.45), (1.0, 0.8), 0,
     {"bzeroflag": 1}),
]


def chem_fixtures():
    """Several element types (random types 1..nelements): positions, types, the reference's neighbour
    list and its per-atom energy, forces and virial from ComputePairSnap3 with InitSnap's per-element
    set-up (element blocks of U and Y with chemflag)."""
    for (name, cells, tj, temp, jit, seed, cseed, rad, wj, chem, flags) in CHEM_CASES:
        p = configs.snap_params_elements(tj, rad, wj, chemflag=chem, seed=cseed, **flags)
        cfg = configs.ta_config(cells, temp=temp, jitter=jit, seed=seed)
        types = np.random.default_rng(seed + 1000).integers(1, p.nelements + 1, cfg.natoms).astype(np.int32)
        xa, al, nl, nn = refpy.neighbor_list(cfg.x, cfg.box, p.rcut, SKIN, NEIGHMAX, neighcell=0)
        e, f, va = refpy.snap_force_me(xa, al, nl, nn, types, p)
        path = os.path.join(HERE, f"{name}.npz")
        np.savez_compressed(path, cells=np.array(cells), twojmax=tj, temp=temp, jitter=jit, seed=seed,
                            coeff_seed=cseed, chemflag=chem, radelems=np.array(rad), wjelems=np.array(wj),
                            flags=np.array([p.bnormflag, p.bzeroflag, p.switchflag, p.wselfallflag]),
                            skin=SKIN, neighmax=NEIGHMAX, x=cfg.x, box=cfg.box, types=types, coeff=p.coeff,
                            xall=xa, alist=al, neighlist=nl, neighnum=nn, eatom=e, fatom=f, vatom=va)
        print(name, cfg.natoms, "atoms", p.nelements, "elements", os.path.getsize(path), "bytes")


def main():
    from oracle.refroot import reference_root
    subprocess.check_call(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "ref", f"REFROOT={reference_root() or ''}"])
    if "--c2" in sys.argv:
        c2_fixture(os.cpu_count() or 1)
        return
    if "--quad" in sys.argv:
        quad_fixtures()
        return
    if "--chem" in sys.argv:
        chem_fixtures()
        return
    fit_fixtures()
    if "--fit-only" in sys.argv:
        return
    tri_fixtures()
    if "--tri-only" in sys.argv:
        return
    for (name, cells, tj, temp, jit, seed, cseed, flags, nsteps, dt) in CASES:
        p = configs.snap_params(tj, seed=cseed, **flags)
        cfg = configs.ta_config(cells, temp=temp, jitter=jit, seed=seed)
        xa0, al0, nl0, nn0 = refpy.neighbor_list(cfg.x, cfg.box, p.rcut, SKIN, NEIGHMAX, neighcell=0)
        xa1, al1, nl1, nn1 = refpy.neighbor_list(cfg.x, cfg.box, p.rcut, SKIN, NEIGHMAX, neighcell=1)
        e, f, va = refpy.snap_force(xa0, al0, nl0, nn0, p)
        out = dict(cells=np.array(cells), twojmax=tj, temp=temp, jitter=jit, seed=seed, coeff_seed=cseed,
                   flags=np.array([p.bnormflag, p.bzeroflag, p.switchflag]), skin=SKIN, neighmax=NEIGHMAX,
                   x=cfg.x, v=cfg.v, box=cfg.box, coeff=p.coeff,
                   xall=xa0, alist=al0, neighlist=nl0, neighnum=nn0,
                   neighlist_cell=nl1, neighnum_cell=nn1,
                   eatom=e, fatom=f, vatom=va)
        if nsteps:
            th, x, v, ff, ee, nreb = ref_md(cfg.x, cfg.v, cfg.box, p, nsteps, dt, configs.TA_MASS)
            out.update(md_dt=dt, md_steps=nsteps, md_thermo=th, md_x=x, md_v=v, md_f=ff, md_e=ee,
                       md_rebuilds=nreb)
        path = os.path.join(HERE, f"{name}.npz")
        np.savez_compressed(path, **out)
        print(name, cfg.natoms, "atoms", xa0.shape[0] - cfg.natoms, "ghosts", os.path.getsize(path), "bytes")


if __name__ == "__main__":
    main()

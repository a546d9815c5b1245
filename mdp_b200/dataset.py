"""Training data of MDP's SNAP fits and the weighted linear fit over it.

Readers:
  read_json          one file of MDP's JSON training format (readJSON.jl:8-165):
                     text before the first '{' is skipped, frames are
                     Dataset.Data[*] with NumAtoms, Lattice (cell vectors as
                     rows), Positions, Forces, Energy, Stress and AtomTypes
                     (mapped to 1-based indices of `species`; unknown types
                     keep type 1, as the reference does)
  read_json_folder   every file of a folder in name order, frames appended
                     (readJSONfromFolder.jl:8-190)
  read_extxyz        extended-XYZ files (readEXTXYZ.jl): per frame an atom
                     count, a comment line of key=value pairs (Lattice as
                     nine numbers, a, b, c in turn; energy; stress; pbc;
                     Properties=name:type:columns...) and one line per atom
                     with the Properties columns (species, pos, forces used)

Fit (fit_groups) follows MDP's fitting/snap/Ta/fitsnap.jl:107-159 with the
"lsq" method of linearfit2 (Optimization/linearfit.jl:355-470): each group of
frames (one data folder) carries an energy weight and a force weight that
multiply its rows (applyweight); energies are divided by the atom count when
normalize_energy is set; the normal equations of all groups are summed and
solved.  The rows are the batched GPU pipeline's (mdp_fit_run): per frame one
energy row [N, sum_i B_i] and one row per force component [0, d(sum B)/dx],
with the one-body column N standing in for the reference's "single"
descriptor.  Stress rows (emldescriptors.jl:199-259, the "energyforcestress"
loss) are six per frame: the GPU's virial descriptors bv times
1.6021765e6 / cell volume (eV/A^3 to bar, normalizestress), reordered as
snapcpp.jl:662 does, against the frame's stress in the order xx, yy, zz, yz,
xz, xy; being six rows of
1 + ncoeff numbers per frame, their outer products are added to the GPU's
normal equations on the host.  With `zbl` = (inner, outer, Z), the ZBL
reference potential of fitsnap.jl:81 is evaluated on the GPU
(mdp_fit_zbl) and its energy, forces and stress are subtracted from the
targets first (emldescriptors.jl:199-259: e - eref, f - fref, s - sref).

Cells narrower than the cutoff (the 2- and 4-atom Elastic / Volume cells)
are replicated along each short cell vector until every perpendicular width
exceeds the cutoff, which is what the batched pipeline's single image shell
needs; the copies reproduce every neighbour of the original cell, so each
atom's descriptors are unchanged.  A frame replicated m times enters with
its energy row per atom (the same row as the original) and its force rows
scaled by 1/sqrt(m), so it adds exactly what the original frame would.
"""
from __future__ import annotations

import dataclasses
import json
import os
import re

import numpy as np

from . import fit as _fit
from .configs import SnapParams


@dataclasses.dataclass
class Frame:
    natoms: int
    lattice: np.ndarray            # (3, 3) cell vectors as rows
    x: np.ndarray                  # (N, 3)
    e: float | None = None         # total energy (eV)
    f: np.ndarray | None = None    # (N, 3) forces (eV/A)
    stress: np.ndarray | None = None
    types: np.ndarray | None = None  # (N,) 1-based species index
    source: str = ""
    pbc: tuple = (True, True, True)  # periodic along a, b, c


def _frames_of(text: str, species, source: str):
    i1 = text.find("{")
    if i1 < 0:
        raise ValueError(f"{source}: no JSON object")
    data = json.loads(text[i1:])["Dataset"]["Data"]
    out = []
    for d in data:
        x = np.asarray(d["Positions"], dtype=np.float64).reshape(-1, 3)
        n = int(d.get("NumAtoms", x.shape[0]))
        if n != x.shape[0]:
            raise ValueError(f"{source}: NumAtoms {n} but {x.shape[0]} positions")
        lat = np.asarray(d["Lattice"], dtype=np.float64).reshape(3, 3)
        e = d.get("Energy")
        e = None if e is None else float(np.asarray(e, dtype=np.float64).ravel()[0])
        f = d.get("Forces")
        f = None if f is None else np.asarray(f, dtype=np.float64).reshape(n, 3)
        st = d.get("Stress")
        st = None if st is None else np.asarray(st, dtype=np.float64).reshape(3, 3)
        types = np.ones(n, dtype=np.int32)
        if "AtomTypes" in d:
            names = list(d["AtomTypes"])
            for k, s in enumerate(species):
                types[[i for i, t in enumerate(names) if t == s]] = k + 1
        out.append(Frame(natoms=n, lattice=lat, x=x, e=e, f=f, stress=st, types=types, source=source))
    return out


def read_json(path: str, species=("Ta",)) -> list[Frame]:
    """Frames of one JSON training file (readJSON.jl:8-165)."""
    with open(path) as fh:
        return _frames_of(fh.read(), species, path)


def read_json_folder(folder: str, species=("Ta",), extension: str = "json") -> list[Frame]:
    """Frames of every file of `folder` with the extension, in name order
    (readJSONfromFolder.jl:8-190 walks readdir, which sorts)."""
    return read_folder(folder, species, extension)


_KV = re.compile(r'([A-Za-z_][\w-]*)\s*=\s*("([^"]*)"|\S+)')


def _comment_fields(line: str) -> dict:
    return {m.group(1).lower(): (m.group(3) if m.group(3) is not None else m.group(2))
            for m in _KV.finditer(line)}


def read_extxyz(path: str, species=("Ta",)) -> list[Frame]:
    """Frames of one extended-XYZ file (readEXTXYZ.jl)."""
    with open(path) as fh:
        lines = [ln for ln in fh.read().splitlines()]
    out, m = [], 0
    while m < len(lines):
        if not lines[m].strip():
            m += 1
            continue
        n = int(lines[m].split()[0])
        kv = _comment_fields(lines[m + 1])
        if "lattice" not in kv or "properties" not in kv:
            raise ValueError(f"{path}: frame at line {m + 1} lacks Lattice or Properties")
        lat = np.array(kv["lattice"].split(), dtype=np.float64).reshape(3, 3)
        props = kv["properties"].split(":")
        if len(props) % 3:
            raise ValueError(f"{path}: bad Properties {kv['properties']}")
        if m + 2 + n > len(lines):
            raise ValueError(f"{path}: frame at line {m + 1} is truncated")
        rows = [lines[m + 2 + i].split() for i in range(n)]
        cols, c0 = {}, 0
        for k in range(0, len(props), 3):
            name, typ, width = props[k].lower(), props[k + 1].upper(), int(props[k + 2])
            cols[name] = (typ, [r[c0:c0 + width] for r in rows])
            c0 += width
        x = np.array(cols["pos"][1], dtype=np.float64).reshape(n, 3)
        f = np.array(cols["forces"][1], dtype=np.float64).reshape(n, 3) if "forces" in cols else None
        types = np.ones(n, dtype=np.int32)
        if "species" in cols:
            names = [r[0] for r in cols["species"][1]]
            for k, sp in enumerate(species):
                types[[i for i, t in enumerate(names) if t == sp]] = k + 1
        e = float(kv["energy"]) if "energy" in kv else None
        st = np.array(kv["stress"].split(), dtype=np.float64).reshape(3, 3) if "stress" in kv else None
        pbc = tuple(t.upper() in ("T", "TRUE", "1") for t in kv["pbc"].split()) if "pbc" in kv else (True,) * 3
        out.append(Frame(natoms=n, lattice=lat, x=x, e=e, f=f, stress=st, types=types, source=path, pbc=pbc))
        m += 2 + n
    return out


def reference_orientation(frame: Frame, transpose_lattice: bool = False) -> Frame:
    """The frame as MDP's training-data reader leaves it (readconfigfile.jl:28-58).

    With transpose_lattice (the `transposelattice` flag of adddata, which
    fitting/snap/Ta/fitsnap.jl sets) the cell vectors are the COLUMNS of the
    file's Lattice array.  The cell is then rotated to the standard
    orientation -- a along x, b in the xy plane (rotatelattice.jl) -- and the
    positions with it (transformcoords.jl: x = [a b c] [A B C]^-1 X).  Forces
    and stresses stay as read, as the reference leaves them.  For a file whose
    rows are already in that orientation the rotation is the identity.

    Files that store the cell vectors as rows (every frame of MDP's Ta set:
    the positions of its 2-atom BCC cells sit exactly at the body centre of the
    row cell) are distorted by the transposition wherever the cell has
    off-diagonal terms; the reference's published force errors of the Elastic
    folders come from exactly that distortion."""
    L = np.asarray(frame.lattice, dtype=np.float64)
    A, B, C = (L.T if transpose_lattice else L)
    An, Bn, Cn = np.linalg.norm(A), np.linalg.norm(B), np.linalg.norm(C)
    bx = B @ A / An
    by = np.sqrt(Bn * Bn - bx * bx)
    cx = C @ A / An
    cy = (B @ C - bx * cx) / by
    cz = np.sqrt(Cn * Cn - cx * cx - cy * cy)
    new = np.array([[An, 0.0, 0.0], [bx, by, 0.0], [cx, cy, cz]])
    R = new.T @ np.linalg.inv(np.stack([A, B, C]).T)
    return dataclasses.replace(frame, lattice=new, x=np.asarray(frame.x) @ R.T)


def read_folder(folder: str, species=("Ta",), extension: str = "json") -> list[Frame]:
    """Frames of every file of `folder` with the extension, in name order;
    "json" files go through read_json, "xyz" / "extxyz" through read_extxyz."""
    reader = read_json if extension == "json" else read_extxyz
    out = []
    for name in sorted(os.listdir(folder)):
        if name.endswith("." + extension):
            out.extend(reader(os.path.join(folder, name), species))
    if not out:
        raise ValueError(f"{folder}: no .{extension} files")
    return out


def cell_widths(lattice: np.ndarray) -> np.ndarray:
    """Perpendicular width of the cell across each of its vectors."""
    H = np.asarray(lattice, dtype=np.float64)
    vol = abs(np.linalg.det(H))
    return np.array([vol / np.linalg.norm(np.cross(H[(k + 1) % 3], H[(k + 2) % 3])) for k in range(3)])


def wrap(x: np.ndarray, lattice: np.ndarray) -> np.ndarray:
    """Positions mapped into the cell (fractional coordinates in [0, 1))."""
    H = np.asarray(lattice, dtype=np.float64)
    s = x @ np.linalg.inv(H)
    s -= np.floor(s)
    s[s >= 1.0] = 0.0
    return s @ H


def replicate(frame: Frame, rcut: float):
    """(FitConfig, copies): the frame's cell repeated along each vector until
    every perpendicular width exceeds rcut, the original atoms first."""
    H = np.asarray(frame.lattice, dtype=np.float64)
    reps = np.maximum(1, np.floor(rcut / cell_widths(H)).astype(int) + 1)
    x0 = wrap(frame.x, H)
    shifts = [i * H[0] + j * H[1] + k * H[2]
              for k in range(reps[2]) for j in range(reps[1]) for i in range(reps[0])]
    x = np.concatenate([x0 + s for s in shifts])
    big = H * reps[:, None]
    return _fit.FitConfig(x=x, box=big, kind=frame.source), int(np.prod(reps))


@dataclasses.dataclass
class Group:
    """One data folder: its frames and the weights of its energy, force and stress rows."""
    name: str
    frames: list
    we: float = 1.0
    wf: float = 1.0
    ws: float = 0.0


EV_PER_A3_IN_BAR = 1.6021765e6
# stress components of the rows, in emldescriptors.jl's order (ind = [1, 5, 9, 6, 3, 2]): xx, yy, zz, yz, xz, xy
VOIGT = ((0, 0), (1, 1), (2, 2), (1, 2), (0, 2), (0, 1))
# the virial descriptors bv come as xx, yy, zz, xy, xz, yz (cpuSnap virial tally); snapcpp.jl:662 reorders
# them to the stress order with bv[[1; 2; 3; 6; 5; 4], :]
BV_TO_VOIGT = (0, 1, 2, 5, 4, 3)


def stress_rows(bv: np.ndarray, cell: np.ndarray, copies: int, normalize_stress: bool = True) -> np.ndarray:
    """(6, 1 + k) stress rows of one frame from the virial descriptors bv
    (k, 6) of its (possibly replicated) cell; the one-body column is zero."""
    scale = EV_PER_A3_IN_BAR / abs(np.linalg.det(cell)) if normalize_stress else 1.0 / copies
    R = np.zeros((6, 1 + bv.shape[0]))
    R[:, 1:] = scale * bv.T[list(BV_TO_VOIGT)]
    return R


def batch_of(groups, rcut: float, normalize_energy: bool = True):
    """(configs, e, f, we, wf, copies, group index) for set_batch.  Every
    frame must be periodic along all three cell vectors."""
    cfgs, e, f, we, wf, copies, gid = [], [], [], [], [], [], []
    for g, grp in enumerate(groups):
        for fr in grp.frames:
            if not all(fr.pbc):
                raise ValueError(f"{fr.source or grp.name}: pbc {fr.pbc}; the batched fit needs periodic cells")
            cfg, m = replicate(fr, rcut)
            cfgs.append(cfg)
            copies.append(m)
            gid.append(g)
            e.append(m * (fr.e if fr.e is not None else 0.0))
            ff = fr.f if fr.f is not None else np.zeros((fr.natoms, 3))
            f.append(np.tile(ff, (m, 1)))
            # rows of data a frame does not carry get zero weight (emldescriptors.jl adds rows only for
            # energies / forces that are present)
            we.append(0.0 if fr.e is None else grp.we / (cfg.natoms if normalize_energy else m))
            wf.append(0.0 if fr.f is None else grp.wf / np.sqrt(m))
    return (cfgs, np.array(e), np.concatenate(f), np.array(we), np.array(wf), np.array(copies),
            np.array(gid))


def zbl_reference(cfgs, params: SnapParams, zbl, device: int = 0):
    """Per configuration: ZBL energy, forces (all atoms, concatenated) and
    summed virial (6,) in the order xx, yy, zz, xy, xz, yz."""
    bf = _fit.BatchFit(params, device)
    try:
        bf.set_batch(cfgs)
        ea, fa, va = bf.zbl(*zbl)
    finally:
        bf.close()
    a0 = np.concatenate([[0], np.cumsum([c.natoms for c in cfgs])])
    e = np.array([ea[a0[c]:a0[c + 1]].sum() for c in range(len(cfgs))])
    w = np.stack([va[:, a0[c]:a0[c + 1]].sum(axis=1) for c in range(len(cfgs))])
    return e, fa, w


def fit_groups(groups, params: SnapParams, normalize_energy: bool = True, normalize_stress: bool = True,
               mode: str = "fp64", device: int = 0, zbl=None):
    """Solve the weighted linear SNAP fit over the groups on the GPU.

    Returns beta (1 + ncoeff: the one-body term, then the bispectrum
    coefficients), the normal equations, and per group the unweighted energy
    (per atom), force and stress MAE / RMSE of the fitted model, as
    validate2 reports them (maespace.jl:210)."""
    rcut = max(params.rcut, zbl[1]) if zbl is not None else params.rcut
    cfgs, e, f, we, wf, copies, gid = batch_of(groups, rcut, normalize_energy)
    sref = [np.zeros(6)] * len(cfgs)
    if zbl is not None:
        ez, fz, wz = zbl_reference(cfgs, params, zbl, device)
        e = e - ez
        f = f - fz
        for c, cfg in enumerate(cfgs):
            scale = EV_PER_A3_IN_BAR / abs(np.linalg.det(cfg.box)) if normalize_stress else 1.0 / copies[c]
            sref[c] = scale * wz[c][list(BV_TO_VOIGT)]
    bf = _fit.BatchFit(params, device)
    try:
        bf.set_batch(cfgs, e, f, we, wf)
        A, b, ms = bf.run(mode)
        bi, bd, bv, _ = bf.descriptors()
    finally:
        bf.close()
    frames = [fr for grp in groups for fr in grp.frames]
    srows = [None] * len(cfgs)
    for c, fr in enumerate(frames):
        if fr.stress is None:
            continue
        srows[c] = stress_rows(bv[c], cfgs[c].box, copies[c], normalize_stress)
        ws = groups[gid[c]].ws
        if ws:
            t = np.array([fr.stress[i, j] for i, j in VOIGT]) - sref[c]
            A = A + ws * ws * (srows[c].T @ srows[c])
            b = b + ws * ws * (srows[c].T @ t)
    try:
        beta = _fit.solve(A, b)
    except np.linalg.LinAlgError:
        beta = np.linalg.lstsq(A, b, rcond=None)[0]
    counts = np.array([c.natoms for c in cfgs])
    a0 = np.concatenate([[0], np.cumsum(counts)])
    e_pred = beta[0] * counts + bi @ beta[1:]
    errors = []
    for g, grp in enumerate(groups):
        de, dfs, dss = [], [], []
        for c in np.nonzero(gid == g)[0]:
            n0 = counts[c] // copies[c]
            if frames[c].e is not None:
                de.append((e_pred[c] - e[c]) / counts[c])
            if frames[c].f is not None:
                fp = bd[a0[c]:a0[c] + n0] @ beta[1:]
                dfs.append((fp - f[a0[c]:a0[c] + n0]).ravel())
            if srows[c] is not None:
                dss.append(srows[c] @ beta + sref[c] - np.array([frames[c].stress[i, j] for i, j in VOIGT]))
        err = dict(group=grp.name, frames=int((gid == g).sum()))
        if de:
            de = np.array(de)
            err.update(energy_mae=float(np.abs(de).mean()), energy_rmse=float(np.sqrt((de ** 2).mean())))
        if dfs:
            dfs = np.concatenate(dfs)
            err.update(force_mae=float(np.abs(dfs).mean()), force_rmse=float(np.sqrt((dfs ** 2).mean())))
        if dss:
            dss = np.concatenate(dss)
            err.update(stress_mae=float(np.abs(dss).mean()), stress_rmse=float(np.sqrt((dss ** 2).mean())))
        errors.append(err)
    return dict(beta=beta, A=A, b=b, graph_ms=ms, errors=errors, configs=len(cfgs),
                atoms=int(counts.sum()), replicated=int((copies > 1).sum()))

"""Batched SNAP descriptors and the linear-fit normal equations on the GPU.

Per configuration this computes what MDP's ComputeSnap computes
(snappotential.cpp:762-910): the summed bispectrum bi, its derivatives bd with
respect to every atom coordinate and the virial bv; over a whole batch it
assembles the normal equations of the linear SNAP fit with the rows of
Regression.cpp:386-404 (one total-energy row per configuration, one row per
force component) in FP64 or from a BF16 hi/lo split with FP32 tensor-core sums.
The whole device pipeline is one CUDA graph (mdp_fit_run).

The synthetic batch (batch_configs) is the fitting workload of the project:
BCC / FCC / A15 Ta supercells of 16-512 atoms at equal volume per atom, with
isotropic strain within +-5 % and Gaussian jitter of width U[0.02, 0.3] A; every
box length is at least rcut + skin = 5.68 A, the single image shell MDP's
cpuPeriodicImages3D builds.
"""
from __future__ import annotations

import ctypes as C
import dataclasses

import numpy as np

from . import _lib
from .configs import SnapParams, TA_LATTICE, _BASIS

# lattice constants at the BCC volume per atom (a^3 / 2 with a = 3.316 A)
LATTICE = {"bcc": TA_LATTICE, "fcc": (4 * TA_LATTICE ** 3 / 2) ** (1 / 3), "a15": (8 * TA_LATTICE ** 3 / 2) ** (1 / 3)}
MIN_WIDTH = 4.67637 + 1.0


@dataclasses.dataclass
class FitConfig:
    x: np.ndarray      # (N, 3) inside the cell
    box: np.ndarray    # (3,) edge lengths of an orthogonal cell, or (3, 3) cell vectors a, b, c as rows
    kind: str

    @property
    def natoms(self):
        return self.x.shape[0]


def supercell(kind: str, target: int, strain: float):
    """Cells (n1, n2, n3), each >= the count that keeps the strained width above
    MIN_WIDTH, whose atom count is nearest to target."""
    m = len(_BASIS[kind])
    a = LATTICE[kind] * (1.0 + strain)
    nmin = int(np.ceil(MIN_WIDTH / a))
    best = None
    for n1 in range(nmin, 9):
        for n2 in range(n1, 9):
            for n3 in range(n2, 9):
                d = abs(m * n1 * n2 * n3 - target)
                if best is None or d < best[0]:
                    best = (d, (n1, n2, n3))
    return best[1], a


def make_config(kind: str, target: int, strain: float, sigma: float, rng) -> FitConfig:
    (n1, n2, n3), a = supercell(kind, target, strain)
    basis = _BASIS[kind]
    ii, jj, kk = np.meshgrid(np.arange(n1), np.arange(n2), np.arange(n3), indexing="ij")
    cells = np.stack([ii.ravel(), jj.ravel(), kk.ravel()], axis=1).astype(np.float64)
    x = ((cells[:, None, :] + basis[None, :, :]).reshape(-1, 3)) * a
    box = np.array([n1 * a, n2 * a, n3 * a])
    x = x + rng.normal(0.0, sigma, size=x.shape)
    x = np.mod(x, box)
    x = np.where(x >= box, x - box, x)
    return FitConfig(x=x, box=box, kind=kind)


def batch_configs(nconf: int = 4096, seed: int = 2024, lo: int = 16, hi: int = 512):
    """The synthetic fitting batch: kinds, sizes, strains and jitters drawn from
    seeded distributions; targets y ~ N(0, 1) for every energy and force row."""
    rng = np.random.default_rng(seed)
    cfgs = []
    for _ in range(nconf):
        kind = ("bcc", "fcc", "a15")[rng.integers(3)]
        target = int(rng.integers(lo, hi + 1))
        cfgs.append(make_config(kind, target, rng.uniform(-0.05, 0.05), rng.uniform(0.02, 0.3), rng))
    e = rng.normal(size=nconf)
    f = rng.normal(size=(sum(c.natoms for c in cfgs), 3))
    return cfgs, e, f


def cell_vectors(box) -> np.ndarray:
    """(3, 3) cell vectors as rows, from edge lengths (3,) or vectors (3, 3)."""
    b = np.asarray(box, dtype=np.float64)
    return np.diag(b) if b.shape == (3,) else b.reshape(3, 3)


class BatchFit:
    """Device state of one batch (ctypes handle over mdp_fit_*)."""

    def __init__(self, params: SnapParams, device: int = 0):
        L = _lib.lib()
        self.params = params
        self._sp, self._keep = _lib.snap_params_c(params)
        self._h = C.c_void_p()
        _lib.check(L.mdp_fit_create(C.byref(self._h), C.byref(self._sp), device), "mdp_fit_create")
        self.ncoeff = L.mdp_fit_ncoeff(self._h)
        self.nconf = 0
        self.natoms = 0

    def close(self):
        if self._h:
            _lib.lib().mdp_fit_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_batch(self, cfgs, e=None, f=None, we=None, wf=None):
        n = np.array([c.natoms for c in cfgs], dtype=np.int32)
        x = np.ascontiguousarray(np.concatenate([c.x for c in cfgs]), dtype=np.float64)
        keep = [None if a is None else np.ascontiguousarray(a, dtype=np.float64) for a in (e, f, we, wf)]
        ptr = [None if a is None else a.ctypes.data for a in keep]
        if all(np.shape(c.box) == (3,) for c in cfgs):
            box = np.ascontiguousarray(np.stack([c.box for c in cfgs]), dtype=np.float64)
            _lib.check(_lib.lib().mdp_fit_set_batch(self._h, len(cfgs), n, box, x, *ptr), "mdp_fit_set_batch")
        else:
            lat = np.ascontiguousarray(np.stack([cell_vectors(c.box) for c in cfgs]), dtype=np.float64)
            _lib.check(_lib.lib().mdp_fit_set_batch_lattice(self._h, len(cfgs), n, lat, x, *ptr),
                       "mdp_fit_set_batch_lattice")
        self.nconf, self.natoms = len(cfgs), int(n.sum())
        self.counts = n

    def set_chunk_bytes(self, nbytes: float):
        _lib.check(_lib.lib().mdp_fit_set_chunk_bytes(self._h, float(nbytes)), "mdp_fit_set_chunk_bytes")

    def nchunks(self) -> int:
        return int(_lib.lib().mdp_fit_nchunks(self._h))

    def npairs(self) -> int:
        return int(_lib.lib().mdp_fit_npairs(self._h))

    def descriptors(self):
        """bi (nconf, k), bd (natoms, 3, k) in the reference's sign, bv (nconf, k, 6), blist (k, natoms)."""
        k = self.ncoeff
        bi = np.zeros((self.nconf, k)); bd = np.zeros((self.natoms, 3, k))
        bv = np.zeros((self.nconf, k, 6)); bl = np.zeros((k, self.natoms))
        _lib.check(_lib.lib().mdp_fit_descriptors(self._h, bi.ctypes.data, bd.ctypes.data, bv.ctypes.data,
                                                  bl.ctypes.data), "mdp_fit_descriptors")
        return bi, bd, bv, bl

    def zbl(self, inner: float = 4.0, outer: float = 4.8, z: float = 73.0):
        """ZBL reference potential of every atom: energy (natoms,), forces
        (natoms, 3), virial (6, natoms) in the order xx, yy, zz, xy, xz, yz."""
        e = np.zeros(self.natoms); f = np.zeros((self.natoms, 3)); v = np.zeros((6, self.natoms))
        _lib.check(_lib.lib().mdp_fit_zbl(self._h, float(inner), float(outer), float(z), e, f, v), "mdp_fit_zbl")
        return e, f, v

    def run(self, mode: str = "fp64"):
        """Normal equations (A (m, m), b (m,), device ms) with m = 1 + ncoeff."""
        A = np.zeros(64 * 64); b = np.zeros(64); ms = C.c_float(0.0)
        _lib.check(_lib.lib().mdp_fit_run(self._h, {"fp64": 0, "bf16": 1}[mode], A, b, C.byref(ms)), "mdp_fit_run")
        m = 1 + self.ncoeff
        return A.reshape(64, 64)[:m, :m].copy(), b[:m].copy(), float(ms.value)

    def tune(self):
        out = np.zeros(3, dtype=np.int32)
        _lib.check(_lib.lib().mdp_fit_tune(self._h, out), "mdp_fit_tune")
        return dict(du_threads=int(out[0]), dbdr_threads=int(out[1]), gram_rows=int(out[2]))


def solve(A: np.ndarray, b: np.ndarray) -> np.ndarray:
    """beta of A beta = b by Cholesky in FP64 (Regression.cpp:420-426 inverts A)."""
    L = np.linalg.cholesky(A)
    y = np.linalg.solve(L, b)
    return np.linalg.solve(L.T, y)


def rows_numpy(cfgs, bi, bd, e, f, we=None, wf=None):
    """The same rows in numpy (test reference): R, t."""
    nc = len(cfgs)
    k = bi.shape[1]
    we = np.ones(nc) if we is None else we
    wf = np.ones(nc) if wf is None else wf
    n = np.array([c.natoms for c in cfgs])
    R = np.zeros((nc + 3 * n.sum(), 1 + k))
    t = np.zeros(R.shape[0])
    R[:nc, 0] = we * n
    R[:nc, 1:] = we[:, None] * bi
    t[:nc] = we * e
    a0 = np.concatenate([[0], np.cumsum(n)])
    for c in range(nc):
        G = -bd[a0[c]:a0[c + 1]]                  # (n, 3, k): d(sum B)/dx
        rows = slice(nc + 3 * a0[c], nc + 3 * a0[c + 1])
        R[rows, 1:] = wf[c] * G.reshape(-1, k)
        t[rows] = -wf[c] * f[a0[c]:a0[c + 1]].reshape(-1)
    return R, t


def benchmark(nconf: int = 4096, seed: int = 2024, coeff_seed: int = 2024, device: int = 0, log=print,
              rank: int = 0, world: int = 1) -> dict:
    """The batched-fitting workload end to end: batch set-up (positions to the
    device, pair lists), autotuning, then one graph launch per assembly mode
    (timed with CUDA events), and the FP64 vs BF16-split solutions.  With
    world > 1 (torch.distributed initialised) every rank takes an atom-balanced
    share of the configurations and one all-reduce sums A and b; times are the
    maximum over ranks."""
    import time
    from . import parallel
    from .configs import snap_params
    cfgs, e, f = batch_configs(nconf, seed=seed)
    counts = np.array([c.natoms for c in cfgs])
    lo, hi = parallel.shard_bounds(counts, rank, world) if world > 1 else (0, nconf)
    a0 = np.concatenate([[0], np.cumsum(counts)])
    p = snap_params(8, seed=coeff_seed)
    bf = BatchFit(p, device=device)
    t0 = time.perf_counter()
    bf.set_batch(cfgs[lo:hi], e[lo:hi], f[a0[lo]:a0[hi]])
    t_set = time.perf_counter() - t0
    tuned = bf.tune()
    out = {"configs": nconf, "atoms": int(counts.sum()), "ranks": world, "pairs_rank0": bf.npairs(),
           "chunks_rank0": bf.nchunks(), "rows": nconf + 3 * int(counts.sum()), "batch_setup_s": t_set,
           "tuned": tuned}
    dev = None
    if world > 1:
        import torch
        dev = torch.device("cuda", device)
    sol = {}
    for mode in ("fp64", "bf16"):
        bf.run(mode)                       # capture and warm
        A, b, ms = bf.run(mode)            # one graph launch
        if world > 1:
            A, b = parallel.allreduce_sum(A, b, device=dev)
            ms = parallel.max_over_ranks(ms, device=dev)
        out[f"graph_ms_{mode}"] = ms
        sol[mode] = (A, b)
    A64, b64 = sol["fp64"]
    A16, b16 = sol["bf16"]
    beta64 = np.linalg.solve(A64, b64)
    beta16 = np.linalg.solve(A16, b16)
    out["A_rel_err_bf16"] = float(np.linalg.norm(A16 - A64) / np.linalg.norm(A64))
    out["b_rel_err_bf16"] = float(np.linalg.norm(b16 - b64) / np.linalg.norm(b64))
    out["beta_rel_err_bf16"] = float(np.linalg.norm(beta16 - beta64) / np.linalg.norm(beta64))
    out["cond_A"] = float(np.linalg.cond(A64))
    dg = 1.0 / np.sqrt(np.diag(A64))
    out["cond_A_equilibrated"] = float(np.linalg.cond(A64 * dg[:, None] * dg[None, :]))
    out["configs_per_s_fp64"] = nconf / (out["graph_ms_fp64"] * 1e-3)
    out["atoms_per_s_fp64"] = out["atoms"] / (out["graph_ms_fp64"] * 1e-3)
    bf.close()
    log(out)
    return out


if __name__ == "__main__":
    import argparse
    import json
    ap = argparse.ArgumentParser(description="batched SNAP descriptors + normal equations benchmark")
    ap.add_argument("--configs", type=int, default=4096)
    a = ap.parse_args()
    print(json.dumps(benchmark(a.configs, log=lambda m: None), indent=1))

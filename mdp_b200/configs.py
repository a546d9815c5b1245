"""Synthetic BCC/FCC/A15 tantalum configurations and SNAP parameter sets.

The workloads are seeded and fully synthetic: a lattice of Ta atoms
(a = 3.316 A, mass 180.88 amu, metal units) with Gaussian position jitter,
Maxwell-Boltzmann velocities with the centre-of-mass drift removed, and SNAP
coefficients beta_k ~ N(0, 0.01) with beta_0 = -11.7 eV.  SNAP hyper-parameters
follow the Ta example of MDP (simulating/snap/snapTA06A.jl:39-57): rcutfac
4.67637, element radius 0.5, rfac0 0.99363, rmin0 0, switching on, weight 1.

Unit constants are MDP's metal units (src/C++/Configuration/setunits.cpp:51-59).
"""
from __future__ import annotations

import dataclasses
import numpy as np

# metal units, setunits.cpp:51-59
BOLTZ = 8.617343e-5
MVV2E = 1.0364269e-4
FTM2V = 1.0 / 1.0364269e-4
NKTV2P = 1.6021765e6

TA_MASS = 180.88
TA_LATTICE = 3.316


@dataclasses.dataclass
class SnapParams:
    """SNAP hyper-parameters (the snaparam[12] vector of MDP, Preprocessing.jl:266)."""
    twojmax: int = 8
    rcutfac: float = 4.67637
    rfac0: float = 0.99363
    rmin0: float = 0.0
    radelem: float = 0.5
    wjelem: float = 1.0
    switchflag: int = 1
    bzeroflag: int = 0
    bnormflag: int = 0
    wselfallflag: int = 0
    quadraticflag: int = 0
    chemflag: int = 0
    coeff: np.ndarray = None  # nelements x ncoeffall values; coeff[e * ncoeffall] = beta_0 of element e
    # several elements (types 1..nelements): per-element radius and weight;
    # None for the single element of radelem / wjelem
    radelems: tuple = None
    wjelems: tuple = None

    @property
    def nelements(self) -> int:
        return len(self.radelems) if self.radelems else 1

    @property
    def rcut(self) -> float:
        """The largest pair cutoff, 2 max(radelem) rcutfac (InitSnap's rcutmax)."""
        r = max(self.radelems) if self.radelems else self.radelem
        return 2.0 * r * self.rcutfac

    @property
    def ncoeff(self) -> int:
        """Linear coefficients per element: the bispectrum components, once
        per element triple with chemflag."""
        return idxb_count(self.twojmax) * (self.nelements ** 3 if self.chemflag else 1)

    @property
    def ncoeffall(self) -> int:
        """1 + ncoeff linear coefficients, plus the ncoeff (ncoeff + 1) / 2
        quadratic ones (upper triangle, row by row) when quadraticflag is set."""
        n = self.ncoeff
        return n + 1 + (n * (n + 1) // 2 if self.quadraticflag else 0)


def idxb_count(twojmax: int) -> int:
    n = 0
    for j1 in range(twojmax + 1):
        for j2 in range(j1 + 1):
            for j in range(j1 - j2, min(twojmax, j1 + j2) + 1, 2):
                if j >= j1:
                    n += 1
    return n


def seeded_coeff(twojmax: int, seed: int, beta0: float = -11.7, sigma: float = 0.01) -> np.ndarray:
    rng = np.random.default_rng(seed)
    n = idxb_count(twojmax)
    c = np.empty(n + 1)
    c[0] = beta0
    c[1:] = rng.normal(0.0, sigma, n)
    return c


def snap_params(twojmax: int = 8, seed: int = 1234, qsigma: float = 1e-5, **kw) -> SnapParams:
    """Seeded parameters; with quadraticflag=1 the quadratic coefficients are
    drawn N(0, qsigma) after the linear ones (1e-5 moves the 2J=8 Ta forces
    by about a tenth of their size)."""
    p = SnapParams(twojmax=twojmax, **kw)
    c = seeded_coeff(twojmax, seed)
    if p.quadraticflag:
        n = p.ncoeff
        q = np.random.default_rng(seed + 7919).normal(0.0, qsigma, n * (n + 1) // 2)
        c = np.concatenate([c, q])
    p.coeff = c
    return p


def snap_params_elements(twojmax: int, radelems, wjelems, chemflag: int = 1, seed: int = 1234,
                         sigma: float = 0.01, **kw) -> SnapParams:
    """Seeded parameters for len(radelems) element types: per element beta_0
    = -11.7 eV plus a seeded offset and N(0, sigma / sqrt(number of element
    triples)) linear coefficients, laid out element after element."""
    p = SnapParams(twojmax=twojmax, chemflag=chemflag, radelems=tuple(float(r) for r in radelems),
                   wjelems=tuple(float(w) for w in wjelems), **kw)
    rng = np.random.default_rng(seed)
    ntri = p.nelements ** 3 if chemflag else 1
    blocks = []
    for _ in range(p.nelements):
        b = np.empty(p.ncoeffall)
        b[0] = -11.7 + rng.normal(0.0, 0.5)
        b[1:] = rng.normal(0.0, sigma / np.sqrt(ntri), p.ncoeff)
        blocks.append(b)
    p.coeff = np.concatenate(blocks)
    return p


_BASIS = {
    "bcc": np.array([[0.0, 0.0, 0.0], [0.5, 0.5, 0.5]]),
    "fcc": np.array([[0.0, 0.0, 0.0], [0.5, 0.5, 0.0], [0.5, 0.0, 0.5], [0.0, 0.5, 0.5]]),
    "a15": np.array([[0.0, 0.0, 0.0], [0.5, 0.5, 0.5],
                     [0.25, 0.5, 0.0], [0.75, 0.5, 0.0],
                     [0.0, 0.25, 0.5], [0.0, 0.75, 0.5],
                     [0.5, 0.0, 0.25], [0.5, 0.0, 0.75]]),
}


@dataclasses.dataclass
class Config:
    """One periodic configuration: orthogonal box [0, L) per axis."""
    x: np.ndarray       # (N, 3) float64 positions
    v: np.ndarray       # (N, 3) float64 velocities (A/ps)
    box: np.ndarray     # (3,) box lengths; box vectors a=(Lx,0,0), b=(0,Ly,0), c=(0,0,Lz)
    mass: float = TA_MASS

    @property
    def natoms(self) -> int:
        return self.x.shape[0]


def lattice(ncell, kind: str = "bcc", a: float = TA_LATTICE):
    """Perfect lattice positions with cells ordered x fastest, then y, then z."""
    nx, ny, nz = ncell
    basis = _BASIS[kind]
    ii, jj, kk = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    cells = np.stack([ii.ravel(order="F"), jj.ravel(order="F"), kk.ravel(order="F")], axis=1).astype(np.float64)
    x = (cells[:, None, :] + basis[None, :, :]).reshape(-1, 3) * a
    box = np.array([nx * a, ny * a, nz * a], dtype=np.float64)
    return x, box


def maxwell_velocities(n: int, temp: float, mass: float, rng) -> np.ndarray:
    """Maxwell-Boltzmann velocities in A/ps at `temp` K, COM drift removed,
    rescaled so the kinetic temperature (3(N-1) dof, Calculation.cpp:436-467)
    equals `temp` exactly."""
    if temp <= 0.0 or n < 2:
        return np.zeros((n, 3))
    sigma = np.sqrt(BOLTZ * temp / (mass * MVV2E))
    v = rng.normal(0.0, sigma, (n, 3))
    v -= v.mean(axis=0)
    t_now = MVV2E * mass * np.sum(v * v) / (3.0 * (n - 1) * BOLTZ)
    v *= np.sqrt(temp / t_now)
    return v


def ta_config(ncell, temp: float = 300.0, jitter: float = 0.05, seed: int = 0,
              kind: str = "bcc", a: float = TA_LATTICE, strain: float = 0.0) -> Config:
    rng = np.random.default_rng(seed)
    x, box = lattice(ncell, kind, a * (1.0 + strain))
    if jitter > 0:
        x = x + rng.normal(0.0, jitter, x.shape)
    x = np.mod(x, box)                      # wrap into [0, L)
    x = np.where(x >= box, x - box, x)      # np.mod can round up to L
    v = maxwell_velocities(x.shape[0], temp, TA_MASS, rng)
    return Config(x=np.ascontiguousarray(x), v=np.ascontiguousarray(v), box=box)

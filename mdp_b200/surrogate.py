"""Learned surrogate of the SNAP energy (no counterpart in MDP).

An MLP 14 -> 64 -> 64 -> 1 with SiLU activations maps the per-atom 2J=4
bispectrum (14 components) to the per-atom energy.  It is trained on the GPU by
the library's own kernels (forward with BF16-rounded weights, FP32 sums and
gradients, Adam on FP32 master weights) on per-atom energies produced by the
plain 2J=8 SNAP model in MD snapshots.  In MD its forces come from the chain
rule dE/dr = sum_i (dE_i/dB_i) . dB_i/dr, computed as a linear-SNAP force with
per-atom coefficients; the plain model judges it every judge_every steps and
takes over when the force RMSE exceeds the tolerance.
"""
from __future__ import annotations

import ctypes as C
import dataclasses

import numpy as np

from . import _lib
from .configs import SnapParams, snap_params, ta_config, TA_MASS

NK, KP, H = 14, 16, 64
OFF_W1 = 0
OFF_B1 = OFF_W1 + H * KP
OFF_W2 = OFF_B1 + H
OFF_B2 = OFF_W2 + H * H
OFF_W3 = OFF_B2 + H
OFF_B3 = OFF_W3 + H
NPAR = OFF_B3 + 1


def unpack(P: np.ndarray) -> dict:
    """Flat parameter vector -> named arrays (W1 [H][KP], W2 [out][in], ...)."""
    return dict(W1=P[OFF_W1:OFF_B1].reshape(H, KP), b1=P[OFF_B1:OFF_W2], W2=P[OFF_W2:OFF_B2].reshape(H, H),
                b2=P[OFF_B2:OFF_W3], w3=P[OFF_W3:OFF_B3], b3=P[OFF_B3:OFF_B3 + 1])


def init_params(seed: int) -> np.ndarray:
    """Glorot-uniform weights (feature padding columns 14, 15 zero), zero biases."""
    rng = np.random.default_rng(seed)
    P = np.zeros(NPAR, dtype=np.float32)
    d = unpack(P)
    a1 = np.sqrt(6.0 / (NK + H))
    d["W1"][:, :NK] = rng.uniform(-a1, a1, size=(H, NK))
    a2 = np.sqrt(6.0 / (H + H))
    d["W2"][:] = rng.uniform(-a2, a2, size=(H, H))
    a3 = np.sqrt(6.0 / (H + 1))
    d["w3"][:] = rng.uniform(-a3, a3, size=H)
    return P


class Surrogate:
    """Device-resident MLP surrogate: parameters, training set and kernels."""

    def __init__(self, params4: SnapParams | None = None, device: int = 0):
        if params4 is None:
            params4 = snap_params(4, seed=0)
        if params4.twojmax != 4:
            raise ValueError("surrogate features are the 2J=4 bispectrum")
        L = _lib.lib()
        self.params4 = params4
        self._sp, self._keep = _lib.snap_params_c(params4)
        self._h = C.c_void_p()
        _lib.check(L.mdp_sur_create(C.byref(self._h), C.byref(self._sp), device), "mdp_sur_create")
        assert L.mdp_sur_nparams() == NPAR

    @property
    def handle(self):
        return self._h

    def close(self):
        if self._h:
            _lib.lib().mdp_sur_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- parameters -----------------------------------------------------------------
    def set_params(self, P: np.ndarray, norm: np.ndarray | None = None):
        P = np.ascontiguousarray(P, dtype=np.float32)
        nv = None if norm is None else np.ascontiguousarray(norm, dtype=np.float32)
        _lib.check(_lib.lib().mdp_sur_set_params(self._h, P, None if nv is None else nv.ctypes.data),
                   "mdp_sur_set_params")
        self._norm_keep = nv

    def params(self):
        P = np.zeros(NPAR, dtype=np.float32)
        norm = np.zeros(2 * NK + 2, dtype=np.float32)
        _lib.check(_lib.lib().mdp_sur_get_params(self._h, P, norm), "mdp_sur_get_params")
        return P, norm

    def save(self, path: str):
        P, norm = self.params()
        np.savez(path, params=P, norm=norm)

    def load(self, path: str):
        d = np.load(path)
        self.set_params(d["params"], d["norm"])

    # -- training set -----------------------------------------------------------------
    def reserve(self, rows: int):
        _lib.check(_lib.lib().mdp_sur_dataset_reserve(self._h, int(rows)), "mdp_sur_dataset_reserve")

    def size(self) -> int:
        return int(_lib.lib().mdp_sur_dataset_size(self._h))

    def load_dataset(self, X: np.ndarray, E: np.ndarray):
        Xp = np.zeros((X.shape[0], KP), dtype=np.float32)
        Xp[:, :NK] = X[:, :NK]
        _lib.check(_lib.lib().mdp_sur_dataset_load(self._h, Xp, np.ascontiguousarray(E, dtype=np.float32),
                                                   X.shape[0]), "mdp_sur_dataset_load")

    def dataset(self, row0: int = 0, n: int | None = None):
        n = self.size() - row0 if n is None else n
        X = np.zeros((n, KP), dtype=np.float32)
        E = np.zeros(n, dtype=np.float32)
        _lib.check(_lib.lib().mdp_sur_dataset_copy(self._h, X.ctypes.data, E.ctypes.data, row0, n),
                   "mdp_sur_dataset_copy")
        return X[:, :NK], E

    def sample(self, md) -> None:
        """Append md's current per-atom features and energies to the training set."""
        _lib.check(_lib.lib().mdp_md_sur_sample(md._h, self._h), "mdp_md_sur_sample")

    def fit_normalization(self):
        _lib.check(_lib.lib().mdp_sur_fit_normalization(self._h), "mdp_sur_fit_normalization")

    # -- kernels ------------------------------------------------------------------------
    def train(self, steps: int, batch: int = 4096, lr: float = 1e-3, seed: int = 0) -> np.ndarray:
        loss = np.zeros(steps, dtype=np.float32)
        _lib.check(_lib.lib().mdp_sur_train(self._h, int(steps), int(batch), float(lr), int(seed), loss),
                   "mdp_sur_train")
        return loss

    def grad(self, X: np.ndarray, E: np.ndarray):
        """Loss gradient over the given rows at the current parameters (no update)."""
        Xp = np.zeros((X.shape[0], KP), dtype=np.float32)
        Xp[:, :NK] = X[:, :NK]
        g = np.zeros(NPAR, dtype=np.float32)
        loss = C.c_float(0.0)
        _lib.check(_lib.lib().mdp_sur_grad(self._h, Xp, np.ascontiguousarray(E, dtype=np.float32), X.shape[0], g,
                                           C.byref(loss)), "mdp_sur_grad")
        return g, float(loss.value)

    def eval(self, B: np.ndarray):
        """B (n, 14) features -> per-atom energies (n,), dE_i/dB_i (n, 14)."""
        n = B.shape[0]
        Bt = np.ascontiguousarray(B[:, :NK].T, dtype=np.float64)
        E = np.zeros(n)
        G = np.zeros((NK, n), dtype=np.float32)
        _lib.check(_lib.lib().mdp_sur_eval(self._h, Bt, n, E, G), "mdp_sur_eval")
        return E, G.T.copy()


def features(md, sur: Surrogate) -> np.ndarray:
    """Per-atom 2J=4 bispectrum (natoms, 14) of md's current positions."""
    B = np.zeros(NK * md.natoms)
    _lib.check(_lib.lib().mdp_md_sur_features(md._h, sur.handle, B), "mdp_md_sur_features")
    return B.reshape(NK, md.natoms).T.copy()


@dataclasses.dataclass
class TrainingSet:
    temps: tuple = (300.0, 600.0, 1000.0, 1500.0, 2000.0, 3000.0)
    snapshots: int = 20000          # total, split evenly over the temperatures
    cells: tuple = (10, 10, 10)     # 2,000 BCC atoms
    every: int = 10                 # MD steps between snapshots
    equilibrate: int = 50
    dt: float = 0.001
    seed: int = 7


def generate(sur: Surrogate, p8: SnapParams, ts: TrainingSet, precision: str = "fp64", device: int = 0) -> int:
    """Runs plain 2J=8 SNAP MD at each temperature and appends snapshots to sur's set."""
    from .snap import SnapMD
    per = max(1, ts.snapshots // len(ts.temps))
    natoms = 2 * int(np.prod(ts.cells))
    sur.reserve(per * len(ts.temps) * natoms)
    for it, T in enumerate(ts.temps):
        # displacement scale grows with temperature so hot snapshots start disordered
        cfg = ta_config(ts.cells, temp=T, jitter=0.05 * np.sqrt(T / 300.0), seed=ts.seed + it)
        md = SnapMD(p8, cfg.box, cfg.natoms, ts.dt, mass=TA_MASS, precision=precision, device=device)
        md.set_state(cfg.x, cfg.v)
        md.setup()
        md.run(ts.equilibrate)
        for _ in range(per):
            md.run(ts.every)
            sur.sample(md)
        md.close()
    return sur.size()

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


def _force_methods():
    """Force-matching methods of Surrogate (kept together for readability)."""

    def force_set(self, snapshots, forces, energies, per: int):
        """snapshots: a fit.BatchFit at 2J=4 holding equal-size snapshots (per atoms);
        forces (natoms, 3), energies (natoms,) of the plain model."""
        self._fset = snapshots
        _lib.check(_lib.lib().mdp_sur_force_set(self._h, snapshots._h,
                                                np.ascontiguousarray(forces, dtype=np.float64).ravel(),
                                                np.ascontiguousarray(energies, dtype=np.float64), int(per)),
                   "mdp_sur_force_set")
        self.f_per = per
        self.f_snaps = snapshots.natoms // per

    def train_forces(self, steps: int, snaps_per_batch: int = 4, lr: float = 1e-3, alpha: float = 1.0,
                     seed: int = 0):
        le = np.zeros(steps, dtype=np.float32)
        lf = np.zeros(steps, dtype=np.float32)
        _lib.check(_lib.lib().mdp_sur_train_forces(self._h, int(steps), int(snaps_per_batch), float(lr),
                                                   float(alpha), int(seed), le.ctypes.data, lf.ctypes.data),
                   "mdp_sur_train_forces")
        return le, lf

    def force_grad(self, snap0: int, snaps: int, alpha: float = 1.0):
        g = np.zeros(NPAR, dtype=np.float32)
        losses = np.zeros(2, dtype=np.float32)
        _lib.check(_lib.lib().mdp_sur_force_grad(self._h, int(snap0), int(snaps), float(alpha), g, losses),
                   "mdp_sur_force_grad")
        return g, (float(losses[0]), float(losses[1]))

    def force_set_copy(self):
        n = self._fset.natoms
        npairs = int(_lib.lib().mdp_sur_force_set_npairs(self._h))
        B = np.zeros((NK, n)); db = np.zeros((npairs, 3, NK), dtype=np.float32)
        pinfo = np.zeros((npairs, 2), dtype=np.int32); poff = np.zeros(n + 1, dtype=np.int32)
        _lib.check(_lib.lib().mdp_sur_force_set_copy(self._h, B.ctypes.data, db.ctypes.data, pinfo.ctypes.data,
                                                     poff.ctypes.data), "mdp_sur_force_set_copy")
        return B.T.copy(), db, pinfo, poff

    for f in (force_set, train_forces, force_grad, force_set_copy):
        setattr(Surrogate, f.__name__, f)


_force_methods()


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
    segment: int = 100              # snapshots per trajectory before a fresh start
    force_every: int = 10           # every n-th snapshot also keeps positions and forces
    equilibrate: int = 50
    dt: float = 0.001
    seed: int = 7
    neighmax: int = 128             # hot snapshots crowd more atoms into rcut + skin


def generate(sur: Surrogate, p8: SnapParams, ts: TrainingSet, precision: str = "fp64", device: int = 0,
             forces: list | None = None) -> int:
    """Runs plain 2J=8 SNAP MD at each temperature and appends snapshots to sur's set.

    Each temperature's snapshots come from short trajectories (ts.segment
    snapshots each) restarted from a freshly jittered lattice with new
    velocities: the seeded-coefficient potential has no repulsive core, so one
    long hot trajectory drifts into collapsed configurations no deployment
    visits.  When forces is a list, every ts.force_every-th snapshot appends
    (positions, box, forces, per-atom energies) to it."""
    from .snap import SnapMD
    per = max(1, ts.snapshots // len(ts.temps))
    natoms = 2 * int(np.prod(ts.cells))
    sur.reserve(per * len(ts.temps) * natoms)
    for it, T in enumerate(ts.temps):
        done, seg = 0, 0
        md = None
        while done < per:
            # displacement scale grows with temperature so hot snapshots start disordered
            cfg = ta_config(ts.cells, temp=T, jitter=0.05 * np.sqrt(T / 300.0), seed=ts.seed + 1000 * it + seg)
            if md is None:
                md = SnapMD(p8, cfg.box, cfg.natoms, ts.dt, mass=TA_MASS, precision=precision, device=device,
                            neighmax=ts.neighmax)
            md.set_state(cfg.x, cfg.v)
            md.setup()
            md.run(ts.equilibrate)
            for _ in range(min(ts.segment, per - done)):
                md.run(ts.every)
                sur.sample(md)
                if forces is not None and done % ts.force_every == 0:
                    x, _, f, e = md.state()
                    forces.append((x, cfg.box.copy(), f, e))
                done += 1
            seg += 1
        md.close()
    return sur.size()


def linear_fit(X: np.ndarray, E: np.ndarray) -> np.ndarray:
    """Least-squares linear SNAP on the same features: E_i ~ c0 + c . B_i (the
    model the surrogate is compared against); returns the 15 coefficients."""
    A = np.hstack([np.ones((X.shape[0], 1)), X[:, :NK].astype(np.float64)])
    c, *_ = np.linalg.lstsq(A, E.astype(np.float64), rcond=None)
    return c


def force_errors(p8: SnapParams, sur: Surrogate | None, lin_coeff: np.ndarray | None, cells=(10, 10, 10),
                 temp: float = 1000.0, seed: int = 99, precision: str = "fp64", device: int = 0) -> dict:
    """Force and per-atom energy RMSE against plain 2J=8 SNAP on one configuration,
    for the surrogate and for the linear 2J=4 fit."""
    from .snap import SnapMD
    cfg = ta_config(cells, temp=temp, jitter=0.05 * np.sqrt(temp / 300.0), seed=seed)
    out = {}
    md = SnapMD(p8, cfg.box, cfg.natoms, 0.001, precision=precision, device=device, neighmax=128)
    md.set_state(cfg.x, cfg.v)
    md.setup()
    _, _, f8, e8 = md.state()
    out["force_rms_2j8"] = float(np.sqrt(np.mean(f8 ** 2)))
    if sur is not None:
        md.set_surrogate(sur, judge_every=0)
        md.set_state(cfg.x, cfg.v)
        md.setup()
        _, _, fs, es = md.state()
        out["surrogate_force_rmse"] = float(np.sqrt(np.mean((fs - f8) ** 2)))
        out["surrogate_energy_rmse"] = float(np.sqrt(np.mean((es - e8) ** 2)))
    md.close()
    if lin_coeff is not None:
        p4 = dataclasses.replace(sur.params4 if sur is not None else snap_params(4, seed=0), coeff=np.asarray(lin_coeff))
        m4 = SnapMD(p4, cfg.box, cfg.natoms, 0.001, precision="fp64", device=device, neighmax=128)
        m4.set_state(cfg.x, cfg.v)
        m4.setup()
        _, _, fl, el = m4.state()
        out["linear_force_rmse"] = float(np.sqrt(np.mean((fl - f8) ** 2)))
        out["linear_energy_rmse"] = float(np.sqrt(np.mean((el - e8) ** 2)))
        m4.close()
    return out


def train_default(p8: SnapParams, ts: TrainingSet, steps: int = 20000, batch: int = 8192, lr: float = 2e-3,
                  seed: int = 1, device: int = 0, log=print, force_steps: int = 30000, force_lr: float = 5e-4,
                  alpha: float = 4.0) -> tuple[Surrogate, dict]:
    """Generate the training set, fit the normalisation and train with Adam on
    per-atom energies, then on energies and forces of every force_every-th
    snapshot (learning rates decayed 10x over the last half of each phase)."""
    import time
    sur = Surrogate(snap_params(4, seed=0), device=device)
    t0 = time.time()
    fsnaps = [] if force_steps > 0 else None
    n = generate(sur, p8, ts, device=device, forces=fsnaps)
    t1 = time.time()
    log(f"training set: {n} atoms from {ts.snapshots} snapshots in {t1 - t0:.1f} s")
    sur.set_params(init_params(seed))
    sur.fit_normalization()
    P, norm = sur.params()
    sur.set_params(P, norm)
    losses = []
    chunk = max(1, steps // 10)
    for i in range(0, steps, chunk):
        frac = i / steps
        lri = lr if frac < 0.5 else lr * 10 ** (-(frac - 0.5) * 2)
        losses.append(sur.train(min(chunk, steps - i), batch=batch, lr=lri, seed=seed + i))
    loss = np.concatenate(losses)
    t2 = time.time()
    log(f"trained {steps} steps (batch {batch}) in {t2 - t1:.1f} s; loss {loss[:20].mean():.4f} -> {loss[-200:].mean():.4f}")
    X, E = sur.dataset()
    info = dict(rows=n, gen_s=t1 - t0, train_s=t2 - t1, loss_first=float(loss[:20].mean()),
                loss_last=float(loss[-200:].mean()), lin_coeff=linear_fit(X, E), force_steps=0)
    if force_steps > 0 and fsnaps:
        from . import fit
        per = fsnaps[0][0].shape[0]
        bf = fit.BatchFit(snap_params(4, seed=0), device=device)
        bf.set_batch([fit.FitConfig(x=np.mod(x, box), box=box, kind="snapshot") for x, box, _, _ in fsnaps])
        sur.force_set(bf, np.concatenate([f for _, _, f, _ in fsnaps]), np.concatenate([e for *_, e in fsnaps]), per)
        t3 = time.time()
        fl, el = [], []
        chunk = max(1, force_steps // 10)
        for i in range(0, force_steps, chunk):
            frac = i / force_steps
            lri = force_lr if frac < 0.5 else force_lr * 10 ** (-(frac - 0.5) * 2)
            le, lf = sur.train_forces(min(chunk, force_steps - i), snaps_per_batch=4, lr=lri, alpha=alpha,
                                      seed=seed + 7 * i)
            el.append(le); fl.append(lf)
        el, fl = np.concatenate(el), np.concatenate(fl)
        t4 = time.time()
        log(f"force matching: {len(fsnaps)} snapshots, {force_steps} steps in {t4 - t3:.1f} s; "
            f"energy loss {el[:20].mean():.4f} -> {el[-100:].mean():.4f}, force loss {fl[:20].mean():.4f} -> {fl[-100:].mean():.4f}")
        info.update(force_steps=force_steps, force_snapshots=len(fsnaps), force_train_s=t4 - t3,
                    force_loss_first=float(fl[:20].mean()), force_loss_last=float(fl[-100:].mean()))
    return sur, info


def main(argv=None):
    import argparse
    import json
    ap = argparse.ArgumentParser(description="train the 2J=4 MLP surrogate of 2J=8 SNAP on MD snapshots")
    ap.add_argument("--snapshots", type=int, default=20000)
    ap.add_argument("--cells", type=int, default=10, help="BCC cells per side of the snapshot box")
    ap.add_argument("--every", type=int, default=5)
    ap.add_argument("--steps", type=int, default=20000)
    ap.add_argument("--batch", type=int, default=8192)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--coeff-seed", type=int, default=1, help="seed of the 2J=8 SNAP coefficients")
    ap.add_argument("--out", default="surrogate_weights.npz")
    a = ap.parse_args(argv)
    p8 = snap_params(8, seed=a.coeff_seed)
    ts = TrainingSet(snapshots=a.snapshots, cells=(a.cells,) * 3, every=a.every)
    sur, info = train_default(p8, ts, steps=a.steps, batch=a.batch, lr=a.lr)
    sur.save(a.out)
    res = {}
    for T in (300.0, 1000.0, 3000.0):
        res[str(T)] = force_errors(p8, sur, info["lin_coeff"], cells=(a.cells,) * 3, temp=T)
    info["lin_coeff"] = info["lin_coeff"].tolist()
    print(json.dumps(dict(info=info, errors=res), indent=1))


if __name__ == "__main__":
    main()

"""Surrogate MLP on the GPU: kernels against the CPU oracle, forces against
finite differences of the surrogate energy, the judge / fallback logic, and
the gain of the trained network over a linear fit on the same features."""
import numpy as np
import pytest

from mdp_b200 import configs
from mdp_b200 import surrogate as su
from oracle import mlp_oracle as mo

pytestmark = pytest.mark.gpu


def _rand_norm(rng):
    return np.concatenate([rng.normal(size=14), rng.uniform(0.5, 2.0, size=14), [0.3, 1.7]]).astype(np.float32)


@pytest.fixture(scope="module")
def sur():
    s = su.Surrogate(configs.snap_params(4, seed=0))
    yield s
    s.close()


def test_eval_matches_oracle(sur):
    rng = np.random.default_rng(1)
    P = su.init_params(3)
    norm = _rand_norm(rng)
    sur.set_params(P, norm)
    B = rng.normal(size=(300, 14)) * 1.5
    E, G = sur.eval(B)
    Eo, Go = mo.energy_and_grad(P, norm, B)
    assert np.max(np.abs(E - Eo)) < 2e-5 * max(1.0, np.max(np.abs(Eo)))
    assert np.max(np.abs(G - Go)) < 2e-4 * max(1.0, np.max(np.abs(Go)))


def test_loss_gradient_matches_oracle(sur):
    rng = np.random.default_rng(2)
    P = su.init_params(4)
    norm = _rand_norm(rng)
    sur.set_params(P, norm)
    X = rng.normal(size=(517, 14)).astype(np.float32)     # several blocks, ragged tail
    E = rng.normal(size=517).astype(np.float32)
    g, loss = sur.grad(X, E)
    go, lo = mo.loss_grad(P, norm, X, E)
    assert abs(loss - lo) < 1e-4 * max(1.0, lo)
    err = np.linalg.norm(g - go) / np.linalg.norm(go)
    assert err < 1e-4, err
    # every parameter group, including the unused feature padding (zero)
    d = su.unpack(g)
    assert np.all(d["W1"][:, 14:] == 0)


def test_training_lowers_loss(sur):
    rng = np.random.default_rng(3)
    X = rng.normal(size=(20000, 14)).astype(np.float32)
    E = (np.sin(X[:, 0]) + 0.5 * X[:, 1] * X[:, 2] - 0.3 * X[:, 3] ** 2).astype(np.float32)
    sur.set_params(su.init_params(5))
    sur.load_dataset(X, E)
    sur.fit_normalization()
    P, norm = sur.params()
    sur.set_params(P, norm)
    loss = sur.train(600, batch=1024, lr=3e-3, seed=11)
    assert np.all(np.isfinite(loss))
    assert loss[-50:].mean() < 0.1 * loss[:10].mean()


def _md(p, cells, temp, seed, precision="fp64"):
    from mdp_b200.snap import SnapMD
    cfg = configs.ta_config(cells, temp=temp, jitter=0.08, seed=seed)
    md = SnapMD(p, cfg.box, cfg.natoms, 0.001, precision=precision)
    md.set_state(cfg.x, cfg.v)
    return md, cfg


def test_surrogate_forces_are_energy_gradients(sur):
    """Forces through G = dE_i/dB_i and the per-atom Y kernel = -dE_total/dx."""
    p8 = configs.snap_params(8, seed=1)
    md, cfg = _md(p8, (3, 3, 3), 600.0, 21)
    md.setup()
    B = su.features(md, sur)
    rng = np.random.default_rng(4)
    P = su.init_params(6)
    norm = np.concatenate([B.mean(0), 1.0 / (B.std(0) + 1e-12), [-11.0, 0.5]]).astype(np.float32)
    sur.set_params(P, norm)
    md.set_surrogate(sur, judge_every=0)
    md.set_state(cfg.x, cfg.v)
    md.setup()
    _, _, f, e = md.state()
    h = 4e-3
    for atom, k in [(0, 0), (7, 1), (30, 2)]:
        es = []
        for sgn in (1, -1):
            x = cfg.x.copy()
            x[atom, k] += sgn * h
            md.set_state(x, cfg.v)
            md.setup()
            es.append(md.state()[3].sum())
        fd = -(es[0] - es[1]) / (2 * h)
        assert abs(fd - f[atom, k]) < 2e-2 * max(1.0, abs(fd)), (atom, k, fd, f[atom, k])
    md.close()


def test_judge_falls_back_to_plain_model(sur):
    p8 = configs.snap_params(8, seed=1)
    ref, cfg = _md(p8, (3, 3, 3), 300.0, 22)
    ref.setup()
    ref.run(4)
    _, _, fref, _ = ref.state()
    ref.close()
    P = su.init_params(7)
    md, _ = _md(p8, (3, 3, 3), 300.0, 22)
    md.setup()
    B = su.features(md, sur)
    sur.set_params(P, np.concatenate([B.mean(0), 1.0 / (B.std(0) + 1e-12), [-11.0, 0.5]]).astype(np.float32))
    # a tolerance nothing meets: the judge at setup hands the run to SNAP
    md.set_surrogate(sur, judge_every=2, tol=1e-12)
    md.set_state(cfg.x, cfg.v)
    md.setup()
    st = md.surrogate_status()
    assert st["fallback_step"] == 0 and not st["active"] and st["judgements"] == 1
    md.run(4)
    _, _, f, _ = md.state()
    assert np.max(np.abs(f - fref)) < 1e-10 * np.max(np.abs(fref))
    assert md.surrogate_status()["judgements"] == 1
    # a tolerance everything meets: judged every 2 steps, stays active
    md.set_surrogate(sur, judge_every=2, tol=1e9)
    md.set_state(cfg.x, cfg.v)
    md.setup()
    md.run(6)
    st = md.surrogate_status()
    assert st["active"] and st["fallback_step"] == -1 and st["judgements"] == 4
    assert np.all(np.diff(st["log"][:, 0]) == 2) and np.all(st["log"][:, 1] > 0)
    md.close()


def _force_set(sur, nsnap=3, seed=40):
    """A small force set: jittered 54-atom cells with plain 2J=8 forces."""
    from mdp_b200 import fit
    from mdp_b200.snap import snap_compute
    p8 = configs.snap_params(8, seed=1)
    snaps, F, E = [], [], []
    for s in range(nsnap):
        cfg = configs.ta_config((3, 3, 3), temp=600.0, jitter=0.12, seed=seed + s)
        out = snap_compute(p8, cfg.x, cfg.box, 1.0, 96, precision="fp64")
        snaps.append(fit.FitConfig(x=cfg.x, box=cfg.box, kind="bcc"))
        F.append(out["fatom"]); E.append(out["eatom"])
    bf = fit.BatchFit(configs.snap_params(4, seed=0))
    bf.set_batch(snaps)
    sur.force_set(bf, np.concatenate(F), np.concatenate(E), 54)
    return np.concatenate(F), np.concatenate(E)


def test_force_matching_gradient_matches_oracle(sur):
    F, E = _force_set(sur)
    B, db, pinfo, poff = sur.force_set_copy()
    norm = np.concatenate([B.mean(0), 1.0 / (B.std(0) + 1e-12), [E.mean(), E.std()]]).astype(np.float32)
    P = su.init_params(9)
    sur.set_params(P, norm)
    var = np.mean(F ** 2)
    g, (le, lf) = sur.force_grad(0, 3, alpha=0.8)
    go, (leo, lfo) = mo.force_loss_grad(P, norm, B, db, pinfo, F, E, 0.8, var)
    assert abs(le - leo) < 1e-4 * max(1.0, leo) and abs(lf - lfo) < 1e-4 * max(1.0, lfo)
    err = np.linalg.norm(g - go) / np.linalg.norm(go)
    assert err < 1e-3, err


def test_force_matching_lowers_force_loss(sur):
    F, E = _force_set(sur, nsnap=8, seed=60)
    B, *_ = sur.force_set_copy()
    norm = np.concatenate([B.mean(0), 1.0 / (B.std(0) + 1e-12), [E.mean(), E.std()]]).astype(np.float32)
    sur.set_params(su.init_params(10), norm)
    le, lf = sur.train_forces(400, snaps_per_batch=2, lr=2e-3, alpha=1.0, seed=3)
    assert np.all(np.isfinite(lf)) and lf[-40:].mean() < 0.5 * lf[:10].mean()


# The network must cut the held-out force error of the method without it -- a
# linear SNAP fit on the same 14 features and the same data -- by at least
# this factor.  (The bench's full training, 20,000 snapshots, measures about
# 6x: 0.23 against 1.34 eV/A at 1,000 K.)
GAIN_FACTOR = 2.5


def test_trained_network_beats_linear_fit():
    """Trains the surrogate on the GPU (energies, then forces) on plain 2J=8 MD
    snapshots, fits the linear 2J=4 model on the same per-atom data, and
    compares both on a held-out 2,000-atom configuration at 1,000 K."""
    p8 = configs.snap_params(8, seed=2024)
    ts = su.TrainingSet(snapshots=1200, cells=(10, 10, 10), every=5, segment=50, force_every=10)
    sur, info = su.train_default(p8, ts, steps=4000, batch=8192, lr=2e-3, seed=1, force_steps=6000,
                                 log=lambda m: None)
    try:
        errs = su.force_errors(p8, sur, info["lin_coeff"], cells=(10, 10, 10), temp=1000.0, seed=4242)
    finally:
        sur.close()
    print(f"held-out 1,000 K: network {errs['surrogate_force_rmse']:.3f} eV/A, linear 2J=4 fit "
          f"{errs['linear_force_rmse']:.3f} eV/A (force RMS {errs['force_rms_2j8']:.2f}); energies "
          f"{errs['surrogate_energy_rmse']:.4f} / {errs['linear_energy_rmse']:.4f} eV")
    assert errs["surrogate_force_rmse"] * GAIN_FACTOR < errs["linear_force_rmse"]
    assert errs["surrogate_energy_rmse"] < errs["linear_energy_rmse"]

"""Small, fixed workloads for kernel profiling.

    python profile_case.py fp64|fp32 CELLS [REPEAT]
        REPEAT (default 2) SNAP force evaluations (snap_compute) on a
        CELLS^3-cell BCC Ta lattice (2*CELLS^3 atoms, jitter 0.05 A, 2J=8).
    python profile_case.py sur CELLS [REPEAT]
        the surrogate force path (random network, normalised on the lattice's
        own features) for REPEAT steps of NVE on the same lattice.
    python profile_case.py fit NCONF [REPEAT]
        REPEAT runs of the batched descriptors + FP64 normal equations over
        NCONF configurations of the fitting workload.

The first call warms the library up, so a capture of one launch of a kernel
skips the first with `-s 1`.  Sizes stay small (20 cells = 16,000 atoms, 64
configurations) so profiler replays finish quickly.
"""
from __future__ import annotations

import os
import sys

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
from mdp_b200 import configs  # noqa: E402


def main(argv=None):
    argv = sys.argv[1:] if argv is None else argv
    kind = argv[0] if argv else "fp64"
    n = int(argv[1]) if len(argv) > 1 else 20
    rep = int(argv[2]) if len(argv) > 2 else 2
    if kind in ("fp64", "fp32"):
        from mdp_b200.snap import snap_compute
        p = configs.snap_params(8, seed=1)
        cfg = configs.ta_config((n, n, n), temp=300, jitter=0.05, seed=1)
        out = None
        for _ in range(rep):
            out = snap_compute(p, cfg.x, cfg.box, 1.0, 64, precision=kind)
        print("ok", cfg.natoms, float(out["eatom"].sum()))
    elif kind == "sur":
        from mdp_b200 import surrogate as su
        from mdp_b200.snap import SnapMD
        p = configs.snap_params(8, seed=1)
        cfg = configs.ta_config((n, n, n), temp=1000, jitter=0.09, seed=1)
        sur = su.Surrogate(configs.snap_params(4, seed=0))
        md = SnapMD(p, cfg.box, cfg.natoms, 0.001)
        md.set_state(cfg.x, cfg.v)
        md.setup()
        B = su.features(md, sur)
        sur.set_params(su.init_params(1), np.concatenate([B.mean(0), 1.0 / (B.std(0) + 1e-12), [-11.7, 0.1]]))
        md.set_surrogate(sur, judge_every=0)
        md.setup()
        md.run(rep)
        print("ok", cfg.natoms, float(md.state()[3].sum()))
    elif kind == "fit":
        from mdp_b200 import fit
        cfgs, e, f = fit.batch_configs(n, seed=3)
        bf = fit.BatchFit(configs.snap_params(8, seed=0))
        bf.set_batch(cfgs, e, f)
        A = None
        for _ in range(rep):
            A, b, ms = bf.run("fp64")
        print("ok", bf.natoms, float(A[0, 0]))
    else:
        raise SystemExit(f"unknown case {kind}")


if __name__ == "__main__":
    main()

"""Small, fixed SNAP force evaluations for kernel profiling.

    python -m mdp_b200.profile_case PREC CELLS [REPEAT]

Runs REPEAT (default 2) calls of snap_compute on a CELLS^3-cell BCC Ta lattice
(2*CELLS^3 atoms, jitter 0.05 A, 2J=8, seeded coefficients) at PREC ("fp64" or
"fp32"); the first call warms the library up, so a capture of one launch of a
kernel skips the first with `-s 1`.  The sizes stay small (20 cells =
16,000 atoms, 40 cells = 128,000 atoms) so profiler replays finish quickly.
"""
from __future__ import annotations

import sys

from . import configs
from .snap import snap_compute


def main(argv=None):
    argv = sys.argv[1:] if argv is None else argv
    prec = argv[0] if argv else "fp64"
    n = int(argv[1]) if len(argv) > 1 else 20
    rep = int(argv[2]) if len(argv) > 2 else 2
    p = configs.snap_params(8, seed=1)
    cfg = configs.ta_config((n, n, n), temp=300, jitter=0.05, seed=1)
    out = None
    for _ in range(rep):
        out = snap_compute(p, cfg.x, cfg.box, 1.0, 64, precision=prec)
    print("ok", cfg.natoms, float(out["eatom"].sum()))


if __name__ == "__main__":
    main()

"""Linear SNAP fit of a training-data folder tree, the counterpart of MDP's
fitting/snap/Ta/fitsnap.jl:1-159.

    python -m mdp_b200.fitsnap --data <dir with the 12 Ta folders> [--twojmax 6] [--mode fp64]

The defaults are fitsnap.jl's: the 12 Ta folders and their (energy, force,
stress) weights, species Ta, rcut 4.67637, rfac0 0.99363, rmin0 0,
switching on, bzero / bnorm / wselfall off, 2J = 6, energies per atom and
stresses per volume, and the ZBL reference potential (inner 4.0, outer 4.8,
Z 73) subtracted from the targets (--no-zbl leaves it out).  Prints the
coefficients and the per-folder unweighted errors (printerrors) as one JSON
object.  fitsnap.jl also sets transposelattice = true, which reads the cell
vectors as the columns of each file's Lattice array; --transpose-lattice does
the same (dataset.reference_orientation) and reproduces the reference's
published errors, while the default reads them as rows, the reading under
which the Ta files' atoms sit at their crystal positions.
"""
from __future__ import annotations

import argparse
import json
import os

from . import configs, dataset

# fitsnap.jl:14-30: folders and their (energy, force, stress) weights
TA_FOLDERS = (
    ("Displaced_A15", 100.0, 1.0, 1e-8),
    ("Displaced_BCC", 100.0, 1.0, 1e-8),
    ("Displaced_FCC", 100.0, 1.0, 1e-8),
    ("Elastic_BCC", 1e-8, 1e-8, 1e-4),
    ("Elastic_FCC", 1e-9, 1e-9, 1e-9),
    ("GSF_110", 100.0, 1.0, 1e-8),
    ("GSF_112", 100.0, 1.0, 1e-8),
    ("Liquid", 467.0, 1.0, 1e-8),
    ("Surface", 100.0, 1.0, 1e-8),
    ("Volume_A15", 1.0, 1e-9, 1e-9),
    ("Volume_BCC", 1.0, 1e-9, 1e-9),
    ("Volume_FCC", 1.0, 1e-9, 1e-9),
)


# fitsnap.jl:81: addpotential("pair", "nonbonded", [1, 1], "zbl", [4.0, 4.8, 73], 4.8)
TA_ZBL = (4.0, 4.8, 73.0)


def load_groups(root: str, folders=TA_FOLDERS, species=("Ta",), extension: str = "json",
                transpose_lattice: bool = False):
    """One Group per folder; transpose_lattice reads the cells as fitsnap.jl
    does (dataset.reference_orientation)."""
    groups = []
    for name, we, wf, ws in folders:
        frames = dataset.read_folder(os.path.join(root, name), species, extension)
        if transpose_lattice:
            frames = [dataset.reference_orientation(fr, True) for fr in frames]
        groups.append(dataset.Group(name, frames, we, wf, ws))
    return groups


def main(argv=None) -> dict:
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--data", required=True, help="folder holding the training-data folders")
    ap.add_argument("--twojmax", type=int, default=6)
    ap.add_argument("--mode", choices=("fp64", "bf16"), default="fp64")
    ap.add_argument("--extension", default="json")
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("--no-zbl", action="store_true", help="fit without the ZBL reference potential")
    ap.add_argument("--transpose-lattice", action="store_true",
                    help="read the cell vectors as the columns of Lattice, as fitsnap.jl's transposelattice = true")
    a = ap.parse_args(argv)
    p = configs.snap_params(a.twojmax, seed=0, rcutfac=4.67637, radelem=0.5, rfac0=0.99363, rmin0=0.0,
                            switchflag=1, bzeroflag=0, bnormflag=0, wselfallflag=0)
    out = dataset.fit_groups(load_groups(a.data, extension=a.extension, transpose_lattice=a.transpose_lattice), p,
                             mode=a.mode, device=a.device, zbl=None if a.no_zbl else TA_ZBL)
    res = dict(coefficients=out["beta"].tolist(), errors=out["errors"], configs=out["configs"],
               atoms=out["atoms"], replicated=out["replicated"], graph_ms=out["graph_ms"])
    print(json.dumps(res))
    return res


if __name__ == "__main__":
    main()

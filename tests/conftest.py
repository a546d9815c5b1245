import glob
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200)")


def golden_names():
    """Force / MD fixtures (the fit_* fixtures hold descriptors and are listed by fit_names)."""
    return sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN, "*.npz"))
                  if not os.path.basename(p).startswith(("fit_", "tri_", "c2_", "chem_", "quad_")))


def tri_names():
    """Sheared-cell force fixtures."""
    return sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN, "tri_*.npz")))


def fit_names():
    return sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN, "fit_*.npz")))


def row_hashes(nl, nn):
    """One 64-bit hash per neighbour row of its sorted index set: the rows of
    a 16,000-atom list are pinned by 128 KB instead of the list itself."""
    nl = np.asarray(nl)
    nn = np.asarray(nn).astype(np.int64)
    cols = np.arange(nl.shape[1])[None, :]
    srt = np.sort(np.where(cols < nn[:, None], nl, np.iinfo(np.int32).max), axis=1).astype(np.uint64)
    h = nn.astype(np.uint64)
    with np.errstate(over="ignore"):
        for k in range(nl.shape[1]):
            h = h * np.uint64(1000003) + np.where(k < nn, srt[:, k] + np.uint64(1), np.uint64(0))
    return h


def load_golden(name):
    return dict(np.load(os.path.join(GOLDEN, name + ".npz")))


def golden_params(g):
    from mdp_b200 import configs
    bnorm, bzero, switch = (int(v) for v in g["flags"])
    p = configs.snap_params(int(g["twojmax"]), seed=int(g["coeff_seed"]), bnormflag=bnorm, bzeroflag=bzero,
                            switchflag=switch)
    assert np.array_equal(p.coeff, g["coeff"])
    return p


@pytest.fixture(scope="session")
def cuda_lib():
    """The CUDA library, built in-tree if needed; GPU tests fail (not skip)
    when it cannot be loaded."""
    from mdp_b200 import _lib, build
    if not os.path.exists(_lib.LIB_PATH):
        build.build()
    return _lib.lib()

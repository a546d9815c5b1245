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
                  if not os.path.basename(p).startswith(("fit_", "tri_")))


def tri_names():
    """Sheared-cell force fixtures."""
    return sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN, "tri_*.npz")))


def fit_names():
    return sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN, "fit_*.npz")))


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

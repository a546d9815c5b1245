"""GPU: MDP's Julia call sequence on the reference CPU library and on ours,
stage by stage, identical inputs."""
import os

import numpy as np
import pytest

import julia_abi
from conftest import golden_params, load_golden
from oracle import refpy

pytestmark = pytest.mark.gpu


def rel_inf(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


@pytest.mark.parametrize("name", ["bcc128_2j6", "bcc250_2j8", "bcc128_2j4", "bcc54_2j8_flags"])
def test_julia_abi_matches_reference_library(cuda_lib, name):
    from mdp_b200 import _lib
    ref = os.path.join(refpy.REF_DIR, "libcpuSnap_ref.so")
    if not os.path.exists(ref):
        pytest.fail("oracle/_ref/libcpuSnap_ref.so missing (build with make -C oracle ref)")
    g = load_golden(name)
    p = golden_params(g)
    a = julia_abi.snap_sequence(julia_abi.bind(ref), g, p)
    b = julia_abi.snap_sequence(julia_abi.bind(_lib.LIB_PATH), g, p)
    assert np.array_equal(a["pairnum"], b["pairnum"]) and np.array_equal(a["pairlist"], b["pairlist"])
    assert np.array_equal(a["rij"], b["rij"]) and np.array_equal(a["aj"], b["aj"])
    for k in (0, 1):
        assert rel_inf(b["u_pairs"][k], a["u_pairs"][k]) < 1e-12
        assert rel_inf(b["u"][k], a["u"][k]) < 1e-12
        assert rel_inf(b["y"][k], a["y"][k]) < 1e-10
    assert rel_inf(b["eatom"], a["eatom"]) < 1e-12
    assert rel_inf(b["blist"], a["blist"]) < 1e-10
    assert rel_inf(b["fatom"], a["fatom"]) < 1e-10
    assert rel_inf(b["vatom"], a["vatom"]) < 1e-10
    # and against the golden ComputePairSnap3 forces
    assert rel_inf(b["fatom"].reshape(-1, 3), g["fatom"]) < 1e-10

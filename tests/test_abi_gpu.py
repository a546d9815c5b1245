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


@pytest.mark.parametrize("name,quadratic", [("bcc128_2j6", 0), ("bcc250_2j8", 0), ("bcc128_2j4", 1),
                                            ("bcc54_2j8_flags", 0), ("bcc250_2j8_hot", 1)])
def test_descriptor_chain_matches_reference_library(cuda_lib, name, quadratic):
    """snapdescriptors' calls (pair U and dU, U totals, Z, B, dB/dr, tallies)
    on the reference CPU library and on ours, stage by stage."""
    from mdp_b200 import _lib
    ref = os.path.join(refpy.REF_DIR, "libcpuSnap_ref.so")
    if not os.path.exists(ref):
        pytest.fail("oracle/_ref/libcpuSnap_ref.so missing (build with make -C oracle ref)")
    g = load_golden(name)
    p = golden_params(g)
    a = julia_abi.descriptor_sequence(julia_abi.bind(ref), g, p, quadratic)
    b = julia_abi.descriptor_sequence(julia_abi.bind(_lib.LIB_PATH), g, p, quadratic)
    for key in ("ulist", "dulist", "sij", "utot", "zlist"):
        for x, y in zip(b[key], a[key]):
            assert rel_inf(x, y) < 1e-12, key
    for key in ("blist", "dblist", "bi", "bd", "bv"):
        assert rel_inf(b[key], a[key]) < 1e-10, key
    # entries the reference leaves alone (dU right of the half plane) stay zero
    dur = a["dulist"][0].reshape(3, -1)
    assert np.count_nonzero(dur) < dur.size
    assert np.array_equal(b["dulist"][0] == 0.0, a["dulist"][0] == 0.0)


CHEM = ["chem_bcc128_2j6", "chem_bcc250_2j8", "chem_bcc54_2j4_3el_flags", "chem_bcc54_2j6_wselfall",
        "chem_bcc128_2j8_chemflag0"]


@pytest.mark.parametrize("name", CHEM)
def test_julia_abi_several_elements_match_reference_library(cuda_lib, name):
    """Several element types through the cpuSnap.h stages: U per element block,
    wself per block, element-triple energies and bispectrum, Y per block, dE/dr
    with per-pair cutoffs, on the reference library and on ours."""
    from mdp_b200 import _lib, configs
    ref = os.path.join(refpy.REF_DIR, "libcpuSnap_ref.so")
    if not os.path.exists(ref):
        pytest.fail("oracle/_ref/libcpuSnap_ref.so missing (build with make -C oracle ref)")
    g = load_golden(name)
    bnorm, bzero, switch, wsa = (int(v) for v in g["flags"])
    p = configs.snap_params_elements(int(g["twojmax"]), g["radelems"], g["wjelems"], chemflag=int(g["chemflag"]),
                                     seed=int(g["coeff_seed"]), bnormflag=bnorm, bzeroflag=bzero,
                                     switchflag=switch, wselfallflag=wsa)
    a = julia_abi.snap_sequence_elements(julia_abi.bind(ref), g, p)
    b = julia_abi.snap_sequence_elements(julia_abi.bind(_lib.LIB_PATH), g, p)
    assert np.array_equal(a["pairnum"], b["pairnum"]) and np.array_equal(a["pairlist"], b["pairlist"])
    for k in (0, 1):
        assert rel_inf(b["u_pairs"][k], a["u_pairs"][k]) < 1e-12
        assert rel_inf(b["u"][k], a["u"][k]) < 1e-12
        assert rel_inf(b["y"][k], a["y"][k]) < 1e-10
    assert rel_inf(b["eatom"], a["eatom"]) < 1e-12
    assert rel_inf(b["blist"], a["blist"]) < 1e-10
    assert rel_inf(b["fatom"], a["fatom"]) < 1e-10
    assert rel_inf(b["vatom"], a["vatom"]) < 1e-10

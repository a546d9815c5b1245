"""CPU: the C-ABI library loads and exports every function include/*.h declares."""
import glob
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import ROOT


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        # only the extern "C" declarations (the template wrappers are header-only)
        text = text.split("#ifdef MDP_B200_GPUCORE_TEMPLATES")[0]
        for m in re.finditer(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b([A-Za-z_]\w*)\s*\(", text, flags=re.M):
            name = m.group(1)
            if name not in ("if", "for", "while", "return", "sizeof"):
                names.add(name)
    return names


def test_library_exports_all_declared_symbols(cuda_lib):
    from mdp_b200 import _lib
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True, text=True, check=True)
    exported = {line.split()[-1] for line in out.stdout.splitlines() if line.strip()}
    want = declared_functions()
    assert len(want) > 40
    missing = sorted(want - exported)
    assert not missing, missing


def test_library_loads_without_gpu(cuda_lib):
    assert cuda_lib.mdp_snap_ncoeff(8) == 55
    assert cuda_lib.mdp_snap_ncoeff(6) == 30
    assert cuda_lib.idxucount(8) == 285 and cuda_lib.idxzcount(8) == 2386 and cuda_lib.idxcgcount(8) == 4098


def test_init_sna_tables_match_reference(cuda_lib):
    """cpuInitSna is host code: compare it with the reference library on the CPU."""
    from oracle import refpy
    import julia_abi
    from mdp_b200 import _lib
    ref = os.path.join(refpy.REF_DIR, "libcpuSnap_ref.so")
    if not os.path.exists(ref):
        pytest.skip("reference build not present")
    for tj in (4, 6, 8):
        a = julia_abi.tables(julia_abi.bind(ref), tj)
        b = julia_abi.tables(julia_abi.bind(_lib.LIB_PATH), tj)
        for k in ("idx_max", "idxz", "idxz_block", "idxb", "idxb_block", "idxu_block", "idxcg_block"):
            assert np.array_equal(a[k][:4] if k == "idx_max" else a[k], b[k][:4] if k == "idx_max" else b[k]), k
        assert np.abs(a["cg"] - b["cg"]).max() < 1e-14
        assert np.abs(a["rootpq"] - b["rootpq"]).max() < 1e-15


# every function of MDP's Julia C ABI (src/Julia/Potential/cpuSnap.h:7-84)
JULIA_ABI = ["idxbcount", "idxcgcount", "idxucount", "idxzcount", "cpuInitSna", "cpuNeighPairList", "cpuNeighPairs",
             "cpuSnapComputeUi", "cpuAddWself2Ui", "cpuSnapComputeEi", "cpuSnapComputeBi", "cpuSnapComputeYi",
             "cpuSnapComputeFi", "cpuComputeSij", "cpuComputeUij", "cpuZeroUarraytot2", "cpuAddUarraytot",
             "cpuComputeZi2", "cpuComputeBi2", "cpuComputeDbidrj", "cpuSnapTallyBispectrum",
             "cpuSnapTallyBispectrumDeriv", "cpuSnapTallyBispectrumVirial"]


def test_library_exports_the_whole_julia_abi(cuda_lib):
    from mdp_b200 import _lib
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True, text=True, check=True)
    exported = {line.split()[-1] for line in out.stdout.splitlines() if line.strip()}
    assert not sorted(set(JULIA_ABI) - exported)
    assert set(JULIA_ABI) <= declared_functions()

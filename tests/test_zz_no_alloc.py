"""GPU: the allocation-free bispectrum entry point.

mdp_gpu_snap_compute_bi_noalloc_f64 serves callers that must not allocate
device memory (a host application whose memory pool owns the device, or a loop
that cannot take cudaMalloc/cudaFree's implicit synchronisation).  It keeps its
scratch in a fixed array inside the library.  This test calls it through the C
ABI twice in a row, on two different configurations, and checks each result
against the existing entry point mdp_gpu_snap_compute_bi_f64 and against the
per-atom bispectrum of the reference's own library (cpuSnapComputeBi of
oracle/_ref/libcpuSnap_ref.so, MDP's src/Julia/Potential/cpuSnap.cpp).  On the
second call it also checks the property the entry point exists for: the free
device memory is the same before and after the call.  A size beyond the fixed
scratch is refused.  The file is named so pytest collects it last."""
import os
import ctypes as C

import numpy as np
import pytest

import julia_abi
from conftest import golden_params, load_golden

pytestmark = pytest.mark.gpu

TOL_FP64 = 1e-10


def rel_inf(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


REF_LIB = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref",
                       "libcpuSnap_ref.so")


def _u_of(name, lib_path):
    """U (wself added, mirrored) of a golden configuration in MDP's layout,
    computed through this library's Julia-ABI entry points, and the
    reference library's per-atom bispectrum of the same configuration."""
    g = load_golden(name)
    p = golden_params(g)
    seq = julia_abi.snap_sequence(julia_abi.bind(lib_path), g, p)
    if not os.path.exists(REF_LIB):
        pytest.fail("oracle/_ref/libcpuSnap_ref.so missing (build with make -C oracle ref)")
    ref = julia_abi.snap_sequence(julia_abi.bind(REF_LIB), g, p)
    return p, g["x"].shape[0], seq["u"], seq["tables"], ref["blist"]


def test_no_alloc_bispectrum_matches_existing_entry(cuda_lib):
    import torch
    from mdp_b200 import _lib
    L = cuda_lib
    L.mdp_gpu_snap_compute_bi_noalloc_f64.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int,
                                                      C.c_int, C.c_int, C.c_void_p]
    L.mdp_gpu_snap_compute_bi_noalloc_f64.restype = C.c_int
    L.mdp_gpu_snap_compute_bi_f64.argtypes = [C.c_void_p] * 9 + [C.c_int] * 9
    L.mdp_gpu_snap_compute_bi_f64.restype = None
    dev = torch.device("cuda:0")
    stream = torch.cuda.current_stream().cuda_stream
    for call, name in enumerate(("bcc250_2j8", "bcc54_2j8_flags")):   # two calls in a row, the second smaller
        p, n, (ur, ui), t, bref = _u_of(name, _lib.LIB_PATH)
        ur_d = torch.tensor(ur, dtype=torch.float64, device=dev)
        ui_d = torch.tensor(ui, dtype=torch.float64, device=dev)
        nb = t["nb"]
        existing = torch.zeros(nb * n, dtype=torch.float64, device=dev)
        L.mdp_gpu_snap_compute_bi_f64(existing.data_ptr(), ur_d.data_ptr(), ui_d.data_ptr(), None, None, None,
                                      None, None, None, p.twojmax, nb, t["nu"], t["nz"], 1, p.bnormflag,
                                      p.bzeroflag, p.wselfallflag, n)
        torch.cuda.synchronize()
        out = torch.full((nb * n,), float("nan"), dtype=torch.float64, device=dev)
        torch.cuda.synchronize()
        free0 = torch.cuda.mem_get_info()[0]
        rc = L.mdp_gpu_snap_compute_bi_noalloc_f64(out.data_ptr(), ur_d.data_ptr(), ui_d.data_ptr(), p.twojmax,
                                                   p.bnormflag, p.bzeroflag, n, stream)
        assert rc == 0, L.mdp_last_error()
        torch.cuda.synchronize()
        if call > 0:   # after the first call (which loads the kernels), nothing is allocated
            assert torch.cuda.mem_get_info()[0] == free0
        a, b = out.cpu().numpy(), existing.cpu().numpy()
        assert np.all(np.isfinite(a))
        assert rel_inf(a, b) < TOL_FP64, name
        assert rel_inf(a, np.asarray(bref).ravel()) < TOL_FP64, name


def test_no_alloc_rejects_sizes_beyond_its_scratch(cuda_lib):
    import torch
    L = cuda_lib
    L.mdp_gpu_snap_compute_bi_noalloc_f64.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int,
                                                      C.c_int, C.c_int, C.c_void_p]
    L.mdp_gpu_snap_compute_bi_noalloc_f64.restype = C.c_int
    buf = torch.zeros(16, dtype=torch.float64, device="cuda:0")
    rc = L.mdp_gpu_snap_compute_bi_noalloc_f64(buf.data_ptr(), buf.data_ptr(), buf.data_ptr(), 8, 0, 0, 2049, None)
    assert rc == -1
    assert b"2048" in L.mdp_last_error()

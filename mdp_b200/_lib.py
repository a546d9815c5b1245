"""ctypes loader for libmdp_b200.so.

The CUDA library is the product path: there is no CPU fallback.  Loading
fails loudly when the library is missing; calls fail loudly when the CUDA
runtime reports an error.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libmdp_b200.so")

_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_ip = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")


class MdpError(RuntimeError):
    pass


class SnapParamsC(C.Structure):
    _fields_ = [("twojmax", C.c_int), ("rcutfac", C.c_double), ("rfac0", C.c_double), ("rmin0", C.c_double),
                ("radelem", C.c_double), ("wjelem", C.c_double), ("switchflag", C.c_int), ("bzeroflag", C.c_int),
                ("bnormflag", C.c_int), ("wselfallflag", C.c_int), ("quadraticflag", C.c_int),
                ("chemflag", C.c_int), ("ncoeffall", C.c_int), ("coeff", C.POINTER(C.c_double)),
                ("nelements", C.c_int), ("radelems", C.POINTER(C.c_double)), ("wjelems", C.POINTER(C.c_double))]


class MDConfigC(C.Structure):
    _fields_ = [("natoms", C.c_int), ("box", C.c_double * 9), ("mass", C.c_double), ("dt", C.c_double),
                ("skin", C.c_double), ("neighmax", C.c_int), ("neighevery", C.c_int), ("neighdelay", C.c_int),
                ("neighcheck", C.c_int), ("precision", C.c_int), ("device", C.c_int)]


_lib = None


def lib():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise MdpError(f"{LIB_PATH} is missing: build it with `python -m mdp_b200.build`")
    L = C.CDLL(LIB_PATH)
    L.mdp_last_error.restype = C.c_char_p
    L.mdp_snap_ncoeff.argtypes = [C.c_int]
    L.mdp_snap_compute_host.argtypes = [C.POINTER(SnapParamsC), C.c_int, C.c_int, _dp, _dp, C.c_double, C.c_int,
                                        C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                        C.c_void_p, C.c_void_p, C.c_int]
    L.mdp_snap_compute_device.argtypes = [C.POINTER(SnapParamsC), C.c_int, C.c_void_p, C.c_void_p, C.c_void_p,
                                          C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p,
                                          C.c_void_p, C.c_void_p]
    L.mdp_snap_compute_host_typed.argtypes = [C.POINTER(SnapParamsC), C.c_int, C.c_int, _dp, _ip, _dp, C.c_double,
                                              C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                              C.c_void_p, C.c_void_p, C.c_void_p, C.c_int]
    L.mdp_snap_compute_device_typed.argtypes = [C.POINTER(SnapParamsC), C.c_int] + [C.c_void_p] * 5 + \
        [C.c_int] * 3 + [C.c_void_p] * 4
    L.mdp_md_set_types.argtypes = [C.c_void_p, _ip]
    L.mdp_md_create.argtypes = [C.POINTER(C.c_void_p), C.POINTER(SnapParamsC), C.POINTER(MDConfigC)]
    L.mdp_md_destroy.argtypes = [C.c_void_p]
    L.mdp_md_destroy.restype = None
    L.mdp_md_set_state.argtypes = [C.c_void_p, _dp, _dp]
    L.mdp_md_set_state_device.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
    L.mdp_md_setup.argtypes = [C.c_void_p]
    L.mdp_md_run.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_int, C.POINTER(C.c_int),
                             C.POINTER(C.c_float)]
    L.mdp_md_get_state.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    L.mdp_md_thermo.argtypes = [C.c_void_p, _dp]
    L.mdp_md_counters.argtypes = [C.c_void_p, np.ctypeslib.ndpointer(dtype=np.int64, flags="C_CONTIGUOUS")]
    L.mdp_md_stage_timing.argtypes = [C.c_void_p, C.c_int]
    L.mdp_md_stage_times.argtypes = [C.c_void_p, _dp, C.POINTER(C.c_longlong)]
    L.mdp_md_stream.argtypes = [C.c_void_p]
    L.mdp_md_stream.restype = C.c_void_p
    L.mdp_md_upload.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
    L.mdp_md_download.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
    L.mdp_md_sync.argtypes = [C.c_void_p]
    L.mdp_launch_count.restype = C.c_longlong
    L.mdp_probe_fma_peak.argtypes = [C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_double)]
    _fp = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
    L.mdp_sur_create.argtypes = [C.POINTER(C.c_void_p), C.POINTER(SnapParamsC), C.c_int]
    L.mdp_sur_destroy.argtypes = [C.c_void_p]
    L.mdp_sur_destroy.restype = None
    L.mdp_sur_set_params.argtypes = [C.c_void_p, _fp, C.c_void_p]
    L.mdp_sur_get_params.argtypes = [C.c_void_p, _fp, _fp]
    L.mdp_sur_dataset_reserve.argtypes = [C.c_void_p, C.c_long]
    L.mdp_sur_dataset_size.argtypes = [C.c_void_p]
    L.mdp_sur_dataset_size.restype = C.c_long
    L.mdp_sur_dataset_load.argtypes = [C.c_void_p, _fp, _fp, C.c_long]
    L.mdp_sur_dataset_copy.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_long, C.c_long]
    L.mdp_sur_fit_normalization.argtypes = [C.c_void_p]
    L.mdp_sur_train.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_float, C.c_ulonglong, _fp]
    L.mdp_sur_grad.argtypes = [C.c_void_p, _fp, _fp, C.c_int, _fp, C.POINTER(C.c_float)]
    L.mdp_sur_eval.argtypes = [C.c_void_p, _dp, C.c_int, _dp, _fp]
    L.mdp_md_sur_sample.argtypes = [C.c_void_p, C.c_void_p]
    L.mdp_md_sur_features.argtypes = [C.c_void_p, C.c_void_p, _dp]
    L.mdp_md_set_surrogate.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_double]
    L.mdp_md_set_zbl.argtypes = [C.c_void_p, C.c_double, C.c_double, C.c_double]
    _ip32 = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
    L.mdp_sur_force_set.argtypes = [C.c_void_p, C.c_void_p, _dp, _dp, C.c_int]
    L.mdp_sur_force_set_npairs.argtypes = [C.c_void_p]
    L.mdp_sur_force_set_npairs.restype = C.c_longlong
    L.mdp_sur_train_forces.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_float, C.c_float, C.c_ulonglong,
                                       C.c_void_p, C.c_void_p]
    L.mdp_sur_force_grad.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_float, _fp, _fp]
    L.mdp_sur_force_set_copy.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    L.mdp_fit_create.argtypes = [C.POINTER(C.c_void_p), C.POINTER(SnapParamsC), C.c_int]
    L.mdp_fit_destroy.argtypes = [C.c_void_p]
    L.mdp_fit_destroy.restype = None
    L.mdp_fit_ncoeff.argtypes = [C.c_void_p]
    L.mdp_fit_set_batch.argtypes = [C.c_void_p, C.c_int, _ip32, _dp, _dp, C.c_void_p, C.c_void_p, C.c_void_p,
                                    C.c_void_p]
    L.mdp_fit_set_batch_lattice.argtypes = [C.c_void_p, C.c_int, _ip32, _dp, _dp, C.c_void_p, C.c_void_p,
                                            C.c_void_p, C.c_void_p]
    L.mdp_fit_zbl.argtypes = [C.c_void_p, C.c_double, C.c_double, C.c_double, _dp, _dp, _dp]
    L.mdp_fit_npairs.argtypes = [C.c_void_p]
    L.mdp_fit_npairs.restype = C.c_longlong
    L.mdp_fit_set_chunk_bytes.argtypes = [C.c_void_p, C.c_double]
    L.mdp_fit_nchunks.argtypes = [C.c_void_p]
    L.mdp_fit_descriptors.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    L.mdp_fit_run.argtypes = [C.c_void_p, C.c_int, _dp, _dp, C.POINTER(C.c_float)]
    L.mdp_fit_tune.argtypes = [C.c_void_p, _ip32]
    L.mdp_md_surrogate_status.argtypes = [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_longlong),
                                          C.POINTER(C.c_int), C.c_void_p, C.c_int]
    _lib = L
    return L


def check(rc: int, what: str = "mdp call"):
    if rc != 0:
        msg = lib().mdp_last_error()
        raise MdpError(f"{what} failed: {msg.decode() if msg else 'unknown error'}")


def snap_params_c(p) -> tuple[SnapParamsC, tuple]:
    """Pack a mdp_b200.configs.SnapParams into the C struct (keeps the
    coefficient and element arrays alive through the returned tuple)."""
    coeff = np.ascontiguousarray(p.coeff, dtype=np.float64)
    radelems = getattr(p, "radelems", None)
    ne = len(radelems) if radelems else 0
    rad = np.ascontiguousarray(radelems if ne else [p.radelem], dtype=np.float64)
    wj = np.ascontiguousarray(p.wjelems if ne else [p.wjelem], dtype=np.float64)
    dptr = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))
    ncoeffall = p.ncoeffall if hasattr(p, "ncoeffall") else coeff.size
    s = SnapParamsC(p.twojmax, p.rcutfac, p.rfac0, p.rmin0, p.radelem, p.wjelem, p.switchflag, p.bzeroflag,
                    p.bnormflag, p.wselfallflag, p.quadraticflag, p.chemflag, ncoeffall, dptr(coeff), ne,
                    dptr(rad) if ne else None, dptr(wj) if ne else None)
    return s, (coeff, rad, wj)

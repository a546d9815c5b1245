"""Python host layer over libmdp_b200.so.

Mirrors the two ways MDP drives the SNAP force path:
  * `snap_compute` -- one energy/force/virial evaluation of a periodic
    configuration (the role of `snappotential` in
    src/Julia/Potential/snapcpp.jl:323-426 and of ComputePairSnap3 in
    src/C++/Descriptors/snappotential.cpp:634-760);
  * `SnapMD` -- the NVE velocity-Verlet run of cpuMDP/gpuMDP
    (src/C++/Integration/Integration.cpp:17-156), with the same thermo
    columns (step, temperature, potential energy/atom, total energy/atom,
    pressure).
Every computation runs in the CUDA library; there is no CPU path.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from .configs import SnapParams, TA_MASS

PREC = {"fp64": 0, "fp32": 1}


def _box9(box) -> np.ndarray:
    b = np.asarray(box, dtype=np.float64)
    if b.shape == (3,):
        return np.array([b[0], 0, 0, 0, b[1], 0, 0, 0, b[2]], dtype=np.float64)
    return np.ascontiguousarray(b.reshape(9), dtype=np.float64)


def _ptr(a):
    return None if a is None else a.ctypes.data


def snap_compute(params: SnapParams, x: np.ndarray, box, skin: float = 1.0, neighmax: int = 64,
                 precision: str = "fp64", want_neighbors: bool = False, types=None) -> dict:
    """Energy per atom, forces (N,3), per-atom virial (6,N) of a periodic
    configuration; optionally the neighbour structure (ghost positions,
    owner list, neighbour rows).  types: atom types 1..nelements, required by
    models with several element types."""
    L = _lib.lib()
    x = np.ascontiguousarray(x, dtype=np.float64)
    n = x.shape[0]
    sp, keep = _lib.snap_params_c(params)
    e = np.zeros(n); f = np.zeros((n, 3)); v = np.zeros((6, n))
    nl = nn = al = xa = None
    anum = C.c_int(0)
    cap = 0
    if want_neighbors:
        nl = np.zeros((n, neighmax), dtype=np.int32); nn = np.zeros(n, dtype=np.int32)
        cap = 30 * n + 4096
        al = np.zeros(cap, dtype=np.int32); xa = np.zeros((cap, 3))
    if types is None:
        rc = L.mdp_snap_compute_host(C.byref(sp), PREC[precision], n, x, _box9(box), float(skin), int(neighmax),
                                     _ptr(e), _ptr(f), _ptr(v), _ptr(nl), _ptr(nn), C.addressof(anum), _ptr(al),
                                     _ptr(xa), cap)
    else:
        t = np.ascontiguousarray(types, dtype=np.int32)
        if t.shape != (n,):
            raise ValueError(f"types must hold one type per atom ({n}), got shape {t.shape}")
        rc = L.mdp_snap_compute_host_typed(C.byref(sp), PREC[precision], n, x, t, _box9(box), float(skin),
                                           int(neighmax), _ptr(e), _ptr(f), _ptr(v), _ptr(nl), _ptr(nn),
                                           C.addressof(anum), _ptr(al), _ptr(xa), cap)
    _lib.check(rc, "mdp_snap_compute_host")
    out = dict(eatom=e, fatom=f, vatom=v)
    if want_neighbors:
        a = anum.value
        out.update(neighlist=nl, neighnum=nn, anum=a, alist=al[:a].copy(), xall=xa[:a].copy())
    return out


class SnapMD:
    """NVE molecular dynamics with SNAP forces on one GPU."""

    def __init__(self, params: SnapParams, box, natoms: int, dt: float, mass: float = TA_MASS,
                 skin: float = 1.0, neighmax: int = 64, precision: str = "fp64", device: int = 0,
                 neighevery: int = 1, neighdelay: int = 0, neighcheck: int = 1):
        L = _lib.lib()
        self._sp, self._keep = _lib.snap_params_c(params)
        cfg = _lib.MDConfigC()
        cfg.natoms = natoms
        cfg.box[:] = list(_box9(box))
        cfg.mass, cfg.dt, cfg.skin = mass, dt, skin
        cfg.neighmax, cfg.neighevery, cfg.neighdelay, cfg.neighcheck = neighmax, neighevery, neighdelay, neighcheck
        cfg.precision, cfg.device = PREC[precision], device
        self.natoms = natoms
        self._h = C.c_void_p()
        _lib.check(L.mdp_md_create(C.byref(self._h), C.byref(self._sp), C.byref(cfg)), "mdp_md_create")

    def close(self):
        if self._h:
            _lib.lib().mdp_md_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_state(self, x: np.ndarray, v: np.ndarray):
        _lib.check(_lib.lib().mdp_md_set_state(self._h, np.ascontiguousarray(x, dtype=np.float64),
                                               np.ascontiguousarray(v, dtype=np.float64)), "mdp_md_set_state")

    def set_types(self, types: np.ndarray):
        """Atom types 1..nelements (models with several element types)."""
        _lib.check(_lib.lib().mdp_md_set_types(self._h, np.ascontiguousarray(types, dtype=np.int32)),
                   "mdp_md_set_types")

    def set_state_device(self, x_ptr: int, v_ptr: int):
        _lib.check(_lib.lib().mdp_md_set_state_device(self._h, C.c_void_p(x_ptr), C.c_void_p(v_ptr)),
                   "mdp_md_set_state_device")

    def setup(self):
        _lib.check(_lib.lib().mdp_md_setup(self._h), "mdp_md_setup")

    def run(self, nsteps: int, thermo_every: int = 0):
        """Runs nsteps; returns (thermo rows (k,5), elapsed ms on the device)."""
        cap = nsteps // thermo_every + 1 if thermo_every > 0 else 0
        th = np.zeros((max(cap, 1), 5))
        nrows = C.c_int(0)
        ms = C.c_float(0.0)
        _lib.check(_lib.lib().mdp_md_run(self._h, int(nsteps), int(thermo_every), th.ctypes.data, cap,
                                         C.byref(nrows), C.byref(ms)), "mdp_md_run")
        return th[: nrows.value].copy(), float(ms.value)

    def state(self):
        n = self.natoms
        x = np.zeros((n, 3)); v = np.zeros((n, 3)); f = np.zeros((n, 3)); e = np.zeros(n)
        _lib.check(_lib.lib().mdp_md_get_state(self._h, x.ctypes.data, v.ctypes.data, f.ctypes.data,
                                               e.ctypes.data), "mdp_md_get_state")
        return x, v, f, e

    def upload(self, x_ptr: int, v_ptr: int):
        """Async H2D of positions/velocities (AoS, host pointers) on the engine stream."""
        _lib.check(_lib.lib().mdp_md_upload(self._h, C.c_void_p(x_ptr), C.c_void_p(v_ptr)), "mdp_md_upload")

    def download(self, f_ptr: int, e_ptr: int):
        """Async D2H of forces (AoS) and per-atom energies on the engine stream."""
        _lib.check(_lib.lib().mdp_md_download(self._h, C.c_void_p(f_ptr), C.c_void_p(e_ptr)), "mdp_md_download")

    def sync(self):
        _lib.check(_lib.lib().mdp_md_sync(self._h), "mdp_md_sync")

    def thermo(self) -> np.ndarray:
        out = np.zeros(5)
        _lib.check(_lib.lib().mdp_md_thermo(self._h, out), "mdp_md_thermo")
        return out

    def counters(self) -> dict:
        out = np.zeros(5, dtype=np.int64)
        _lib.check(_lib.lib().mdp_md_counters(self._h, out), "mdp_md_counters")
        return dict(steps=int(out[0]), rebuilds=int(out[1]), pairs=int(out[2]), ghosts=int(out[3]),
                    neighbors=int(out[4]))

    def set_zbl(self, inner: float = 4.0, outer: float = 4.8, z: float = 73.0):
        """Add the ZBL pair term of MDP's snapTA06A example (defaults: its Ta
        parameters); z <= 0 removes it.  Call setup() afterwards."""
        _lib.check(_lib.lib().mdp_md_set_zbl(self._h, float(inner), float(outer), float(z)), "mdp_md_set_zbl")

    def set_surrogate(self, sur, judge_every: int = 50, tol: float = 0.05):
        """Drive the forces by a trained surrogate (None: the plain model), judged
        every judge_every steps against the plain model with force-RMSE tolerance tol."""
        _lib.check(_lib.lib().mdp_md_set_surrogate(self._h, None if sur is None else sur.handle, int(judge_every),
                                                   float(tol)), "mdp_md_set_surrogate")

    def surrogate_status(self, cap: int = 4096) -> dict:
        act = C.c_int(0); fb = C.c_longlong(-1); nj = C.c_int(0)
        log = np.zeros(2 * cap)
        _lib.check(_lib.lib().mdp_md_surrogate_status(self._h, C.byref(act), C.byref(fb), C.byref(nj),
                                                      log.ctypes.data, cap), "mdp_md_surrogate_status")
        k = min(nj.value, cap)
        return dict(active=bool(act.value), fallback_step=int(fb.value), judgements=int(nj.value),
                    log=log[: 2 * k].reshape(k, 2))

    def stage_timing(self, enable: bool):
        _lib.check(_lib.lib().mdp_md_stage_timing(self._h, int(enable)), "mdp_md_stage_timing")

    def stage_times(self) -> dict:
        ms = np.zeros(6)
        calls = C.c_longlong(0)
        _lib.check(_lib.lib().mdp_md_stage_times(self._h, ms, C.byref(calls)), "mdp_md_stage_times")
        names = ["pairs", "ui", "yi", "fi", "tally", "force"]
        return dict(zip(names, ms.tolist()), calls=int(calls.value))

    @property
    def stream(self) -> int:
        return int(_lib.lib().mdp_md_stream(self._h) or 0)


def launch_count() -> int:
    return int(_lib.lib().mdp_launch_count())


def probe_fma_peak(device: int = 0) -> tuple[float, float]:
    a = C.c_double(0.0); b = C.c_double(0.0)
    _lib.check(_lib.lib().mdp_probe_fma_peak(device, C.byref(a), C.byref(b)), "mdp_probe_fma_peak")
    return a.value, b.value

"""ctypes front-end of the CPU checkers.  TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline / reference
legs import this module.  It loads

* ``_build/liboracle.so`` -- the C restatement (oracle/hydro_oracle.c) of the
  HydroC99_2Domp time step; built on demand with gcc (``make -C oracle``);
* ``_ref/libhydroref.so`` -- the reference's own objects behind a small harness
  (oracle/ref_shim.c), present only where the reference sources were available
  to compile (``make -C oracle ref``);
* ``_ref/libhydroref_sp.so`` -- the same objects built single precision
  (the reference's ``SP=O`` option, ``-DPREC_SP``), the context figure for the
  mixed-precision form's error against FP64.

Both take the same flat parameter record (oracle/orc_param.h).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import threading

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_ORACLE = os.path.join(HERE, "_build", "liboracle.so")
_LIB_REF = os.path.join(HERE, "_ref", "libhydroref.so")
_LIB_REF_SP = os.path.join(HERE, "_ref", "libhydroref_sp.so")
_lock = threading.Lock()


class OrcParam(C.Structure):
    """Mirror of orc_param_t (oracle/orc_param.h)."""

    _fields_ = [
        ("nx", C.c_int), ("ny", C.c_int),
        ("boundary_left", C.c_int), ("boundary_right", C.c_int),
        ("boundary_down", C.c_int), ("boundary_up", C.c_int),
        ("iorder", C.c_int), ("scheme", C.c_int), ("niter_riemann", C.c_int),
        ("slope_type", C.c_double), ("gamma", C.c_double), ("smallr", C.c_double),
        ("smallc", C.c_double), ("dx", C.c_double), ("courant_factor", C.c_double),
    ]


def make_param(nx, ny, dx=None, boundary=(1, 1, 1, 1), iorder=2, scheme=1, niter_riemann=10,
               slope_type=1.0, gamma=1.4, smallr=1e-10, smallc=1e-10, courant_factor=0.8):
    """boundary = (left, right, down, up), the reference's boundary_* keys."""
    p = OrcParam()
    p.nx, p.ny = nx, ny
    p.boundary_left, p.boundary_right, p.boundary_down, p.boundary_up = boundary
    p.iorder, p.scheme, p.niter_riemann = iorder, scheme, niter_riemann
    p.slope_type, p.gamma, p.smallr, p.smallc = slope_type, gamma, smallr, smallc
    p.dx = (1.0 / nx) if dx is None else dx
    p.courant_factor = courant_factor
    return p


_DP = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_P = C.POINTER(OrcParam)


def _build_oracle():
    subprocess.run(["make", "-s", "-C", HERE, "_build/liboracle.so"], check=True)


_oracle = None
_ref: dict = {}


def oracle_lib():
    global _oracle
    with _lock:
        if _oracle is None:
            if not os.path.exists(_LIB_ORACLE):
                _build_oracle()
            lib = C.CDLL(_LIB_ORACLE)
            lib.orc_init.argtypes = [_P, C.c_int, _DP]
            lib.orc_init.restype = C.c_int
            lib.orc_make_boundary.argtypes = [_P, C.c_int, _DP]
            lib.orc_godunov.argtypes = [_P, C.c_int, C.c_double, _DP]
            lib.orc_sweep.argtypes = [_P, C.c_int, C.c_double, _DP]
            lib.orc_courant.argtypes = [_P, _DP, C.POINTER(C.c_double), C.POINTER(C.c_double)]
            lib.orc_courant.restype = C.c_double
            lib.orc_run.argtypes = [_P, _DP, C.c_int, C.c_double, C.c_void_p,
                                    C.POINTER(C.c_double)]
            lib.orc_run.restype = C.c_int
            lib.orc_set_threads.argtypes = [C.c_int]
            lib.orc_set_threads.restype = C.c_int
            _oracle = lib
    return _oracle


def ref_available(sp: bool = False) -> bool:
    return os.path.exists(_LIB_REF_SP if sp else _LIB_REF)


def ref_lib(sp: bool = False):
    """The reference harness; ``sp`` selects the single-precision build.  The
    state crosses it as doubles either way."""
    with _lock:
        if sp not in _ref:
            lib = C.CDLL(_LIB_REF_SP if sp else _LIB_REF)
            lib.ref_create.argtypes = [_P, C.c_int, C.c_int]
            lib.ref_create.restype = C.c_void_p
            lib.ref_destroy.argtypes = [C.c_void_p]
            lib.ref_get.argtypes = [C.c_void_p, _DP]
            lib.ref_set.argtypes = [C.c_void_p, _DP]
            lib.ref_compute_deltat.argtypes = [C.c_void_p]
            lib.ref_compute_deltat.restype = C.c_double
            lib.ref_godunov.argtypes = [C.c_void_p, C.c_int, C.c_double]
            lib.ref_make_boundary.argtypes = [C.c_void_p, C.c_int]
            lib.ref_vtkfile.argtypes = [C.c_void_p, C.c_int]
            lib.ref_run.argtypes = [C.c_void_p, C.c_int, C.c_double, C.c_void_p,
                                    C.POINTER(C.c_double), C.POINTER(C.c_double),
                                    C.POINTER(C.c_double)]
            lib.ref_run.restype = C.c_int
            lib.ref_param_layout.argtypes = [C.POINTER(C.c_long), C.c_int]
            lib.ref_param_layout.restype = C.c_int
            lib.ref_real_size.restype = C.c_int
            if lib.ref_real_size() != (4 if sp else 8):
                raise RuntimeError(f"{lib._name}: real_t of {lib.ref_real_size()} bytes")
            _ref[sp] = lib
    return _ref[sp]


def state_shape(p: OrcParam):
    return (4, p.ny + 4, p.nx + 4)


# ----------------------------------------------------------------- restatement
def init_state(p: OrcParam, testcase: int) -> np.ndarray:
    u = np.zeros(state_shape(p), dtype=np.float64)
    rc = oracle_lib().orc_init(C.byref(p), testcase, u)
    if rc != 0:
        raise ValueError(f"testcase {testcase} not implemented")
    return u


def godunov(p: OrcParam, idim: int, dt: float, u: np.ndarray) -> None:
    oracle_lib().orc_godunov(C.byref(p), idim, dt, u)


def sweep(p: OrcParam, idim: int, dt: float, u: np.ndarray) -> None:
    """make_boundary(idim) and one sweep (hydro_godunov.c:74-139)."""
    oracle_lib().orc_sweep(C.byref(p), idim, dt, u)


def make_boundary(p: OrcParam, idim: int, u: np.ndarray) -> None:
    oracle_lib().orc_make_boundary(C.byref(p), idim, u)


def courant(p: OrcParam, u: np.ndarray):
    cx, cy = C.c_double(), C.c_double()
    dt = oracle_lib().orc_courant(C.byref(p), u, C.byref(cx), C.byref(cy))
    return dt, cx.value, cy.value


def run(p: OrcParam, u: np.ndarray, nstepmax: int, tend: float = 1e300, threads: int = 0):
    """main.c:344-408 on the restatement.  Returns (nsteps, dts, t)."""
    lib = oracle_lib()
    if threads:
        lib.orc_set_threads(threads)
    dts = np.zeros(max(nstepmax, 1), dtype=np.float64)
    t = C.c_double()
    n = lib.orc_run(C.byref(p), u, nstepmax, tend, dts.ctypes.data, C.byref(t))
    return n, dts[:n].copy(), t.value


# ------------------------------------------------------------------ reference
class RefState:
    """The reference's own state, work space and driver loop (oracle/_ref)."""

    def __init__(self, p: OrcParam, testcase: int, nxystep: int = -1, sp: bool = False):
        self.p = p
        self.lib = ref_lib(sp)
        self.h = self.lib.ref_create(C.byref(p), testcase, nxystep)

    def get(self) -> np.ndarray:
        u = np.empty(state_shape(self.p), dtype=np.float64)
        self.lib.ref_get(self.h, u)
        return u

    def set(self, u: np.ndarray) -> None:
        self.lib.ref_set(self.h, np.ascontiguousarray(u, dtype=np.float64))

    def compute_deltat(self) -> float:
        return self.lib.ref_compute_deltat(self.h)

    def godunov(self, idim: int, dt: float) -> None:
        self.lib.ref_godunov(self.h, idim, dt)

    def make_boundary(self, idim: int) -> None:
        self.lib.ref_make_boundary(self.h, idim)

    def vtkfile(self, step: int) -> None:
        """vtkfile.c on the state, writing into the current directory."""
        self.lib.ref_vtkfile(self.h, step)

    def run(self, nstepmax: int, tend: float = 1e300):
        dts = np.zeros(max(nstepmax, 1), dtype=np.float64)
        t, mcs, el = C.c_double(), C.c_double(), C.c_double()
        n = self.lib.ref_run(self.h, nstepmax, tend, dts.ctypes.data, C.byref(t), C.byref(mcs),
                             C.byref(el))
        return n, dts[:n].copy(), t.value, mcs.value, el.value

    def close(self):
        if self.h:
            self.lib.ref_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def ref_param_layout():
    out = (C.c_long * 64)()
    n = ref_lib().ref_param_layout(out, 64)
    return [out[i] for i in range(n)]

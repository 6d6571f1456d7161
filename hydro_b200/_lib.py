"""ctypes binding of libhydro_b200.so (include/hydro_b200.h).

The structures mirror the reference's parametres.h:31-122 field for field
(hydroparam_t is passed by value to the reference entry points, so its layout
is part of the ABI; tests/test_abi.py checks it against the reference).

Loading fails loudly: there is no CPU fallback for any entry point.
"""
from __future__ import annotations

import ctypes as C
import os

PKG_DIR = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG_DIR, "libhydro_b200.so")

# Boxes of parametres.h:20-29.
MAX_BOX = 8

HB_OK, HB_ERR_ARG, HB_ERR_CUDA, HB_ERR_NODEV, HB_ERR_NOMEM, HB_ERR_STATE, HB_ERR_TIMEOUT = range(7)
HB_PREC_FP64, HB_PREC_MIXED, HB_PREC_FP64_FMA = 0, 1, 2
PRECISIONS = {"fp64": HB_PREC_FP64, "mixed": HB_PREC_MIXED, "fma": HB_PREC_FP64_FMA}
HB_XSWEEP_MARCH, HB_XSWEEP_CELL = 0, 1
HB_NOALLOC_MAX_CELLS = 1 << 20  # include/hydro_b200.h
XSWEEPS = {"march": HB_XSWEEP_MARCH, "cell": HB_XSWEEP_CELL}
HB_KERNEL_AUTO, HB_KERNEL_MARCH, HB_KERNEL_WARP, HB_KERNEL_COOP, HB_KERNEL_COOP8 = -1, 0, 1, 2, 3
HB_KERNEL_BULK = 4
KERNELS = {"auto": HB_KERNEL_AUTO, "march": HB_KERNEL_MARCH, "warp": HB_KERNEL_WARP,
           "coop": HB_KERNEL_COOP, "coop8": HB_KERNEL_COOP8, "bulk": HB_KERNEL_BULK}


class HydroParam(C.Structure):
    """hydroparam_t (parametres.h:31-80)."""

    _fields_ = [
        ("prt", C.c_int),
        ("t", C.c_double), ("tend", C.c_double),
        ("nstep", C.c_int), ("nstepmax", C.c_int),
        ("noutput", C.c_int),
        ("dtoutput", C.c_double),
        ("nimage", C.c_int),
        ("dtimage", C.c_double),
        ("imin", C.c_int), ("imax", C.c_int), ("jmin", C.c_int), ("jmax", C.c_int),
        ("nx", C.c_int), ("ny", C.c_int), ("nxt", C.c_int), ("nyt", C.c_int),
        ("nxyt", C.c_int), ("nxystep", C.c_int),
        ("nproc", C.c_int), ("mype", C.c_int),
        ("globnx", C.c_int), ("globny", C.c_int),
        ("box", C.c_int * MAX_BOX),
        ("nvar", C.c_int),
        ("dx", C.c_double),
        ("gamma", C.c_double),
        ("courant_factor", C.c_double),
        ("smallc", C.c_double), ("smallr", C.c_double),
        ("niter_riemann", C.c_int),
        ("iorder", C.c_int),
        ("slope_type", C.c_double),
        ("scheme", C.c_int),
        ("boundary_right", C.c_int), ("boundary_left", C.c_int),
        ("boundary_down", C.c_int), ("boundary_up", C.c_int),
        ("testCase", C.c_int),
        ("shrinkSize", C.c_int),
        ("shrink", C.c_int),
        ("fp", C.c_void_p),
    ]


class HydroVar(C.Structure):
    """hydrovar_t (parametres.h:87-89)."""

    _fields_ = [("uold", C.POINTER(C.c_double))]


class HydroVarWork(C.Structure):
    """hydrovarwork_t (parametres.h:97-100); ignored by the device path."""

    _fields_ = [(n, C.POINTER(C.c_double)) for n in
                ("u", "q", "qxm", "qxp", "dq", "qleft", "qright", "qgdnv", "flux")]


class HydroWork(C.Structure):
    """hydrowork_t (parametres.h:107-122); ignored by the device path."""

    _fields_ = (
        [(n, C.POINTER(C.c_double)) for n in ("c", "e", "tmpm1", "tmpm2",
                                               "rl", "ul", "pl", "cl", "wl",
                                               "rr", "ur", "pr", "cr", "wr",
                                               "ro", "uo", "po", "co", "wo",
                                               "rstar", "ustar", "pstar", "cstar",
                                               "spin", "spout", "ushock")]
        + [("sgnm", C.POINTER(C.c_int)), ("goon", C.POINTER(C.c_int))]
        + [(n, C.POINTER(C.c_double)) for n in ("frac", "scr", "delp", "pold")]
        + [("ind", C.POINTER(C.c_int)), ("ind2", C.POINTER(C.c_int))]
    )


# Every function include/hydro_b200.h declares: (name, restype, argtypes).
_P = C.POINTER(HydroParam)
_V = C.POINTER(HydroVar)
_W = C.POINTER(HydroWork)
_VW = C.POINTER(HydroVarWork)
_D = C.c_void_p  # hb_domain*
_DP = C.POINTER(C.c_double)

SIGNATURES = [
    ("hydro_godunov", None, [C.c_int, C.c_double, HydroParam, _V, _W, _VW]),
    ("compute_deltat", None, [_DP, HydroParam, _W, _V, _VW]),
    ("make_boundary", None, [C.c_int, HydroParam, _V]),
    ("compute_deltat_init_mem", None, [HydroParam, _W, _VW]),
    ("compute_deltat_clean_mem", None, [HydroParam, _W, _VW]),
    ("hydro_b200_last_error", C.c_int, []),
    ("hydro_b200_last_error_message", C.c_char_p, []),
    ("hydro_b200_clear_error", None, []),
    ("hydro_b200_sync_to_host", C.c_int, [_P, _V]),
    ("hydro_b200_sync_to_device", C.c_int, [_P, _V]),
    ("hydro_b200_release", C.c_int, [_V]),
    ("hydro_b200_mirror_stream", C.c_void_p, [_P, _V]),
    ("hydro_b200_run", C.c_int, [_P, _V, C.c_int, C.c_double, _DP, C.POINTER(C.c_int), _DP,
                                 _DP]),
    ("hydro_b200_domain_create", _D, [_P]),
    ("hydro_b200_domain_destroy", None, [_D]),
    ("hydro_b200_domain_state", C.c_void_p, [_D]),
    ("hydro_b200_domain_stream", C.c_void_p, [_D]),
    ("hydro_b200_domain_upload", C.c_int, [_D, C.c_void_p]),
    ("hydro_b200_domain_download", C.c_int, [_D, C.c_void_p]),
    ("hydro_b200_domain_synchronize", C.c_int, [_D]),
    ("hydro_b200_domain_godunov", C.c_int, [_D, C.c_int, C.c_double, C.c_int]),
    ("hydro_b200_domain_make_boundary", C.c_int, [_D, C.c_int]),
    ("hydro_b200_domain_courant", C.c_int, [_D, _DP, _DP]),
    ("hydro_b200_domain_sweep", C.c_int, [_D, C.c_int, C.c_int, C.c_double, C.c_int]),
    ("hydro_b200_domain_halo_count", C.c_longlong, [_D, C.c_int]),
    ("hydro_b200_domain_halo_pack", C.c_int, [_D, C.c_int, C.c_int, C.c_int, C.c_void_p]),
    ("hydro_b200_domain_halo_unpack", C.c_int, [_D, C.c_int, C.c_int, C.c_void_p]),
    ("hydro_b200_vtk_base64_len", C.c_longlong, [C.c_int, C.c_int]),
    ("hydro_b200_domain_vtk_base64", C.c_int, [_D, C.c_int, C.c_void_p, C.c_longlong]),
    ("vtkfile", None, [C.c_int, HydroParam, _V]),
    ("hydro_b200_domain_set_clock", C.c_int, [_D, C.c_double, C.c_int, C.c_double]),
    ("hydro_b200_domain_launch_steps", C.c_int, [_D, C.c_int, C.c_int, C.c_double]),
    ("hydro_b200_domain_get_clock", C.c_int, [_D, _DP, C.POINTER(C.c_int), _DP]),
    ("hydro_b200_domain_get_dts", C.c_int, [_D, _DP, C.c_int]),
    ("hydro_b200_domain_reserve_dts", C.c_int, [_D, C.c_int]),
    ("hydro_b200_domain_launch_count", C.c_longlong, [_D]),
    ("hydro_b200_domain_set_precision", C.c_int, [_D, C.c_int]),
    ("hydro_b200_domain_set_xsweep", C.c_int, [_D, C.c_int, C.c_int]),
    ("hydro_b200_domain_set_kernel", C.c_int, [_D, C.c_int, C.c_int, C.c_int]),
    ("hydro_b200_domain_sweep_part", C.c_int, [_D, C.c_int, C.c_int, C.c_double, C.c_int,
                                                C.c_int]),
    ("hydro_b200_domain_get_kernel", C.c_int, [_D, C.c_int, C.c_int]),
    ("hydro_b200_domain_profile", C.c_int, [_D, C.c_int]),
    ("hydro_b200_domain_profile_read", C.c_int, [_D, _DP, C.POINTER(C.c_longlong), C.c_int]),
    ("hydro_b200_batch_create", _D, [_P, C.c_int, C.c_size_t, C.c_int]),
    ("hydro_b200_batch_destroy", None, [_D]),
    ("hydro_b200_batch_bytes_needed", C.c_longlong, [_P]),
    ("hydro_b200_batch_arena_free", C.c_longlong, [_D]),
    ("hydro_b200_batch_add", C.c_int, [_D, _P, C.c_void_p, C.c_double, C.c_int]),
    ("hydro_b200_batch_add_resume", C.c_int, [_D, _P, C.c_void_p, C.c_double, C.c_double,
                                              C.c_int]),
    ("hydro_b200_batch_add_blast", C.c_int, [_D, _P, C.c_double, C.c_double, C.c_int, C.c_int,
                                             C.c_double, C.c_double, C.c_int]),
    ("hydro_b200_batch_remove", C.c_int, [_D, C.c_int]),
    ("hydro_b200_batch_steps", C.c_int, [_D, C.c_int]),
    ("hydro_b200_batch_synchronize", C.c_int, [_D]),
    ("hydro_b200_batch_status", C.c_int, [_D, C.c_int, _DP, C.POINTER(C.c_int), _DP,
                                          C.POINTER(C.c_int), C.POINTER(C.c_longlong)]),
    ("hydro_b200_batch_poll", C.c_int, [_D, C.POINTER(C.c_int), C.c_int]),
    ("hydro_b200_batch_table", C.c_int, [_D, C.POINTER(C.c_int), C.POINTER(C.c_int), _DP,
                                         C.c_int]),
    ("hydro_b200_batch_download", C.c_int, [_D, C.c_int, C.c_void_p]),
    ("hydro_b200_batch_global_step", C.c_longlong, [_D]),
    ("hydro_b200_batch_launch_count", C.c_longlong, [_D]),
    ("hydro_b200_batch_stream", C.c_void_p, [_D]),
    ("hydro_b200_batch_set_tuning", C.c_int, [_D, C.c_int, C.c_int, C.c_int, C.c_int]),
    ("hydro_b200_batch_get_tuning", C.c_int, [_D, C.POINTER(C.c_int), C.POINTER(C.c_int),
                                              C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    ("hydro_b200_batch_autotune", C.c_int, [_D, C.c_int]),
    ("hydro_b200_set_device", C.c_int, [C.c_int]),
    ("hydro_b200_godunov_noalloc", C.c_int, [_P, C.c_void_p, C.c_int, C.c_double, C.c_void_p]),
    ("hydro_b200_build_info", C.c_char_p, []),
]

_lib = None


class HydroB200Error(RuntimeError):
    pass


def load() -> C.CDLL:
    """Load the in-tree library; raise if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise HydroB200Error(
                f"{LIB_PATH} is missing: build it with `make -C hydro_b200/csrc` "
                "(or __graft_entry__.build()); there is no CPU fallback")
        lib = C.CDLL(LIB_PATH)
        for name, res, args in SIGNATURES:
            f = getattr(lib, name)
            f.restype = res
            f.argtypes = args
        _lib = lib
    return _lib


def check(rc: int | None = None) -> None:
    """Raise HydroB200Error if the library recorded an error."""
    lib = load()
    err = lib.hydro_b200_last_error()
    if err != HB_OK or (rc is not None and rc not in (0,) and rc < 0):
        msg = lib.hydro_b200_last_error_message().decode(errors="replace")
        lib.hydro_b200_clear_error()
        raise HydroB200Error(f"hydro_b200 error {err}: {msg}")

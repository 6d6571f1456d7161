"""hydro_b200 -- B200 (sm_100a) implementation of HydroC's dimensionally split
Godunov/MUSCL time step behind the reference's C entry points.

The product is libhydro_b200.so (hydro_b200/csrc, C ABI in
include/hydro_b200.h).  This package is its Python host side: the ctypes
binding, the reference's .nml parameter handling and the run drivers.
"""
from ._lib import (HydroB200Error, HydroParam, HydroVar, HydroVarWork, HydroWork, LIB_PATH,
                   load)
from .params import (HSCHEME_COLLELA, HSCHEME_MUSCL, HSCHEME_PLMDE, default_params, finalize,
                     init_state, make_params, read_nml, state_shape)
from .solver import Domain, HydroRun
from .batch import Batch, make_blast_mix

__all__ = [
    "HydroB200Error", "HydroParam", "HydroVar", "HydroVarWork", "HydroWork", "LIB_PATH", "load",
    "HSCHEME_COLLELA", "HSCHEME_MUSCL", "HSCHEME_PLMDE", "default_params", "finalize",
    "init_state", "make_params", "read_nml", "state_shape", "Domain", "HydroRun",
    "Batch", "make_blast_mix",
]

"""Run parameters: the reference's .nml parameter set and initial states.

Mirrors HydroC/HydroC99_2Domp/Src/parametres.c (defaults :22-71, the
key=value reader :73-228, the nxystep rule :333-341) and the single-process
set-up of hydro_funcs.c:15-40 and the test cases of :42-110, producing the
hydroparam_t record (hydro_b200._lib.HydroParam) the C ABI takes by value.
"""
from __future__ import annotations

import re

import numpy as np

from ._lib import HydroParam, MAX_BOX

HSCHEME_MUSCL, HSCHEME_PLMDE, HSCHEME_COLLELA = 1, 2, 3
_SCHEMES = {"muscl": HSCHEME_MUSCL, "plmde": HSCHEME_PLMDE, "collela": HSCHEME_COLLELA}
INT_MAX = 2**31 - 1

_INT_KEYS = ("nstepmax", "prt", "nx", "ny", "nxystep", "boundary_left", "boundary_right",
             "boundary_up", "boundary_down", "niter_riemann", "noutput", "nimage", "iorder")
_REAL_KEYS = ("slope_type", "tend", "dx", "courant_factor", "smallr", "smallc", "dtoutput",
              "dtimage")


def default_params() -> HydroParam:
    """parametres.c:22-71."""
    H = HydroParam()
    H.prt = 0
    H.nx = 20
    H.ny = 20
    H.globnx, H.globny = H.nx, H.ny
    H.nproc, H.mype = 1, 0
    for b in range(MAX_BOX):
        H.box[b] = -1
    H.nxystep = -1
    H.nvar = 4
    H.dx = 1.0
    H.t = 0.0
    H.nstep = 0
    H.tend = 0.0
    H.gamma = 1.4
    H.courant_factor = 0.5
    H.smallc = 1e-10
    H.smallr = 1e-10
    H.niter_riemann = 10
    H.iorder = 2
    H.slope_type = 1.0
    H.scheme = HSCHEME_MUSCL
    H.boundary_right = H.boundary_left = H.boundary_up = H.boundary_down = 1
    H.noutput = 0
    H.nstepmax = INT_MAX
    H.dtoutput = 0.0
    H.testCase = 0
    H.shrink = 1
    H.shrinkSize = 1000
    H.nimage = 0
    H.dtimage = 0.0
    return H


_INT_RE = re.compile(r"\s*([+-]?\d+)")
_REAL_RE = re.compile(r"\s*([+-]?(?:\d+\.?\d*(?:[eE][+-]?\d+)?|\.\d+(?:[eE][+-]?\d+)?|inf|nan))",
                      re.IGNORECASE)


def _keyval(line: str):
    """parametres.c:73-98: key up to the first blank after leading blanks,
    value = everything after the first '=' (newline cut)."""
    line = line.split("\n", 1)[0]
    key = line.lstrip(" \t")
    val = None
    if "=" in key:
        key, val = key.split("=", 1)
    key = re.split(r"[ \t]", key, maxsplit=1)[0]
    return key, val


def apply_nml_text(H: HydroParam, text: str) -> HydroParam:
    """parametres.c:100-228: known keys are read with sscanf, anything else
    (section lines, comments, unknown keys) is ignored."""
    for raw in text.splitlines():
        key, val = _keyval(raw[:1023])
        if val is None:
            val = ""
        if key in _INT_KEYS:
            m = _INT_RE.match(val)
            if m:
                setattr(H, key, int(m.group(1)))
        elif key in _REAL_KEYS:
            m = _REAL_RE.match(val)
            if m:
                setattr(H, key, float(m.group(1)))
        elif key == "testcase":
            m = _INT_RE.match(val)
            if m:
                H.testCase = int(m.group(1))
        elif key == "scheme":
            if val not in _SCHEMES:
                raise ValueError(f"Scheme name <{val}> is unknown, should be one of "
                                 "[muscl,plmde,collela]")
            H.scheme = _SCHEMES[val]
    return H


def finalize(H: HydroParam) -> HydroParam:
    """parametres.c:307-341 (single process) and hydro_funcs.c:19-33."""
    H.globnx, H.globny = H.nx, H.ny
    H.box[0], H.box[1], H.box[2], H.box[3] = 0, H.nx, 0, H.ny
    if H.nxystep == -1:
        H.nxystep = min(H.nx, H.ny)
    else:
        H.nxystep = min(H.nxystep, H.nx, H.ny)
    H.imin = H.jmin = 0
    H.imax = H.nx + 4
    H.jmax = H.ny + 4
    H.nxt = H.imax - H.imin
    H.nyt = H.jmax - H.jmin
    H.nxyt = max(H.nxt, H.nyt)
    return H


def read_nml(path: str) -> HydroParam:
    with open(path, "r", errors="replace") as f:
        return finalize(apply_nml_text(default_params(), f.read()))


def make_params(nx: int, ny: int, *, dx: float | None = None, tend: float = 0.0,
                nstepmax: int = INT_MAX, courant_factor: float = 0.8, niter_riemann: int = 10,
                iorder: int = 2, slope_type: float = 1.0, scheme: int = HSCHEME_MUSCL,
                boundary=(1, 1, 1, 1), testcase: int = 0, gamma: float = 1.4,
                smallr: float = 1e-10, smallc: float = 1e-10, nxystep: int = -1) -> HydroParam:
    """Parameter record from keyword arguments (boundary = left, right, down, up)."""
    H = default_params()
    H.nx, H.ny = nx, ny
    H.dx = (1.0 / nx) if dx is None else dx
    H.tend, H.nstepmax = tend, nstepmax
    H.courant_factor, H.niter_riemann = courant_factor, niter_riemann
    H.iorder, H.slope_type, H.scheme = iorder, slope_type, scheme
    H.boundary_left, H.boundary_right, H.boundary_down, H.boundary_up = boundary
    H.testCase = testcase
    H.gamma, H.smallr, H.smallc = gamma, smallr, smallc
    H.nxystep = nxystep
    return finalize(H)


def state_shape(H: HydroParam):
    """uold[v][j][i] (parametres.h:92-93)."""
    return (4, H.ny + 4, H.nx + 4)


def init_state(H: HydroParam, testcase: int | None = None, out: np.ndarray | None = None):
    """hydro_funcs.c:42-110 for one process: rho = 1, u = v = 0, E = 1e-5 in
    the interior, ghosts 0, and the blast E = one/dx/dx at the padded centre
    (testcase 0), at the corner cell (2, 2) (1) or along the column x = 2 from
    j = 2 up to the last row (2)."""
    tc = H.testCase if testcase is None else testcase
    u = np.zeros(state_shape(H), dtype=np.float64) if out is None else out
    u[...] = 0.0
    u[0, 2:-2, 2:-2] = 1.0
    u[3, 2:-2, 2:-2] = 1e-5
    eblast = 1.0 / H.dx / H.dx
    nxt, nyt = H.nx + 4, H.ny + 4
    if tc == 0:
        u[3, nyt // 2, nxt // 2] = eblast
    elif tc == 1:
        u[3, 2, 2] = eblast
    elif tc == 2:
        u[3, 2:, 2] = eblast
    else:
        raise ValueError("Test case not implemented")
    return u


# ---------------------------------------------------------------- seeded inputs
_SM_GAMMA = np.uint64(0x9E3779B97F4A7C15)
_SM_M1 = np.uint64(0xBF58476D1CE4E5B9)
_SM_M2 = np.uint64(0x94D049BB133111EB)


def splitmix64(x: np.ndarray) -> np.ndarray:
    """SplitMix64 finaliser (Steele, Lea & Flood, OOPSLA 2014) on uint64 counters."""
    with np.errstate(over="ignore"):
        z = x.astype(np.uint64) + _SM_GAMMA
        z = (z ^ (z >> np.uint64(30))) * _SM_M1
        z = (z ^ (z >> np.uint64(27))) * _SM_M2
        return z ^ (z >> np.uint64(31))


def uniform_pm1(seed: int, counters: np.ndarray) -> np.ndarray:
    """U(-1, 1) doubles from SplitMix64(seed XOR counter), 53-bit mantissas."""
    z = splitmix64(np.uint64(seed) ^ counters.astype(np.uint64))
    u = (z >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)
    return 2.0 * u - 1.0


def init_noisy_blast(H: HydroParam, seed: int, amplitude: float = 0.01, testcase: int = 1,
                     var: int = 0):
    """The test-case state with the interior of conserved variable `var`
    (0: density -- the mixed-precision workload's input; 3: total energy)
    scaled by 1 + amplitude * U(-1, 1), U drawn per interior cell
    (counter = j*nx + i, interior coordinates)."""
    u = init_state(H, testcase)
    j, i = np.meshgrid(np.arange(H.ny, dtype=np.uint64), np.arange(H.nx, dtype=np.uint64),
                       indexing="ij")
    noise = uniform_pm1(seed, j * np.uint64(H.nx) + i)
    u[var, 2:-2, 2:-2] *= 1.0 + amplitude * noise
    return u

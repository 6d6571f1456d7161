"""Generate the golden fixtures of tests/golden from the REFERENCE itself.

Run in a container where the reference sources are present (it builds
oracle/_ref/libhydroref.so from them with `make -C oracle ref`):

    python tests/golden/make_golden.py

Outputs (committed):
  ref_runs.npz       final states and dt sequences of small runs of the
                     reference driver loop (main.c:344-408) over every
                     boundary type, test case and scheme;
  ref_c0.json        the 250x125 corner case (100 steps): dt sequence,
                     per-variable exact sums (math.fsum) and the SHA-256 of
                     the final state bytes (ghosts included);
  abi_layout.json    size and field offsets of hydroparam_t as the reference
                     compiles it (parametres.h:31-80);
  nml_parse.json     what the reference's own reader (parametres.c:230-357)
                     makes of each tests/golden/nml/*.nml file.
"""
from __future__ import annotations

import glob
import hashlib
import json
import math
import os
import subprocess
import sys
import ctypes as C

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402

# name: (nx, ny, testcase, nsteps, boundary (l, r, d, u), extra parameters)
SMALL_CASES = {
    "reflect_centre_32x24": (32, 24, 0, 30, (1, 1, 1, 1), {}),
    "absorb_corner_29x35": (29, 35, 1, 30, (2, 2, 2, 2), {}),
    "periodic_centre_31x27": (31, 27, 0, 30, (3, 3, 3, 3), {}),
    "mixed_sod_24x24_plmde": (24, 24, 2, 20, (1, 2, 3, 1), {"scheme": 2}),
    "collela_first_order_30x30": (30, 30, 0, 20, (1, 1, 1, 1), {"scheme": 3, "iorder": 1}),
    "slope_half_niter3_28x20": (28, 20, 0, 24, (1, 1, 1, 1),
                                {"slope_type": 0.5, "niter_riemann": 3}),
    "open_sides_26x22": (26, 22, 0, 16, (0, 1, 0, 1), {}),
}

NML_FIELDS = ["nx", "ny", "nxystep", "nstepmax", "iorder", "niter_riemann", "scheme",
              "boundary_left", "boundary_right", "boundary_down", "boundary_up", "testCase",
              "tend", "dx", "courant_factor", "smallr", "smallc", "slope_type", "gamma"]

LAYOUT_FIELDS = ["sizeof", "prt", "t", "tend", "nstep", "nstepmax", "noutput", "dtoutput",
                 "nimage", "dtimage", "imin", "imax", "jmin", "jmax", "nx", "ny", "nxt", "nyt",
                 "nxyt", "nxystep", "nproc", "mype", "globnx", "globny", "box", "nvar", "dx",
                 "gamma", "courant_factor", "smallc", "smallr", "niter_riemann", "iorder",
                 "slope_type", "scheme", "boundary_right", "boundary_left", "boundary_down",
                 "boundary_up", "testCase", "shrinkSize", "shrink", "fp",
                 "sizeof_hydrovar_t", "sizeof_hydrowork_t", "sizeof_hydrovarwork_t"]


def state_digest(u: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(u, dtype=np.float64).tobytes()).hexdigest()


def exact_sums(u: np.ndarray):
    return [math.fsum(u[v].ravel().tolist()) for v in range(4)]


def main():
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "ref"], check=True)
    out = {}
    for name, (nx, ny, tc, nsteps, bnd, extra) in SMALL_CASES.items():
        p = O.make_param(nx, ny, boundary=bnd, **extra)
        r = O.RefState(p, tc)
        u0 = r.get()
        n, dts, t, _, _ = r.run(nsteps)
        assert n == nsteps
        out[f"{name}__init"] = u0
        out[f"{name}__final"] = r.get()
        out[f"{name}__dts"] = dts
        out[f"{name}__meta"] = np.array([nx, ny, tc, nsteps, *bnd], dtype=np.int64)
        r.close()
    np.savez_compressed(os.path.join(HERE, "ref_runs.npz"), **out)

    p = O.make_param(250, 125, boundary=(1, 1, 1, 1))
    r = O.RefState(p, 1)
    n, dts, t, _, _ = r.run(100)
    u = r.get()
    c0 = {"nx": 250, "ny": 125, "testcase": 1, "nsteps": n, "dx": p.dx, "t": t,
          "dts": [float(x).hex() for x in dts], "sums": [float(s).hex() for s in exact_sums(u)],
          "sha256": state_digest(u),
          "row64_rho": [float(x).hex() for x in u[0, 64, :]],
          "col125_E": [float(x).hex() for x in u[3, :, 125]]}
    r.close()
    with open(os.path.join(HERE, "ref_c0.json"), "w") as f:
        json.dump(c0, f, indent=1)

    lay = O.ref_param_layout()
    with open(os.path.join(HERE, "abi_layout.json"), "w") as f:
        json.dump(dict(zip(LAYOUT_FIELDS, lay)), f, indent=1)

    lib = O.ref_lib()
    lib.ref_parse_nml.argtypes = [C.c_char_p, C.POINTER(C.c_double)]
    lib.ref_parse_nml.restype = C.c_int
    parsed = {}
    for path in sorted(glob.glob(os.path.join(HERE, "nml", "*.nml"))):
        buf = (C.c_double * 32)()
        k = lib.ref_parse_nml(path.encode(), buf)
        parsed[os.path.basename(path)] = dict(zip(NML_FIELDS, [buf[i] for i in range(k)]))
    with open(os.path.join(HERE, "nml_parse.json"), "w") as f:
        json.dump(parsed, f, indent=1)
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    main()

"""Helpers shared by the tests (parameter conversion, comparisons)."""
import numpy as np

from hydro_b200 import make_params


def orc_from_H(O, H):
    """The oracle's flat parameter record from a hydroparam_t mirror."""
    return O.make_param(H.nx, H.ny, dx=H.dx,
                        boundary=(H.boundary_left, H.boundary_right, H.boundary_down,
                                  H.boundary_up),
                        iorder=H.iorder, scheme=H.scheme, niter_riemann=H.niter_riemann,
                        slope_type=H.slope_type, gamma=H.gamma, smallr=H.smallr,
                        smallc=H.smallc, courant_factor=H.courant_factor)


def H_from_meta(nx, ny, tc, bnd, **extra):
    return make_params(nx, ny, boundary=tuple(bnd), testcase=tc, **extra)


def bitwise_equal(a, b) -> bool:
    a = np.ascontiguousarray(a, dtype=np.float64)
    b = np.ascontiguousarray(b, dtype=np.float64)
    return a.shape == b.shape and np.array_equal(a.view(np.uint64), b.view(np.uint64))


def describe_mismatch(a, b, name="state"):
    d = np.abs(a - b)
    idx = np.unravel_index(np.argmax(d), d.shape)
    nbad = int(np.count_nonzero(a.view(np.uint64) != b.view(np.uint64)))
    return f"{name}: {nbad} cells differ bitwise; max |diff| {d[idx]:.3e} at {idx}"

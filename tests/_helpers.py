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


def random_state(nx: int, ny: int, seed: int, kind: str, gamma: float = 1.4) -> np.ndarray:
    """A padded state with every cell drawn at random, to reach the branches
    a blast does not: "rough" -- independent cells (shocks and rarefactions
    in both directions, sonic points, every Riemann sampling case);
    "smooth" -- a smooth field with small noise (Newton converging in several
    iterations); "vacuum" -- rough, plus near-vacuum cells (density below
    smallr, pressure below smallp) and cells whose kinetic energy exceeds E
    (negative internal energy), which trigger the clamps."""
    rng = np.random.default_rng(seed)
    shape = (ny + 4, nx + 4)
    if kind == "smooth":
        y, x = np.meshgrid(np.linspace(0, 1, shape[0]), np.linspace(0, 1, shape[1]), indexing="ij")
        rho = 1.0 + 0.5 * np.sin(6.3 * x + 1.0) * np.cos(4.1 * y) + 0.01 * rng.standard_normal(shape)
        u = 0.8 * np.sin(3.1 * y) + 0.01 * rng.standard_normal(shape)
        v = -0.6 * np.cos(2.7 * x) + 0.01 * rng.standard_normal(shape)
        p = 1.0 + 0.3 * np.cos(5.0 * x * y) + 0.01 * rng.standard_normal(shape)
    else:
        rho = np.exp(rng.uniform(np.log(1e-3), np.log(10.0), shape))
        u = rng.uniform(-3.0, 3.0, shape)
        v = rng.uniform(-3.0, 3.0, shape)
        p = np.exp(rng.uniform(np.log(1e-4), np.log(100.0), shape))
    E = p / (gamma - 1.0) + 0.5 * rho * (u * u + v * v)
    if kind == "vacuum":
        m = rng.random(shape) < 0.08
        rho[m] = 10.0 ** rng.uniform(-14, -11, m.sum())
        E[m] = 10.0 ** rng.uniform(-30, -24, m.sum())
        k = rng.random(shape) < 0.04  # kinetic energy above E: p < 0 before the clamp
        E[k] = 0.25 * 0.5 * rho[k] * (u[k] ** 2 + v[k] ** 2)
    return np.ascontiguousarray(np.stack([rho, rho * u, rho * v, E]))

"""The CPU restatement (oracle/hydro_oracle.c) pinned against the reference:
against the golden fixtures made from the reference's own code
(tests/golden/make_golden.py) and, where the reference was compiled here
(oracle/_ref), against the reference run side by side."""
import hashlib
import json
import math
import os

import numpy as np
import pytest

from _helpers import bitwise_equal, describe_mismatch

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")

CASE_EXTRA = {
    "reflect_centre_32x24": {},
    "absorb_corner_29x35": {},
    "periodic_centre_31x27": {},
    "mixed_sod_24x24_plmde": {"scheme": 2},
    "collela_first_order_30x30": {"scheme": 3, "iorder": 1},
    "slope_half_niter3_28x20": {"slope_type": 0.5, "niter_riemann": 3},
    "open_sides_26x22": {},
}


def _golden_runs():
    z = np.load(os.path.join(GOLDEN, "ref_runs.npz"))
    names = sorted({k.split("__")[0] for k in z.files})
    return z, names


@pytest.mark.parametrize("name", sorted(CASE_EXTRA))
def test_restatement_matches_reference_golden(oracle, name):
    z, names = _golden_runs()
    assert name in names
    nx, ny, tc, nsteps, *bnd = [int(v) for v in z[f"{name}__meta"]]
    p = oracle.make_param(nx, ny, boundary=tuple(bnd), **CASE_EXTRA[name])
    u = oracle.init_state(p, tc)
    assert bitwise_equal(u, z[f"{name}__init"]), "initial state (hydro_funcs.c:15-112)"
    n, dts, _ = oracle.run(p, u, nsteps)
    assert n == nsteps
    assert bitwise_equal(dts, z[f"{name}__dts"]), "dt sequence"
    ref = z[f"{name}__final"]
    assert bitwise_equal(u, ref), describe_mismatch(u, ref)


def test_restatement_matches_reference_c0_golden(oracle):
    with open(os.path.join(GOLDEN, "ref_c0.json")) as f:
        g = json.load(f)
    p = oracle.make_param(g["nx"], g["ny"], boundary=(1, 1, 1, 1))
    assert p.dx == g["dx"]
    u = oracle.init_state(p, g["testcase"])
    n, dts, t = oracle.run(p, u, g["nsteps"])
    assert [float(x).hex() for x in dts] == g["dts"]
    assert hashlib.sha256(u.tobytes()).hexdigest() == g["sha256"]
    assert [math.fsum(u[v].ravel().tolist()).hex() for v in range(4)] == g["sums"]


def test_restatement_is_thread_count_independent(oracle):
    p = oracle.make_param(60, 44, boundary=(1, 1, 1, 1))
    a = oracle.init_state(p, 0)
    b = a.copy()
    oracle.run(p, a, 20, threads=1)
    oracle.run(p, b, 20, threads=4)
    assert bitwise_equal(a, b)


ref_needed = pytest.mark.skipif(
    not __import__("oracle.oracle", fromlist=["x"]).ref_available(),
    reason="reference not compiled here (oracle/_ref)")


@ref_needed
@pytest.mark.parametrize("case", [
    (250, 125, 1, 100, (1, 1, 1, 1), {}),
    (61, 47, 0, 40, (2, 1, 3, 2), {"scheme": 2}),
    (40, 64, 2, 30, (3, 3, 1, 1), {"slope_type": 1.7, "niter_riemann": 2}),
])
def test_restatement_matches_reference_live(oracle, case):
    nx, ny, tc, nsteps, bnd, extra = case
    p = oracle.make_param(nx, ny, boundary=bnd, **extra)
    r = oracle.RefState(p, tc, nxystep=7)
    u = oracle.init_state(p, tc)
    n, dts, _ = oracle.run(p, u, nsteps)
    n2, dts2, _, _, _ = r.run(nsteps)
    ur = r.get()
    r.close()
    assert n == n2 and bitwise_equal(dts, dts2)
    assert bitwise_equal(u, ur), describe_mismatch(u, ur)


@ref_needed
def test_make_boundary_matches_reference_live(oracle):
    rng = np.random.default_rng(5)
    for bnd in [(1, 1, 1, 1), (2, 2, 2, 2), (3, 3, 3, 3), (0, 2, 1, 0)]:
        p = oracle.make_param(23, 19, boundary=bnd)
        r = oracle.RefState(p, 0)
        u = rng.standard_normal(oracle.state_shape(p))
        r.set(u)
        for idim in (1, 2):
            oracle.make_boundary(p, idim, u)
            r.make_boundary(idim)
            assert bitwise_equal(u, r.get()), (bnd, idim)
        r.close()


@ref_needed
@pytest.mark.parametrize("kind,seed,extra", [
    ("rough", 1, {}), ("smooth", 2, {}), ("vacuum", 3, {}),
    ("rough", 4, {"scheme": 2}), ("vacuum", 5, {"scheme": 3, "slope_type": 0.7}),
    ("rough", 6, {"iorder": 1, "niter_riemann": 3}),
])
def test_restatement_matches_reference_on_random_states(oracle, kind, seed, extra):
    """Random states (see _helpers.random_state), 16 steps, both codes from
    the same input: every cell and every dt bit for bit."""
    from _helpers import random_state
    p = oracle.make_param(37, 29, boundary=(1, 2, 3, 1) if seed % 2 else (1, 1, 1, 1), **extra)
    u = random_state(37, 29, seed, kind)
    r = oracle.RefState(p, 0, nxystep=5)
    r.set(u)
    n, dts, _ = oracle.run(p, u, 16)
    n2, dts2, _, _, _ = r.run(16)
    ur = r.get()
    r.close()
    assert np.all(np.isfinite(u))
    assert n == n2 and bitwise_equal(dts, dts2)
    assert bitwise_equal(u, ur), describe_mismatch(u, ur)


@pytest.mark.skipif(
    not __import__("oracle.oracle", fromlist=["x"]).ref_available(sp=True),
    reason="single-precision reference not compiled here (oracle/_ref)")
def test_reference_fp32_build_is_a_single_precision_run(oracle):
    """The reference's all-FP32 build (SP=O, -DPREC_SP), the context figure
    for the mixed form's error: on the 250x125 corner blast (100 steps) its
    state holds float32 values only and stays within single-precision
    distance of the FP64 build, dt sequence included."""
    from hydro_b200.metrics import field_errors
    p = oracle.make_param(250, 125)
    a, b = oracle.RefState(p, 1), oracle.RefState(p, 1, sp=True)
    na, da, *_ = a.run(100)
    nb, db, *_ = b.run(100)
    ua, ub = a.get(), b.get()
    a.close()
    b.close()
    assert na == nb == 100
    assert np.array_equal(ub, ub.astype(np.float32).astype(np.float64))
    assert not np.array_equal(ua, ua.astype(np.float32).astype(np.float64))
    np.testing.assert_allclose(db, da, rtol=1e-5)
    err = field_errors(ub, ua)
    for v in ("rho", "E"):
        assert 0 < err[v]["l1_rel"] < 1e-5, err

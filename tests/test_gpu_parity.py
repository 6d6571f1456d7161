"""Parity of the CUDA path with the oracle (and the reference's golden runs).

The FP64 kernels round every operation once in the reference's order, so the
comparison is bitwise: the state (interior AND ghost cells) and every dt.
The required tolerance (1e-12 relative per cell over the run) is therefore
met with margin 0; the tests assert bit equality and report the first
mismatch otherwise.
"""
import hashlib
import json
import math
import os

import numpy as np
import pytest

from hydro_b200 import Domain, HydroRun, init_state, make_params
from _helpers import bitwise_equal, describe_mismatch, orc_from_H

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def run_oracle(O, H, tc, nsteps, u=None):
    p = orc_from_H(O, H)
    u = O.init_state(p, tc) if u is None else u.copy()
    n, dts, t = O.run(p, u, nsteps)
    return u, dts, t


def test_c0_corner_250x125_matches_reference_golden(product_lib):
    """250x125 corner blast, dx = 1/250, 100 steps: the CPU-runnable case,
    compared with the reference's own run (digest of the full state)."""
    g = json.load(open(os.path.join(GOLDEN, "ref_c0.json")))
    H = make_params(250, 125, testcase=1)
    run = HydroRun(H)
    dts = run.run_host_loop(g["nsteps"])
    u = run.sync_to_host()
    run.close()
    assert [float(x).hex() for x in dts] == g["dts"]
    assert [math.fsum(u[v].ravel().tolist()).hex() for v in range(4)] == g["sums"]
    assert hashlib.sha256(u.tobytes()).hexdigest() == g["sha256"]


CASES = {
    "reflect_centre_32x24": {},
    "absorb_corner_29x35": {},
    "periodic_centre_31x27": {},
    "mixed_sod_24x24_plmde": {"scheme": 2},
    "collela_first_order_30x30": {"scheme": 3, "iorder": 1},
    "slope_half_niter3_28x20": {"slope_type": 0.5, "niter_riemann": 3},
    "open_sides_26x22": {},
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_reference_golden_runs(product_lib, name):
    z = np.load(os.path.join(GOLDEN, "ref_runs.npz"))
    nx, ny, tc, nsteps, *bnd = [int(v) for v in z[f"{name}__meta"]]
    H = make_params(nx, ny, boundary=tuple(bnd), testcase=tc, **CASES[name])
    run = HydroRun(H, z[f"{name}__init"].copy())
    dts = run.run_host_loop(nsteps)
    u = run.sync_to_host()
    run.close()
    assert bitwise_equal(dts, z[f"{name}__dts"])
    assert bitwise_equal(u, z[f"{name}__final"]), describe_mismatch(u, z[f"{name}__final"])


@pytest.mark.parametrize("nx,ny,tc,nsteps,bnd,extra", [
    (37, 41, 0, 40, (1, 1, 1, 1), {}),
    (130, 67, 1, 60, (1, 1, 1, 1), {}),          # several segments per line, ragged last
    (67, 130, 0, 60, (2, 3, 1, 2), {}),
    (200, 3, 2, 20, (1, 1, 1, 1), {}),            # thinnest grid accepted
    (3, 150, 0, 20, (3, 3, 3, 3), {}),
    (96, 96, 0, 50, (1, 1, 1, 1), {"scheme": 3, "courant_factor": 0.5}),
    (80, 50, 0, 30, (1, 1, 1, 1), {"iorder": 1, "niter_riemann": 1}),
    (64, 64, 0, 30, (1, 1, 1, 1), {"niter_riemann": 0}),
])
def test_device_loop_matches_oracle(product_lib, oracle, nx, ny, tc, nsteps, bnd, extra):
    """hydro_b200_run (dt and t on the device) against the oracle (x sweep:
    the default cell-per-lane kernel)."""
    H = make_params(nx, ny, boundary=bnd, testcase=tc, **extra)
    want, wdts, wt = run_oracle(oracle, H, tc, nsteps)
    run = HydroRun(H)
    dts = run.run(nsteps)
    u = run.sync_to_host()
    run.close()
    assert len(dts) == nsteps and bitwise_equal(dts, wdts)
    assert run.t == wt
    assert bitwise_equal(u, want), describe_mismatch(u, want)


@pytest.mark.parametrize("nx,ny,tc,nsteps,bnd,extra", [
    (37, 41, 0, 40, (1, 1, 1, 1), {}),
    (130, 67, 1, 60, (2, 3, 1, 2), {}),
    (29, 35, 1, 30, (2, 2, 2, 2), {}),
    (200, 3, 2, 20, (1, 1, 1, 1), {}),
    (3, 150, 0, 20, (3, 3, 3, 3), {}),
    (80, 50, 0, 30, (0, 1, 0, 1), {"iorder": 1, "scheme": 2}),
    (300, 64, 0, 30, (1, 1, 1, 1), {"slope_type": 0.5}),
])
@pytest.mark.parametrize("kernels", [("march", "march"), ("coop", "coop"), ("coop8", "coop8"),
                                     ("coop", "warp")])
def test_kernel_variants_match_oracle(product_lib, oracle, nx, ny, tc, nsteps, bnd, extra,
                                      kernels):
    """The same with the other sweep kernels: row-marching x sweep (shared-
    memory row ring) and marching y sweep, and the 4- and 8-warp cooperative
    windows, on odd, ragged and 3-cell-thin grids."""
    H = make_params(nx, ny, boundary=bnd, testcase=tc, **extra)
    want, wdts, wt = run_oracle(oracle, H, tc, nsteps)
    d = Domain(H, kernels=kernels)
    d.upload(init_state(H, tc))
    d.set_clock()
    d.launch_steps(nsteps)
    got = d.download()
    d.close()
    assert bitwise_equal(got, want), describe_mismatch(got, want)


def test_device_loop_and_reference_entry_points_agree(product_lib):
    """The library driver and the reference driver over the C ABI give the
    same state; both also stop at tend like main.c:344."""
    H = make_params(90, 70, testcase=0)
    a = HydroRun(H)
    da = a.run_host_loop(33)
    ua = a.sync_to_host().copy()
    a.close()
    b = HydroRun(H)
    db = b.run(33)
    ub = b.sync_to_host()
    b.close()
    assert bitwise_equal(da, db) and bitwise_equal(ua, ub)
    # stop on tend: t after 5 steps
    c = HydroRun(H)
    d5 = c.run(5)
    tend = float(np.sum(d5[:4])) + d5[4] * 0.5  # inside step 5
    c.close()
    d = HydroRun(H)
    dd = d.run(100, tend=tend)
    d.close()
    assert len(dd) == 5


def test_resume_from_odd_step(product_lib, oracle):
    """Splitting a run at an odd step (dt carried over) changes nothing."""
    H = make_params(72, 60, testcase=1)
    want, wdts, _ = run_oracle(oracle, H, 1, 21)
    r = HydroRun(H)
    d1 = r.run(7)
    d2 = r.run(21)
    u = r.sync_to_host()
    r.close()
    assert bitwise_equal(np.concatenate([d1, d2]), wdts)
    assert bitwise_equal(u, want)


@pytest.mark.parametrize("bnd", [(1, 1, 1, 1), (2, 2, 2, 2), (3, 3, 3, 3), (0, 2, 1, 0)])
def test_make_boundary_entry_point(product_lib, oracle, bnd):
    rng = np.random.default_rng(11)
    H = make_params(29, 23, boundary=bnd)
    u = rng.standard_normal((4, 27, 33))
    want = u.copy()
    run = HydroRun(H, u)
    for idim in (1, 2):
        run.make_boundary(idim)
        oracle.make_boundary(orc_from_H(oracle, H), idim, want)
    got = run.sync_to_host()
    run.close()
    assert bitwise_equal(got, want)


def test_single_godunov_both_orders(product_lib, oracle):
    """One hydro_godunov call per order from a perturbed state."""
    rng = np.random.default_rng(3)
    H = make_params(45, 38, testcase=0)
    u0 = init_state(H)
    u0[0, 2:-2, 2:-2] *= 1.0 + 0.05 * rng.uniform(-1, 1, (38, 45))
    u0[1, 2:-2, 2:-2] = 0.01 * rng.standard_normal((38, 45))
    p = orc_from_H(oracle, H)
    for idim in (1, 2):
        want = u0.copy()
        oracle.godunov(p, idim, 1.3e-3, want)
        run = HydroRun(H, u0.copy())
        run.godunov(idim, 1.3e-3)
        got = run.sync_to_host()
        run.close()
        assert bitwise_equal(got, want), (idim, describe_mismatch(got, want))


def test_compute_deltat_fused_equals_standalone(product_lib, oracle):
    """The Courant maxima fused into hydro_godunov(2, ...) equal the
    standalone reduction and the oracle's."""
    H = make_params(100, 80, testcase=0)
    r = HydroRun(H)
    r.run_host_loop(6)  # ends after an odd step: the next compute_deltat uses the fused value
    dt_fused = r.compute_deltat()
    u = r.sync_to_host().copy()
    r.sync_to_device()  # invalidates the cache: standalone reduction
    dt_plain = r.compute_deltat()
    r.close()
    dt_orc, _, _ = oracle.courant(orc_from_H(oracle, H), u)
    assert dt_fused == dt_plain == dt_orc


def test_1024_centre_against_oracle(product_lib, oracle):
    """A grid with many CTAs per sweep (1024^2, 40 steps)."""
    H = make_params(1024, 1024, testcase=0)
    want, wdts, _ = run_oracle(oracle, H, 0, 40)
    d = Domain(H)
    d.upload(init_state(H))
    d.set_clock()
    d.launch_steps(40)
    got = d.download()
    t, n, dt = d.get_clock()
    d.close()
    assert n == 40 and dt == wdts[-1]
    assert bitwise_equal(got, want), describe_mismatch(got, want)


def test_full_size_4096_first_steps_and_conservation(product_lib, oracle):
    """The 4096^2 centred blast: the first 2 steps bitwise against the oracle
    (multi-threaded on the host), and 40 steps of the device loop conserving
    mass and energy with reflecting walls (to summation round-off)."""
    H = make_params(4096, 4096, testcase=0)
    p = orc_from_H(oracle, H)
    u0 = init_state(H)
    want = u0.copy()
    oracle.oracle_lib().orc_set_threads(os.cpu_count() or 1)
    n, wdts, _ = oracle.run(p, want, 2)
    d = Domain(H)
    d.upload(u0)
    d.set_clock()
    d.launch_steps(2)
    got = d.download()
    assert bitwise_equal(got, want), describe_mismatch(got, want)
    m0 = math.fsum(u0[0, 2:-2, 2:-2].ravel().tolist())
    e0 = math.fsum(u0[3, 2:-2, 2:-2].ravel().tolist())
    d.launch_steps(38)
    u = d.download()
    d.close()
    m1 = math.fsum(u[0, 2:-2, 2:-2].ravel().tolist())
    e1 = math.fsum(u[3, 2:-2, 2:-2].ravel().tolist())
    assert abs(m1 - m0) <= 1e-12 * m0
    assert abs(e1 - e0) <= 1e-12 * e0
    assert np.all(np.isfinite(u)) and np.all(u[0, 2:-2, 2:-2] > 0)


def test_full_size_4096_200_steps_against_the_reference(product_lib, reference_4096_200):
    """The 4096^2 centred blast over its whole 200-step run, per cell and per
    dt, against the reference's own C99/OpenMP code (oracle/_ref, built from
    the reference sources), run on all host cores.  Skipped, not downgraded,
    where the reference was not compiled."""
    want, wdts, wt = reference_4096_200
    H = make_params(4096, 4096, testcase=0)
    u0 = init_state(H)
    run = HydroRun(H, u0.copy())
    dts = run.run(200)
    got = run.sync_to_host().copy()
    t_gpu = run.t
    run.close()
    assert len(dts) == 200
    assert bitwise_equal(dts, wdts) and t_gpu == wt
    assert bitwise_equal(got, want), describe_mismatch(got, want)


@pytest.mark.parametrize("kind,seed,nx,ny,extra", [
    ("rough", 11, 37, 29, {}),
    ("smooth", 12, 130, 67, {}),
    ("vacuum", 13, 67, 130, {}),
    ("rough", 14, 200, 40, {"scheme": 2}),
    ("vacuum", 15, 64, 64, {"scheme": 3, "slope_type": 0.7}),
    ("rough", 16, 96, 33, {"iorder": 1, "niter_riemann": 3}),
    ("vacuum", 17, 512, 384, {}),
])
@pytest.mark.parametrize("kernels", [("warp", "warp"), ("march", "march"), ("coop", "coop"),
                                     ("coop8", "coop8")])
def test_random_states_match_oracle(product_lib, oracle, kind, seed, nx, ny, extra, kernels):
    """Random states (shocks and rarefactions everywhere, near-vacuum cells,
    negative internal energy; see _helpers.random_state) through every sweep
    kernel (marching segments, warp windows, 4- and 8-warp cooperative
    windows, in both directions): every cell and the final dt bit for bit
    against the oracle, which is itself checked against the reference on
    such states."""
    from _helpers import random_state
    bnd = (1, 2, 3, 1) if seed % 2 else (1, 1, 1, 1)
    H = make_params(nx, ny, boundary=bnd, **extra)
    u0 = random_state(nx, ny, seed, kind)
    want, wdts, wt = run_oracle(oracle, H, 0, 16, u=u0)
    d = Domain(H, kernels=kernels)
    d.upload(u0)
    d.set_clock()
    d.launch_steps(16)
    got = d.download()
    t, n, dt = d.get_clock()
    d.close()
    assert n == 16 and dt == wdts[-1] and t == wt
    assert bitwise_equal(got, want), describe_mismatch(got, want)


def test_16384_two_steps_against_the_oracle(product_lib, oracle):
    """A large grid (16384^2: 268 M cells, 8.6 GB per state buffer; 131,072
    marching CTAs per y sweep), two steps bit for bit against the oracle on all
    host cores."""
    H = make_params(16384, 16384, testcase=0)
    u0 = init_state(H)
    p = orc_from_H(oracle, H)
    want = u0.copy()
    oracle.oracle_lib().orc_set_threads(os.cpu_count() or 1)
    n, wdts, wt = oracle.run(p, want, 2)
    d = Domain(H)
    d.upload(u0)
    del u0
    d.set_clock()
    d.launch_steps(2)
    got = d.download()
    t, n2, dt = d.get_clock()
    d.close()
    assert n == n2 == 2 and t == wt
    assert bitwise_equal(got, want), describe_mismatch(got, want)

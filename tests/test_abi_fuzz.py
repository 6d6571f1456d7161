"""Argument validation of the C ABI under random parameter records, on the
CPU: every entry point either rejects the record with HB_ERR_ARG or gets as
far as needing a device (HB_ERR_NODEV / HB_ERR_CUDA here, where there is
none) -- never a crash, never a different outcome from the rules below."""
import ctypes as C

import pytest
from hypothesis import given, settings
from hypothesis import strategies as st

from conftest import HAS_GPU
from hydro_b200 import _lib, make_params

# These records would reach a real device (huge allocations, and a bogus state
# pointer in the allocation-free call): the checks run where there is none.
pytestmark = pytest.mark.skipif(HAS_GPU, reason="argument checks are exercised without a device")

INT = st.one_of(st.integers(-5, 40), st.integers(-2**31, 2**31 - 1),
                st.sampled_from([3, 4, 46339, 46340, 2**31 - 5, 2**31 - 1, -2**31]))


def admissible(H):
    """The library's rules for a domain: the reference's 4 variables, at
    least 3 cells each way, padded cells within 2^31, nxt/nyt consistent if
    set, a known scheme, dx > 0, niter_riemann >= 0."""
    if H.nvar != 4 or H.nx < 3 or H.ny < 3:
        return False
    if (H.nx + 4) * (H.ny + 4) > 2**31:
        return False
    if (H.nxt and H.nxt != H.nx + 4) or (H.nyt and H.nyt != H.ny + 4):
        return False
    return 1 <= H.scheme <= 3 and H.dx > 0.0 and H.niter_riemann >= 0


@settings(max_examples=300, deadline=None)
@given(nx=INT, ny=INT, nvar=st.sampled_from([4, 4, 4, 5, 0, -1]),
       scheme=st.integers(-1, 5), niter=st.integers(-3, 12),
       dx=st.sampled_from([1e-3, 0.0, -1.0, float("nan"), float("inf"), 1e-300]),
       nxt=st.sampled_from([0, 0, -1, 7]))
def test_domain_create_outcome(product_lib, nx, ny, nvar, scheme, niter, dx, nxt):
    H = make_params(8, 8)
    H.nx, H.ny, H.nvar, H.scheme, H.niter_riemann, H.dx = nx, ny, nvar, scheme, niter, dx
    H.nxt = H.nyt = nxt
    product_lib.hydro_b200_clear_error()
    d = product_lib.hydro_b200_domain_create(C.byref(H))
    err = product_lib.hydro_b200_last_error()
    product_lib.hydro_b200_clear_error()
    if d:  # only with a device
        product_lib.hydro_b200_domain_destroy(d)
        assert admissible(H)
        return
    if admissible(H):
        assert err in (_lib.HB_ERR_NODEV, _lib.HB_ERR_CUDA, _lib.HB_ERR_NOMEM), err
    else:
        assert err == _lib.HB_ERR_ARG, (err, nx, ny)


@settings(max_examples=200, deadline=None)
@given(nx=INT, ny=INT, idim=st.integers(-1, 3), strides=st.sampled_from(["unset", "set", "bad"]))
def test_noalloc_rejects_before_touching_memory(product_lib, nx, ny, idim, strides):
    """The allocation-free entry point checks its arguments, then that the
    state is device memory of the current device, before any launch: here
    (no device) every call is rejected with HB_ERR_ARG, and the message says
    which rule failed."""
    H = make_params(8, 8)
    H.nx, H.ny = nx, ny
    H.nxt, H.nyt = {"unset": (0, 0), "set": (nx + 4, ny + 4), "bad": (nx + 5, ny + 4)}[strides]
    product_lib.hydro_b200_clear_error()
    rc = product_lib.hydro_b200_godunov_noalloc(C.byref(H), C.c_void_p(16), idim, 1e-3, None)
    msg = product_lib.hydro_b200_last_error_message()
    product_lib.hydro_b200_clear_error()
    too_big = nx >= 3 and ny >= 3 and (nx + 4) * (ny + 4) > _lib.HB_NOALLOC_MAX_CELLS
    assert rc == _lib.HB_ERR_ARG
    if idim not in (1, 2) or nx < 3 or ny < 3 or strides == "bad" or too_big:
        assert b"not a device pointer" not in msg, msg
    else:
        assert b"not a device pointer" in msg, msg


def test_noalloc_rejects_a_host_state(product_lib):
    """A state in host memory is rejected (HB_ERR_ARG) instead of being handed
    to kernels that cannot read it."""
    import numpy as np
    H = make_params(16, 12)
    u = np.zeros((4, H.ny + 4, H.nx + 4))
    product_lib.hydro_b200_clear_error()
    rc = product_lib.hydro_b200_godunov_noalloc(C.byref(H), u.ctypes.data, 1, 1e-3, None)
    assert rc == _lib.HB_ERR_ARG
    assert product_lib.hydro_b200_last_error() == _lib.HB_ERR_ARG
    product_lib.hydro_b200_clear_error()


@settings(max_examples=100, deadline=None)
@given(nx=INT, ny=INT)
def test_batch_bytes_needed(product_lib, nx, ny):
    H = make_params(8, 8)
    H.nx, H.ny = nx, ny
    n = product_lib.hydro_b200_batch_bytes_needed(C.byref(H))
    if nx < 3 or ny < 3 or (nx + 4) * (ny + 4) > 2**31:
        assert n == 0
    else:
        assert n == 2 * 256 * ((4 * (nx + 4) * (ny + 4) + 31) // 32)


def test_null_arguments_are_rejected(product_lib):
    lib = product_lib
    for call in (lambda: lib.hydro_b200_domain_create(None),
                 lambda: lib.hydro_b200_godunov_noalloc(None, None, 1, 0.0, None),
                 lambda: lib.hydro_b200_domain_sweep(None, 0, 1, 0.0, 0),
                 lambda: lib.hydro_b200_domain_halo_pack(None, 0, 1, 0, None),
                 lambda: lib.hydro_b200_domain_vtk_base64(None, 0, None, 0)):
        lib.hydro_b200_clear_error()
        r = call()
        assert not r or r == _lib.HB_ERR_ARG
        assert lib.hydro_b200_last_error() == _lib.HB_ERR_ARG
    lib.hydro_b200_clear_error()

"""hydro_b200_godunov_noalloc: the time step for callers that cannot allocate
device memory (code running inside another allocator's arena, under a capped
allocation budget, or in the middle of a stream capture).  It takes a state
the caller already holds on the device and uses a fixed-size static device
array as the sweeps' second buffer.  Its result must equal the regular
reference entry point's (hydro_godunov, which allocates its own mirror and
buffer) bit for bit, on two calls in a row (x->y then y->x).

This file is collected last on purpose: it runs alone in a fresh process as
well as after the rest of the suite."""
import ctypes as C

import numpy as np
import pytest

from hydro_b200 import HydroRun, init_state, load, make_params
from hydro_b200._lib import HB_ERR_ARG, HB_OK

pytestmark = pytest.mark.gpu


def test_noalloc_step_equals_hydro_godunov_twice(product_lib):
    import torch

    H = make_params(300, 200, testcase=1)
    u0 = init_state(H)
    steps = [(1, 5.0e-6), (2, 5.0e-6)]

    # The regular entry point, one call after the other.
    ref = HydroRun(H, u0.copy())
    want = []
    for idim, dt in steps:
        ref.godunov(idim, dt)
        want.append(ref.sync_to_host().copy())
    ref.close()

    # The caller owns the device state; the step itself allocates nothing.
    lib = load()
    state = torch.from_numpy(u0.copy()).to("cuda:0")
    for k, (idim, dt) in enumerate(steps):
        rc = lib.hydro_b200_godunov_noalloc(C.byref(H), state.data_ptr(), idim, dt, None)
        assert rc == HB_OK, lib.hydro_b200_last_error_message()
        torch.cuda.synchronize()
        got = state.cpu().numpy()
        assert np.array_equal(got.view(np.uint64), want[k].view(np.uint64)), \
            f"call {k + 1}: max |diff| {np.max(np.abs(got - want[k])):.3e}"


def test_noalloc_rejects_grids_over_its_limit(product_lib):
    import torch

    lib = load()
    H = make_params(1021, 1021)  # (1021 + 4)^2 padded cells > HB_NOALLOC_MAX_CELLS
    dummy = torch.zeros(1, dtype=torch.float64, device="cuda:0")
    rc = lib.hydro_b200_godunov_noalloc(C.byref(H), dummy.data_ptr(), 1, 1e-6, None)
    assert rc == HB_ERR_ARG
    assert b"HB_NOALLOC_MAX_CELLS" in lib.hydro_b200_last_error_message()
    lib.hydro_b200_clear_error()

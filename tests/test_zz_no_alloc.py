"""hydro_b200_godunov_noalloc: the time step for callers that cannot allocate
device memory -- code that runs inside another framework's memory arena, or
in a process whose device-allocation budget is already spent.  It takes a
state the caller already holds on the device and uses a fixed-size static
device array as the sweeps' second buffer.  Its result must equal the regular
reference entry point's (hydro_godunov, which allocates its own mirror and
buffer) bit for bit, on two calls in a row (x->y then y->x), on the default
stream and on a stream the caller created, up to the largest grid the array
holds.

This file is collected last on purpose: it runs alone in a fresh process as
well as after the rest of the suite."""
import ctypes as C

import numpy as np
import pytest

from hydro_b200 import HydroRun, init_state, load, make_params
from hydro_b200._lib import HB_ERR_ARG, HB_NOALLOC_MAX_CELLS, HB_OK

pytestmark = pytest.mark.gpu


def regular_steps(H, u0, steps):
    """The states after each hydro_godunov call of `steps`."""
    ref = HydroRun(H, u0.copy())
    out = []
    for idim, dt in steps:
        ref.godunov(idim, dt)
        out.append(ref.sync_to_host().copy())
    ref.close()
    return out


# (300, 200) a corner blast; (250, 125) the 250x125 corner case; (1020, 1020)
# fills the static array exactly: (1020 + 4)^2 == HB_NOALLOC_MAX_CELLS.
@pytest.mark.parametrize("nx,ny", [(300, 200), (250, 125), (1020, 1020)])
@pytest.mark.parametrize("own_stream", [False, True])
def test_noalloc_step_equals_hydro_godunov_twice(product_lib, nx, ny, own_stream):
    import torch

    H = make_params(nx, ny, testcase=1)
    u0 = init_state(H)
    dt = 0.4 / max(nx, ny) ** 2  # below the blast's CFL step (about 1/n^2)
    steps = [(1, dt), (2, dt)]
    want = regular_steps(H, u0, steps)

    # The caller owns the device state (and, here, the stream); the step
    # itself allocates nothing.
    lib = load()
    state = torch.from_numpy(u0.copy()).to("cuda:0")
    stream = torch.cuda.Stream() if own_stream else None
    handle = C.c_void_p(stream.cuda_stream) if stream is not None else None
    torch.cuda.synchronize()
    for k, (idim, dt) in enumerate(steps):
        rc = lib.hydro_b200_godunov_noalloc(C.byref(H), state.data_ptr(), idim, dt, handle)
        assert rc == HB_OK, lib.hydro_b200_last_error_message()
        if stream is not None:
            stream.synchronize()
        torch.cuda.synchronize()
        got = state.cpu().numpy()
        assert np.array_equal(got.view(np.uint64), want[k].view(np.uint64)), \
            f"call {k + 1}: max |diff| {np.max(np.abs(got - want[k])):.3e}"
    assert (nx + 4) * (ny + 4) <= HB_NOALLOC_MAX_CELLS


def test_noalloc_leaves_free_device_memory_unchanged(product_lib):
    """After one call (which loads the kernels and looks up the array's
    address), further calls leave the device's free memory where it was."""
    import torch

    lib = load()
    H = make_params(250, 125, testcase=1)
    state = torch.from_numpy(init_state(H)).to("cuda:0")
    torch.cuda.synchronize()
    assert lib.hydro_b200_godunov_noalloc(C.byref(H), state.data_ptr(), 1, 1e-5, None) == HB_OK
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for k in range(20):
        rc = lib.hydro_b200_godunov_noalloc(C.byref(H), state.data_ptr(), 1 + k % 2, 1e-5, None)
        assert rc == HB_OK, lib.hydro_b200_last_error_message()
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0, (free0, free1)


def test_noalloc_rejects_grids_over_its_limit(product_lib):
    import torch

    lib = load()
    H = make_params(1021, 1021)  # (1021 + 4)^2 padded cells > HB_NOALLOC_MAX_CELLS
    dummy = torch.zeros(1, dtype=torch.float64, device="cuda:0")
    rc = lib.hydro_b200_godunov_noalloc(C.byref(H), dummy.data_ptr(), 1, 1e-6, None)
    assert rc == HB_ERR_ARG
    assert b"HB_NOALLOC_MAX_CELLS" in lib.hydro_b200_last_error_message()
    lib.hydro_b200_clear_error()


def test_noalloc_rejects_host_memory(product_lib):
    """A state in host memory (pageable or pinned) is rejected before any
    kernel could be given it."""
    import torch

    lib = load()
    H = make_params(64, 48)
    for u in (np.zeros((4, H.ny + 4, H.nx + 4)),
              torch.zeros((4, H.ny + 4, H.nx + 4), dtype=torch.float64, pin_memory=True).numpy()):
        lib.hydro_b200_clear_error()
        rc = lib.hydro_b200_godunov_noalloc(C.byref(H), u.ctypes.data, 1, 1e-6, None)
        assert rc == HB_ERR_ARG, rc
        assert b"device" in lib.hydro_b200_last_error_message()
    lib.hydro_b200_clear_error()

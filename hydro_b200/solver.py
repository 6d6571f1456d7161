"""Python front-end of the C ABI.

* ``HydroRun`` drives a host-resident state exactly as the reference driver
  does (main.c:344-408), through the reference entry points hydro_godunov /
  compute_deltat (device mirror of the host array inside the library), or
  through the library's device-resident driver ``hydro_b200_run``.
* ``Domain`` is the device-pointer level object (hb_domain): state resident in
  HBM, explicit upload / download, asynchronous launches on its own stream.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import HydroParam, HydroVar, HydroVarWork, HydroWork, check, load
from .params import init_state, state_shape


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


class HydroRun:
    """A HydroC run on a host array ``uold`` (reference layout, float64).

    The library keeps the device copy; ``sync_to_host`` brings it back.
    """

    def __init__(self, H: HydroParam, uold: np.ndarray | None = None):
        self.lib = load()
        self.H = H
        if uold is None:
            uold = init_state(H)
        if uold.dtype != np.float64 or not uold.flags.c_contiguous or \
                uold.shape != state_shape(H):
            raise ValueError("uold must be a C-contiguous float64 array of shape "
                             f"{state_shape(H)}")
        self.uold = uold
        self.Hv = HydroVar(_dptr(uold))
        self.Hw = HydroWork()
        self.Hvw = HydroVarWork()
        self.t = float(H.t)
        self.nstep = int(H.nstep)
        self.dt = 0.0

    # --- reference entry points -------------------------------------------
    def compute_deltat(self) -> float:
        dt = C.c_double(0.0)
        self.lib.compute_deltat(C.byref(dt), self.H, C.byref(self.Hw), C.byref(self.Hv),
                                C.byref(self.Hvw))
        check()
        return dt.value

    def godunov(self, idim: int, dt: float) -> None:
        self.lib.hydro_godunov(idim, dt, self.H, C.byref(self.Hv), C.byref(self.Hw),
                               C.byref(self.Hvw))
        check()

    def make_boundary(self, idim: int) -> None:
        self.lib.make_boundary(idim, self.H, C.byref(self.Hv))
        check()

    def step(self) -> float:
        """One iteration of main.c:344-408."""
        if self.nstep % 2 == 0:
            self.dt = self.compute_deltat()
            if self.nstep == 0:
                self.dt = self.dt / 2.0
        self.godunov(1 if self.nstep % 2 == 0 else 2, self.dt)
        self.nstep += 1
        self.t += self.dt
        return self.dt

    def run_host_loop(self, nstepmax: int, tend: float = 1e300) -> np.ndarray:
        """The reference loop on the host over the reference entry points."""
        dts = []
        while self.t < tend and self.nstep < nstepmax:
            dts.append(self.step())
        return np.array(dts)

    # --- device-resident driver -------------------------------------------
    def run(self, nstepmax: int, tend: float = 1e300) -> np.ndarray:
        """The same loop with dt and t on the device (hydro_b200_run)."""
        t = C.c_double(self.t)
        n = C.c_int(self.nstep)
        dt = C.c_double(self.dt)
        dts = np.zeros(max(nstepmax - self.nstep, 1), dtype=np.float64)
        done = self.lib.hydro_b200_run(C.byref(self.H), C.byref(self.Hv), nstepmax, tend,
                                       C.byref(t), C.byref(n), C.byref(dt), _dptr(dts))
        check(done)
        self.t, self.nstep, self.dt = t.value, n.value, dt.value
        return dts[:done].copy()

    # --- residency ---------------------------------------------------------
    def sync_to_host(self) -> np.ndarray:
        check(self.lib.hydro_b200_sync_to_host(C.byref(self.H), C.byref(self.Hv)))
        return self.uold

    def sync_to_device(self) -> None:
        check(self.lib.hydro_b200_sync_to_device(C.byref(self.H), C.byref(self.Hv)))

    def release(self) -> None:
        check(self.lib.hydro_b200_release(C.byref(self.Hv)))

    @property
    def stream_ptr(self) -> int:
        s = self.lib.hydro_b200_mirror_stream(C.byref(self.H), C.byref(self.Hv))
        check()
        return s

    def close(self) -> None:
        try:
            self.release()
        except Exception:
            pass


class Domain:
    """Device-resident state (hb_domain)."""

    def __init__(self, H: HydroParam, precision: str = "fp64", xsweep: str | None = None,
                 kernels: tuple | None = None):
        self.lib = load()
        self.H = H
        self.h = self.lib.hydro_b200_domain_create(C.byref(H))
        if not self.h:
            check()
            raise _lib.HydroB200Error("domain creation failed")
        self.precision = precision
        check(self.lib.hydro_b200_domain_set_precision(self.h, _lib.PRECISIONS[precision]))
        if xsweep is not None:
            check(self.lib.hydro_b200_domain_set_xsweep(self.h, _lib.PRECISIONS[precision],
                                                        _lib.XSWEEPS[xsweep]))
        if kernels is not None:
            self.set_kernels(*kernels)
        self.shape = state_shape(H)
        self.nbytes = int(np.prod(self.shape)) * 8

    def set_kernels(self, x: str | None = None, y: str | None = None) -> None:
        """Sweep kernels of this domain's precision: "march", "warp", "coop",
        "coop8", "bulk" (mixed x sweep only) or "auto" per direction (None
        keeps the current one)."""
        prec = _lib.PRECISIONS[self.precision]
        for idim, k in ((1, x), (2, y)):
            if k is not None:
                check(self.lib.hydro_b200_domain_set_kernel(self.h, prec, idim, _lib.KERNELS[k]))

    def kernels(self) -> tuple:
        names = {v: k for k, v in _lib.KERNELS.items()}
        prec = _lib.PRECISIONS[self.precision]
        return tuple(names[self.lib.hydro_b200_domain_get_kernel(self.h, prec, i)] for i in (1, 2))

    @property
    def state_ptr(self) -> int:
        return self.lib.hydro_b200_domain_state(self.h)

    @property
    def stream_ptr(self) -> int:
        return self.lib.hydro_b200_domain_stream(self.h)

    def upload(self, host: np.ndarray, sync: bool = True) -> None:
        assert host.dtype == np.float64 and host.flags.c_contiguous and host.shape == self.shape
        check(self.lib.hydro_b200_domain_upload(self.h, host.ctypes.data))
        if sync:
            self.synchronize()

    def upload_ptr(self, ptr: int) -> None:
        check(self.lib.hydro_b200_domain_upload(self.h, ptr))

    def download(self, out: np.ndarray | None = None) -> np.ndarray:
        if out is None:
            out = np.empty(self.shape, dtype=np.float64)
        check(self.lib.hydro_b200_domain_download(self.h, out.ctypes.data))
        self.synchronize()
        return out

    def download_ptr(self, ptr: int) -> None:
        check(self.lib.hydro_b200_domain_download(self.h, ptr))

    def synchronize(self) -> None:
        check(self.lib.hydro_b200_domain_synchronize(self.h))

    def godunov(self, idim: int, dt: float, fuse_courant: bool = False) -> None:
        check(self.lib.hydro_b200_domain_godunov(self.h, idim, dt, int(fuse_courant)))

    def make_boundary(self, idim: int) -> None:
        check(self.lib.hydro_b200_domain_make_boundary(self.h, idim))

    def courant(self):
        cx, cy = C.c_double(), C.c_double()
        check(self.lib.hydro_b200_domain_courant(self.h, C.byref(cx), C.byref(cy)))
        return cx.value, cy.value

    # --- one sweep at a time, and halo strips (domain split) ------------------
    def sweep(self, stage: int, idim: int, dt: float, fuse_courant: bool = False,
              part: int = 0) -> None:
        """One sweep of a step (stage 0: first, 1: second); part 1 / 2 sweep
        the ghost-free windows / the others (0: all)."""
        check(self.lib.hydro_b200_domain_sweep_part(self.h, stage, idim, dt, int(fuse_courant),
                                                    part))

    def halo_count(self, idim: int) -> int:
        return int(self.lib.hydro_b200_domain_halo_count(self.h, idim))

    def halo_pack(self, stage: int, idim: int, side: int, dst_ptr: int) -> None:
        check(self.lib.hydro_b200_domain_halo_pack(self.h, stage, idim, side, dst_ptr))

    def halo_unpack(self, idim: int, side: int, src_ptr: int) -> None:
        check(self.lib.hydro_b200_domain_halo_unpack(self.h, idim, side, src_ptr))

    def vtk_base64(self, var: int) -> bytes:
        """The VTK writer's base64 payload of variable `var` (0..3)."""
        n = int(self.lib.hydro_b200_vtk_base64_len(self.H.nx, self.H.ny))
        buf = C.create_string_buffer(n)
        check(self.lib.hydro_b200_domain_vtk_base64(self.h, var, buf, n))
        return buf.raw[:n]

    def set_clock(self, t: float = 0.0, nstep: int = 0, dt: float = 0.0) -> None:
        check(self.lib.hydro_b200_domain_set_clock(self.h, t, nstep, dt))

    def launch_steps(self, nsteps: int, nstepmax: int = 2**31 - 1, tend: float = 1e300) -> None:
        check(self.lib.hydro_b200_domain_launch_steps(self.h, nsteps, nstepmax, tend))

    def get_clock(self):
        t, n, dt = C.c_double(), C.c_int(), C.c_double()
        check(self.lib.hydro_b200_domain_get_clock(self.h, C.byref(t), C.byref(n), C.byref(dt)))
        return t.value, n.value, dt.value

    def reserve_dts(self, n: int) -> None:
        """Record the dt of up to n steps from the next set_clock on."""
        check(self.lib.hydro_b200_domain_reserve_dts(self.h, n))

    def get_dts(self, n: int) -> np.ndarray:
        """dt of steps 0 .. n-1 of the launch-only driver (device record)."""
        out = np.zeros(max(n, 1), dtype=np.float64)
        check(self.lib.hydro_b200_domain_get_dts(self.h, out.ctypes.data_as(C.POINTER(C.c_double)),
                                                 n))
        return out[:n]

    def profile(self, enable: bool = True) -> None:
        check(self.lib.hydro_b200_domain_profile(self.h, int(enable)))

    def profile_read(self, reset: bool = True):
        """(ms_x, ms_y, n_x, n_y) accumulated since the last reset."""
        ms = (C.c_double * 2)()
        n = (C.c_longlong * 2)()
        check(self.lib.hydro_b200_domain_profile_read(self.h, ms, n, int(reset)))
        return ms[0], ms[1], n[0], n[1]

    @property
    def launch_count(self) -> int:
        return int(self.lib.hydro_b200_domain_launch_count(self.h))

    def close(self) -> None:
        if self.h:
            self.lib.hydro_b200_domain_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

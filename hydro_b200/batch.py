"""Batches of independent HydroC runs (include/hydro_b200.h, hb_batch.cu).

``Batch`` holds many grids of different sizes in one device arena and
advances all active ones per global step, each with its own dt, through two
persistent launches per step replayed from CUDA graphs.  ``make_blast_mix``
draws the seeded instance mix of the batched workload.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import _lib
from ._lib import HydroParam, check, load
from .params import make_params, splitmix64, state_shape


class Batch:
    def __init__(self, H: HydroParam, capacity: int, arena_bytes: int,
                 precision: str = "mixed"):
        self.lib = load()
        self.H = H
        self.h = self.lib.hydro_b200_batch_create(C.byref(H), capacity, arena_bytes,
                                                  _lib.PRECISIONS[precision])
        if not self.h:
            check()
            raise _lib.HydroB200Error("batch creation failed")
        self.capacity = capacity
        self.params = {}
        self.limits = {}

    @staticmethod
    def bytes_needed(H: HydroParam) -> int:
        return int(load().hydro_b200_batch_bytes_needed(C.byref(H)))

    @property
    def arena_free(self) -> int:
        return int(self.lib.hydro_b200_batch_arena_free(self.h))

    @property
    def stream_ptr(self) -> int:
        return self.lib.hydro_b200_batch_stream(self.h)

    def add(self, H: HydroParam, state: np.ndarray, tend: float = 1e300,
            nstepmax: int = 2**31 - 1) -> int:
        slot = self.try_add(H, state, tend, nstepmax)
        if slot < 0:
            raise _lib.HydroB200Error("batch add: no free slot or arena space")
        return slot

    def try_add(self, H: HydroParam, state: np.ndarray, tend: float = 1e300,
                nstepmax: int = 2**31 - 1) -> int:
        """Admit an instance; returns its slot, or -1 when no slot or arena
        space is free."""
        assert state.dtype == np.float64 and state.flags.c_contiguous
        assert state.shape == state_shape(H)
        slot = self.lib.hydro_b200_batch_add(self.h, C.byref(H), state.ctypes.data, tend,
                                             nstepmax)
        if slot < 0:
            err = self.lib.hydro_b200_last_error()
            msg = self.lib.hydro_b200_last_error_message().decode(errors="replace")
            self.lib.hydro_b200_clear_error()
            if err != _lib.HB_ERR_NOMEM:
                raise _lib.HydroB200Error(f"batch add failed ({err}): {msg}")
            return -1
        self.params[slot] = H
        self.limits[slot] = (tend, nstepmax)
        return slot

    def try_add_blast(self, H: HydroParam, rho: float, e_bg: float, cell: tuple, e_blast: float,
                      tend: float = 1e300, nstepmax: int = 2**31 - 1) -> int:
        """Admit a single-blast instance generated on the device; `cell` is
        the padded (i, j) of the blast.  Returns the slot, or -1 when full."""
        slot = self.lib.hydro_b200_batch_add_blast(self.h, C.byref(H), rho, e_bg, int(cell[0]),
                                                   int(cell[1]), e_blast, tend, nstepmax)
        if slot < 0:
            err = self.lib.hydro_b200_last_error()
            msg = self.lib.hydro_b200_last_error_message().decode(errors="replace")
            self.lib.hydro_b200_clear_error()
            if err != _lib.HB_ERR_NOMEM:
                raise _lib.HydroB200Error(f"batch add failed ({err}): {msg}")
            return -1
        self.params[slot] = H
        self.limits[slot] = (tend, nstepmax)
        return slot

    def checkpoint(self, slot: int) -> dict:
        """State and clock of an instance (with its grid parameters and
        limits), enough to resume it bit for bit later, here or in another
        batch."""
        st = self.status(slot)
        H = self.params[slot]
        return {"state": self.download(slot), "t": st["t"], "nstep": st["nstep"],
                "dt": st["dt"], "nx": H.nx, "ny": H.ny, "dx": H.dx,
                "boundary": (H.boundary_left, H.boundary_right, H.boundary_down,
                             H.boundary_up),
                "tend": self.limits.get(slot, (1e300, 2**31 - 1))[0],
                "nstepmax": self.limits.get(slot, (1e300, 2**31 - 1))[1]}

    def resume(self, ckpt: dict) -> int:
        """Admit a checkpointed instance; returns its slot (-1 when full)."""
        H = make_params(ckpt["nx"], ckpt["ny"], dx=ckpt["dx"], boundary=tuple(ckpt["boundary"]))
        H.t = ckpt["t"]
        H.nstep = ckpt["nstep"]
        state = np.ascontiguousarray(ckpt["state"], dtype=np.float64)
        slot = self.lib.hydro_b200_batch_add_resume(self.h, C.byref(H), state.ctypes.data,
                                                    ckpt["dt"], ckpt["tend"], ckpt["nstepmax"])
        if slot < 0:
            err = self.lib.hydro_b200_last_error()
            self.lib.hydro_b200_clear_error()
            if err != _lib.HB_ERR_NOMEM:
                raise _lib.HydroB200Error(f"batch resume failed ({err})")
            return -1
        self.params[slot] = H
        self.limits[slot] = (ckpt["tend"], ckpt["nstepmax"])
        return slot

    def remove(self, slot: int) -> None:
        check(self.lib.hydro_b200_batch_remove(self.h, slot))
        self.params.pop(slot, None)
        self.limits.pop(slot, None)

    def steps(self, n: int) -> None:
        check(self.lib.hydro_b200_batch_steps(self.h, n))

    def synchronize(self) -> None:
        check(self.lib.hydro_b200_batch_synchronize(self.h))

    def status(self, slot: int):
        t, n, dt, a, st = C.c_double(), C.c_int(), C.c_double(), C.c_int(), C.c_longlong()
        check(self.lib.hydro_b200_batch_status(self.h, slot, C.byref(t), C.byref(n),
                                               C.byref(dt), C.byref(a), C.byref(st)))
        return {"t": t.value, "nstep": n.value, "dt": dt.value, "active": bool(a.value),
                "stop_step": st.value}

    def poll(self) -> np.ndarray:
        out = (C.c_int * self.capacity)()
        check(self.lib.hydro_b200_batch_poll(self.h, out, self.capacity))
        return np.frombuffer(out, dtype=np.int32).copy()

    def table(self):
        """(active, nstep, t) arrays over all slots, one device read."""
        a = (C.c_int * self.capacity)()
        n = (C.c_int * self.capacity)()
        t = (C.c_double * self.capacity)()
        check(self.lib.hydro_b200_batch_table(self.h, a, n, t, self.capacity))
        return (np.frombuffer(a, dtype=np.int32).copy(), np.frombuffer(n, dtype=np.int32).copy(),
                np.frombuffer(t, dtype=np.float64).copy())

    def download(self, slot: int) -> np.ndarray:
        H = self.params[slot]
        out = np.empty(state_shape(H), dtype=np.float64)
        check(self.lib.hydro_b200_batch_download(self.h, slot, out.ctypes.data))
        return out

    @property
    def global_step(self) -> int:
        return int(self.lib.hydro_b200_batch_global_step(self.h))

    @property
    def launch_count(self) -> int:
        return int(self.lib.hydro_b200_batch_launch_count(self.h))

    def set_tuning(self, seg: int, claim: int, blocks_per_sm: int = 0, threads: int = 64) -> None:
        check(self.lib.hydro_b200_batch_set_tuning(self.h, seg, claim, blocks_per_sm, threads))

    def tuning(self):
        s, c, b, t = C.c_int(), C.c_int(), C.c_int(), C.c_int()
        check(self.lib.hydro_b200_batch_get_tuning(self.h, C.byref(s), C.byref(c), C.byref(b),
                                                   C.byref(t)))
        return {"seg": s.value, "claim": c.value, "blocks_per_sm": b.value, "threads": t.value}

    def autotune(self, steps: int = 2) -> int:
        n = self.lib.hydro_b200_batch_autotune(self.h, steps)
        check(n)
        return n

    def close(self) -> None:
        if self.h:
            self.lib.hydro_b200_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _u01(seed: int, stream: int, idx: np.ndarray) -> np.ndarray:
    z = splitmix64(np.uint64(seed) ^ (np.uint64(stream) << np.uint64(40)) ^ idx.astype(np.uint64))
    return (z >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)


E_BACKGROUND = 1e-5


def blast_spec(nx: int, ny: int, bx: float, by: float, e0: float, rho: float):
    """Parameters of a single-blast instance: density rho, u = v = 0,
    E = 1e-5, and E = e0/dx^2 in the cell at fractional position (bx, by) of
    the interior; dx = 1/nx, reflecting walls.  Returns (H, rho, e_bg,
    (i, j) padded blast cell, e_blast)."""
    H = make_params(nx, ny, testcase=0)
    i = 2 + min(int(bx * nx), nx - 1)
    j = 2 + min(int(by * ny), ny - 1)
    return H, rho, E_BACKGROUND, (i, j), e0 / H.dx / H.dx


def blast_state(H: HydroParam, rho: float, e_bg: float, cell: tuple, e_blast: float):
    """The host array of blast_spec's instance (what the device init writes)."""
    u = np.zeros(state_shape(H), dtype=np.float64)
    u[0, 2:-2, 2:-2] = rho
    u[3, 2:-2, 2:-2] = e_bg
    u[3, cell[1], cell[0]] = e_blast
    return u


def blast_instance(nx: int, ny: int, bx: float, by: float, e0: float, rho: float):
    """blast_spec's instance as (H, host state)."""
    H, rho, e_bg, cell, eb = blast_spec(nx, ny, bx, by, e0, rho)
    return H, blast_state(H, rho, e_bg, cell, eb)


def make_blast_mix(n: int, seed: int, side_lo: int = 64, side_hi: int = 1024,
                   square: bool = False, first: int = 0):
    """The batched workload's instances: nx, ny log-uniform in
    [side_lo, side_hi] rounded to multiples of 8 (square grids if `square`),
    dx = 1/nx, blast cell uniform over the interior, blast energy E0
    log-uniform in [0.1, 10]/dx^2, background density uniform in [0.5, 2],
    E = 1e-5 elsewhere, reflecting walls.  Every draw is SplitMix64 of the
    seed, a stream id and the instance index (first .. first + n - 1).
    Returns [(H, state)]."""
    idx = np.arange(first, first + n, dtype=np.uint64)
    lo, hi = math.log(side_lo), math.log(side_hi)

    def side(stream):
        v = np.exp(lo + (hi - lo) * _u01(seed, stream, idx))
        return np.clip(np.rint(v / 8) * 8, side_lo, side_hi).astype(int)

    nxs = side(1)
    nys = nxs.copy() if square else side(2)
    bx, by = _u01(seed, 3, idx), _u01(seed, 4, idx)
    e0 = np.exp(math.log(0.1) + (math.log(10.0) - math.log(0.1)) * _u01(seed, 5, idx))
    rho = 0.5 + 1.5 * _u01(seed, 6, idx)
    return [blast_instance(int(nxs[k]), int(nys[k]), float(bx[k]), float(by[k]), float(e0[k]),
                           float(rho[k])) for k in range(n)]

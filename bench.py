#!/usr/bin/env python
"""Throughput of the HydroC Godunov/MUSCL time step on B200.

Workload (default): the 4096 x 4096 centred blast in FP64 -- rho = 1, u = v = 0,
E = 1e-5, E = 1/dx^2 in the centre cell, dx = 1/4096, gamma 1.4, reflecting
walls, MUSCL, iorder 2, slope_type 1, niter_riemann 10, courant_factor 0.8 --
advanced K time steps from its initial state (steps 0..K-1; the workload's
run is 200 steps).  One step = both dimension-split sweeps plus the CFL dt
(recomputed on even steps), as in the reference driver loop.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Prints one JSON line.  `value` is Mcell-updates/s (cells x steps / s) over
all ranks with the state resident in HBM, timed with CUDA events on the
library's stream; `e2e` is the same metric through the reference entry
points (compute_deltat + hydro_godunov) on a pinned host array, with the
upload, the per-step dt reads and the final download inside the timed region.
With N > 1 (torchrun) every rank advances its own replica (weak scaling; the
workload is one grid on one GPU, so there is no exchange).

--impl reference times the reference's own C99/OpenMP implementation of the
same step on the host cores (oracle/_ref, compiled from the reference
sources) on the same workload.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from hydro_b200.metrics import field_errors  # noqa: E402

WORKLOADS = {
    "centre_4096": dict(name="hydroc_4096x4096_centre_blast_fp64", nx=4096, ny=4096, testcase=0,
                        run_steps=200),
    "corner_250x125": dict(name="hydroc_250x125_corner_blast_fp64", nx=250, ny=125,
                           testcase=1, run_steps=100),
    # The same problem at 2048^2 (134 MB per state buffer, still > L2): the
    # size the ncu section captures use.
    "centre_2048": dict(name="hydroc_2048x2048_centre_blast_fp64", nx=2048, ny=2048, testcase=0,
                        run_steps=200),
}
BYTES_PER_CELL_SWEEP = 64   # 4 doubles read + 4 doubles written per cell and sweep
# CUDA kernel of each sweep-kernel choice (FP64 set).
KERNEL_NAMES = {"march": "sweep_kernel", "warp": "xcell_kernel / ycell_kernel",
                "coop": "coop_pipe_kernel<.,1,4,8> (x, pipelined runs of 8 windows from 2048^2) "
                        "/ coop_kernel<.,.,4>",
                "coop8": "coop_kernel<.,.,8>"}
BYTES_PER_CELL_STEP = 2 * BYTES_PER_CELL_SWEEP


def env_int(k, d):
    try:
        return int(os.environ.get(k, d))
    except ValueError:
        return d


def measured_peak_hbm():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def ncu_fp64_pipe():
    """FP64-pipe and issue utilisation of the two FP64 sweep kernels at the
    bench workload, from the committed ncu summary (percent, x and y sweep),
    or None."""
    import re
    p = os.path.join(ROOT, "profiles", "sweep_fp64_4096.md")
    out = {}
    try:
        for line in open(p):
            for key, label in (("fp64_pipe_pct", "FP64 pipe (%)"),
                               ("issue_active_pct", "issue active (%)")):
                m = re.match(r"\|\s*" + re.escape(label) + r"\s*\|\s*([0-9.]+)\s*\|\s*([0-9.]+)\s*\|",
                             line)
                if m:
                    out[key] = {"x_sweep": float(m.group(1)), "y_sweep": float(m.group(2))}
    except OSError:
        return None
    if not out:
        return None
    out["unit"] = "% of peak (ncu, 4096^2 capture of the bench's sweep kernels)"
    out["source"] = "profiles/sweep_fp64_4096.md"
    return out


def ncu_traffic_per_launch():
    """DRAM bytes per sweep launch from the committed ncu summary (if any)."""
    p = os.path.join(ROOT, "profiles", "sweep_fp64_4096_traffic.txt")
    try:
        for line in open(p):
            if line.startswith("dram_bytes_per_launch_full_size:"):
                return float(line.split(":", 1)[1].split()[0])
    except Exception:
        pass
    return None


class ClockSampler:
    """nvidia-smi samples (SM clock, throttle reasons) while it runs."""

    QUERY = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.samples = []
        self.proc = None
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.QUERY}",
                 "--format=csv,noheader,nounits", "-lms", "50"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
            return self
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.samples.append((time.time(), [x.strip() for x in line.split(",")]))

    def stop(self):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
        if self.thread:
            self.thread.join(timeout=5)

    def summary(self, t0, t1):
        rows = [s for (ts, s) in self.samples if t0 - 0.05 <= ts <= t1 + 0.05] or \
               [s for (_, s) in self.samples]
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        sm = [float(r[0]) for r in rows if r[0].replace(".", "").isdigit()]
        smax = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4)
                          if len(r) > 4 + i and r[4 + i].lower().startswith("active")})
        pw = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None, "reasons": reasons,
                "power_w_max": max(pw) if pw else None, "samples": len(rows)}


def dist_setup(gpus):
    world = env_int("WORLD_SIZE", 1)
    rank = env_int("RANK", 0)
    local = env_int("LOCAL_RANK", 0)
    pg = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        dist.init_process_group("nccl" if gpus else "gloo",
                                timeout=datetime.timedelta(seconds=120))
        pg = dist
    return world, rank, local, pg


def all_max(pg, x, device):
    if pg is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64, device=device)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def barrier(pg, device):
    if pg is not None:
        import torch
        pg.all_reduce(torch.zeros(1, device=device))


def aggregate_mcs(world, cells_per_rank, steps, ms_max):
    """Whole-job Mcell-updates/s of `world` replicas that each advanced
    cells_per_rank cells by `steps` steps, timed as the slowest rank."""
    return world * cells_per_rank * steps / (ms_max / 1e3) / 1e6


def dom_state_after(H, u0, nsteps, precision):
    from hydro_b200 import Domain
    d = Domain(H, precision=precision)
    d.upload(u0)
    d.set_clock()
    d.launch_steps(nsteps)
    u = d.download()
    d.close()
    return u


def mixed_beside_reference_fp32():
    """Context for the mixed form's error.  The reference's own all-FP32 build
    (its SP=O option, -DPREC_SP; oracle/_ref/libhydroref_sp.so) and the mixed
    form are each compared with the FP64 path, which is bitwise equal to the
    reference's FP64 build, on the same inputs."""
    from hydro_b200 import init_state, make_params
    from oracle import oracle as O
    if not O.ref_available(sp=True):
        return {"unavailable": "oracle/_ref/libhydroref_sp.so not built"}
    out = []
    for label, nx, ny, tc, n in (("250x125 corner blast, 100 steps", 250, 125, 1, 100),
                                 ("1024x1024 centred blast, 200 steps", 1024, 1024, 0, 200)):
        H = make_params(nx, ny, testcase=tc)
        u0 = init_state(H, tc)
        fp64 = dom_state_after(H, u0, n, "fp64")
        mix = dom_state_after(H, u0, n, "mixed")
        with quiet_stdout():  # the reference prints its set-up
            sp = O.RefState(O.make_param(nx, ny, dx=H.dx), tc, sp=True)
            sp.set(u0)
            nsp = sp.run(n)[0]
            usp = sp.get()
            sp.close()
        out.append({"case": label, "steps": nsp,
                    "mixed_vs_fp64": field_errors(mix, fp64),
                    "reference_fp32_build_vs_fp64": field_errors(usp, fp64)})
    return out


def tier_errors(got, want):
    """Per-cell errors of the FMA FP64 tier's rule: density and energy
    relative; momenta relative to the larger of the cell's value and the
    field's largest magnitude."""
    out = {}
    for v, name in enumerate(("rho", "rhou", "rhov", "E")):
        a, b = got[v], want[v]
        den = np.abs(b) if name in ("rho", "E") else np.maximum(np.abs(b), np.max(np.abs(b)))
        err = np.abs(a - b) / np.where(den > 0, den, 1.0)
        out[name] = float(f"{float(err.max()):.3g}")
    return out


def run_fma_form(H, u0, K, W, ref_state, ref_dts, pg, device, world):
    """The FMA FP64 tier on the same workload and steps: FP64 throughout with
    FMA contraction and refined reciprocals; per-cell errors and dt errors
    against the bit-exact FP64 run (itself bitwise the reference's)."""
    import torch
    from hydro_b200 import Domain
    d = Domain(H, precision="fma")
    d.upload(u0)
    d.set_clock()
    d.launch_steps(W)
    d.synchronize()
    d.upload(u0)
    d.reserve_dts(K)
    d.set_clock()
    st = torch.cuda.ExternalStream(d.stream_ptr, device=device)
    barrier(pg, device)
    g0, g1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    g0.record(st)
    d.launch_steps(K)
    g1.record(st)
    g1.synchronize()
    ms = all_max(pg, g0.elapsed_time(g1), device)
    u = d.download()
    dts = d.get_dts(K)
    kern = d.kernels()
    d.close()
    dt_rel = float(np.max(np.abs(dts - ref_dts) / ref_dts))
    return {"value": round(world * H.nx * H.ny * K / (ms / 1e3) / 1e6, 3),
            "unit": "Mcell-updates/s", "ms_per_step": round(ms / K, 4),
            "kernels": {"x": kern[0], "y": kern[1]},
            "max_err_vs_fp64": tier_errors(u, ref_state), "dt_max_rel_vs_fp64": float(f"{dt_rel:.3g}"),
            "rule": "rho, E relative per cell; momenta relative to max(|cell|, field max); "
                    "the FP64 run is bitwise the reference's",
            "precision": "FP64, FMA contraction, refined reciprocals (HB_PREC_FP64_FMA)"}


def run_energy_noise_form(H, K, W, pg, device, world, seed=20261205):
    """The default workload with the interior total energy scaled by
    1 + 0.01 U(-1, 1) per cell: every interface then has unequal pressures,
    so no Riemann problem is trivial and every one iterates.  Times the
    bit-exact FP64 path and the mixed form over the same steps, with the mixed
    errors against the FP64 state."""
    import torch
    from hydro_b200 import Domain
    from hydro_b200.params import init_noisy_blast
    u0 = init_noisy_blast(H, seed, testcase=H.testCase, var=3)
    out = {"workload": f"{H.nx}x{H.ny} centred blast, interior E x (1 + 0.01 U(-1,1)), "
                       f"steps 0..{K - 1}"}
    states = {}
    for prec in ("fp64", "mixed"):
        d = Domain(H, precision=prec)
        d.upload(u0)
        d.set_clock()
        d.launch_steps(W)
        d.synchronize()
        d.upload(u0)
        d.set_clock()
        st = torch.cuda.ExternalStream(d.stream_ptr, device=device)
        barrier(pg, device)
        g0, g1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        g0.record(st)
        d.launch_steps(K)
        g1.record(st)
        g1.synchronize()
        ms = all_max(pg, g0.elapsed_time(g1), device)
        states[prec] = d.download()
        d.close()
        out[prec] = {"value": round(world * H.nx * H.ny * K / (ms / 1e3) / 1e6, 3),
                     "unit": "Mcell-updates/s", "ms_per_step": round(ms / K, 4)}
    out["mixed"]["errors_vs_fp64"] = field_errors(states["mixed"], states["fp64"])
    return out


def run_mixed_bulk_x(H, u0, K, W, pg, device, world, want):
    """The mixed form with its x sweep staged by TMA-engine bulk copies
    (kernel "bulk") over the same steps: whole-job rate, the mean x-sweep
    launch time beside the default x kernel's, and bitwise equality of the
    final state with the default kernels' (`want`)."""
    import torch
    from hydro_b200 import Domain
    out = {}
    for k in ("bulk", "auto"):
        d = Domain(H, precision="mixed", kernels=(k, None))
        d.upload(u0)
        d.set_clock()
        d.launch_steps(W)
        d.synchronize()
        d.upload(u0)
        d.set_clock()
        st = torch.cuda.ExternalStream(d.stream_ptr, device=device)
        barrier(pg, device)
        g0, g1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        g0.record(st)
        d.launch_steps(K)
        g1.record(st)
        g1.synchronize()
        d.synchronize()
        ms = all_max(pg, g0.elapsed_time(g1), device)
        if k == "bulk":
            got = d.download()
            out["value"] = round(world * H.nx * H.ny * K / (ms / 1e3) / 1e6, 3)
            out["unit"] = "Mcell-updates/s"
            out["bitwise_equal_to_default"] = bool(np.array_equal(got.view(np.uint64),
                                                                  want.view(np.uint64)))
            del got
        d.upload(u0)
        d.set_clock()
        d.profile(True)
        d.profile_read(reset=True)
        d.launch_steps(K)
        msx, _, nx_, _ = d.profile_read(reset=True)
        out["x_sweep_ms" if k == "bulk" else "default_x_sweep_ms"] = round(msx / max(nx_, 1), 4)
        d.close()
    return out


def run_mixed_corner_8192(K, W, pg, device, world, nsteps=500, seed=20261203):
    """The mixed-precision form on its own workload: 8192^2, corner blast,
    interior density times 1 + 0.01 U(-1, 1), 500 steps, timed with CUDA
    events (state resident), with its L1 / Linf errors against the bit-exact
    FP64 run of the same input, which is timed too."""
    import torch
    from hydro_b200 import Domain, make_params
    from hydro_b200.params import init_noisy_blast
    H = make_params(8192, 8192, testcase=1)
    u0 = init_noisy_blast(H, seed, testcase=1)
    out = {"workload": "8192x8192 corner blast, interior density x (1 + 0.01 U(-1,1)), "
                       f"{nsteps} steps"}
    states = {}
    for prec in ("fp64", "mixed"):
        d = Domain(H, precision=prec)
        d.upload(u0)
        d.set_clock()
        d.launch_steps(W)
        d.synchronize()
        d.upload(u0)
        d.set_clock()
        st = torch.cuda.ExternalStream(d.stream_ptr, device=device)
        barrier(pg, device)
        g0, g1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        g0.record(st)
        d.launch_steps(nsteps)
        g1.record(st)
        g1.synchronize()
        ms = all_max(pg, g0.elapsed_time(g1), device)
        t, n, _ = d.get_clock()
        states[prec] = (d.download(), t)
        d.close()
        out[prec] = {"value": round(world * H.nx * H.ny * nsteps / (ms / 1e3) / 1e6, 3),
                     "unit": "Mcell-updates/s", "ms_per_step": round(ms / nsteps, 4),
                     "steps": n}
    out["mixed"]["errors_vs_fp64"] = field_errors(states["mixed"][0], states["fp64"][0])
    out["mixed"]["t_rel_diff"] = float(f"{abs(states['mixed'][1] / states['fp64'][1] - 1):.3g}")
    return out


def run_noalloc_form(device):
    """The allocation-free step against the regular domain step on the same
    grids (CUDA events, fixed dt, 50 steps each after 5 warm-up steps)."""
    import ctypes as C
    import torch
    from hydro_b200 import Domain, init_state, load, make_params
    lib = load()
    out = []
    for nx, ny in ((250, 125), (1020, 1020)):
        H = make_params(nx, ny, testcase=1)
        u0 = init_state(H)
        dt = 0.4 / max(nx, ny) ** 2
        d = Domain(H)
        d.upload(u0)
        st = torch.cuda.ExternalStream(d.stream_ptr, device=device)
        for k in range(5):
            d.godunov(1 + k % 2, dt)
        d.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        for k in range(50):
            d.godunov(1 + k % 2, dt)
        e1.record(st)
        e1.synchronize()
        reg = e0.elapsed_time(e1) / 50
        d.close()
        state = torch.from_numpy(u0).to(device)
        s2 = torch.cuda.Stream(device=device)
        h = C.c_void_p(s2.cuda_stream)
        torch.cuda.synchronize(device)
        for k in range(5):
            lib.hydro_b200_godunov_noalloc(C.byref(H), state.data_ptr(), 1 + k % 2, dt, h)
        f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        f0.record(s2)
        for k in range(50):
            lib.hydro_b200_godunov_noalloc(C.byref(H), state.data_ptr(), 1 + k % 2, dt, h)
        f1.record(s2)
        f1.synchronize()
        na = f0.elapsed_time(f1) / 50
        out.append({"grid": f"{nx}x{ny}", "noalloc_ms_per_step": round(na, 4),
                    "regular_ms_per_step": round(reg, 4), "ratio": round(na / reg, 3)})
    return out


def run_vtk_form(H, u):
    """One VTK output of the state `u` (the output path, vtkfile.c:140-352):
    the library's vtkfile, which encodes on the GPU from the device mirror.
    Its CPU baseline is the reference's own vtkfile.c (oracle/_ref), fed by a
    device-to-host copy of the state (what a host writer needs when the state
    lives on the GPU).  Both write the same files, compared byte for byte, to
    local temporary directories; wall time of one call each."""
    import ctypes as C
    import filecmp
    import shutil
    import tempfile

    from hydro_b200 import HydroRun
    from hydro_b200._lib import check
    run = HydroRun(H, u.copy())
    run.sync_to_device()  # the state is resident before the timed call
    lib = run.lib
    out = {"unit": "ms per output", "cells": H.nx * H.ny,
           "text_bytes": 4 * int(lib.hydro_b200_vtk_base64_len(H.nx, H.ny))}
    cwd = os.getcwd()
    dirs = [tempfile.mkdtemp(prefix="hb_vtk_"), tempfile.mkdtemp(prefix="hb_vtk_")]
    try:
        os.chdir(dirs[0])
        lib.vtkfile(1, H, C.byref(run.Hv))  # first call: buffers, directories
        t0 = time.perf_counter()
        lib.vtkfile(1, H, C.byref(run.Hv))
        out["value"] = round((time.perf_counter() - t0) * 1e3, 2)
        check()
        try:
            from oracle import oracle as O
            if not O.ref_available():
                raise RuntimeError("reference not compiled")
            os.chdir(dirs[1])
            with quiet_stdout():  # the reference prints its set-up and decomposition
                ref = O.RefState(O.make_param(H.nx, H.ny), 0)
                t0 = time.perf_counter()
                ref.set(run.sync_to_host())
                ref.vtkfile(1)
                ref_ms = (time.perf_counter() - t0) * 1e3
                ref.close()
            names = [os.path.relpath(os.path.join(dp, f), dirs[0])
                     for dp, _, fs in os.walk(dirs[0]) for f in fs]
            out["files_identical"] = all(filecmp.cmp(os.path.join(dirs[0], n),
                                                     os.path.join(dirs[1], n), shallow=False)
                                         for n in names)
            out["cpu_baseline"] = {"value": round(ref_ms, 2), "unit": "ms per output",
                                   "cores": 1, "kind": "reference",
                                   "sample": "device-to-host copy of the state, then "
                                             "vtkfile.c on it (one output)"}
        except Exception as e:  # the reference build is optional here
            out["cpu_baseline"] = None
            out["cpu_baseline_note"] = str(e)[:200]
    finally:
        os.chdir(cwd)
        run.close()
        for d in dirs:
            shutil.rmtree(d, ignore_errors=True)
    return out


def run_batched_form(device, seed=20261203, n=256, nsteps=100):
    """The batched workload: n seeded instances (sides log-uniform in
    [64, 1024], multiples of 8), mixed precision, nsteps steps each, one
    persistent launch per sweep, CUDA graphs, autotuned tiles (tuned on a
    throwaway batch of the same mix, then timed on a fresh one)."""
    import torch
    from hydro_b200 import Batch, make_blast_mix
    mix = make_blast_mix(n, seed)
    H0 = mix[0][0]
    arena = sum(Batch.bytes_needed(H) for H, _ in mix) + (1 << 20)
    tb = Batch(H0, n, arena, precision="mixed")
    for H, u in mix:
        tb.add(H, u, nstepmax=nsteps)
    tb.autotune(steps=1)
    tuning = tb.tuning()
    tb.close()
    b = Batch(H0, n, arena, precision="mixed")
    slots = [b.add(H, u, nstepmax=nsteps) for H, u in mix]
    b.autotune(steps=1)  # cache hit: applies the tuning without stepping
    b.steps(0)
    b.synchronize()
    st = torch.cuda.ExternalStream(b.stream_ptr, device=device)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    l0 = b.launch_count
    e0.record(st)
    b.steps(nsteps)
    e1.record(st)
    e1.synchronize()
    ms = e0.elapsed_time(e1)
    active, nstep, _ = b.table()
    done = int(sum(1 for s in slots if nstep[s] == nsteps))
    cells = sum(H.nx * H.ny for H, _ in mix)
    launches = b.launch_count - l0
    # Accuracy of every instance against its FP64 run: the same mix as an FP64
    # batch, whose instances equal their single-grid runs bit for bit (tested).
    got = [b.download(s) for s in slots]
    b.close()
    fb = Batch(H0, n, arena, precision="fp64")
    fslots = [fb.add(H, u, nstepmax=nsteps) for H, u in mix]
    fb.steps(nsteps)
    fb.synchronize()
    worst = {"rho": 0.0, "E": 0.0}
    for i, s in enumerate(fslots):
        err = field_errors(got[i], fb.download(s))
        for v in worst:
            worst[v] = max(worst[v], err[v]["l1_rel"])
    fb.close()
    seq = run_batched_sequential(device, mix, nsteps, got)
    return {"workload": f"{n} seeded blast instances, sides 64..1024, {nsteps} steps each",
            "value": round(cells * nsteps / (ms / 1e3) / 1e6, 3), "unit": "Mcell-updates/s",
            "ms": round(ms, 3), "instances_finished": done, "cells": cells,
            "graph_launches": nsteps, "kernel_launches": launches, "tuning": tuning,
            "precision": "mixed",
            "l1_rel_vs_fp64_max": {"sample": f"all {n} instances (FP64 batch of the same mix)",
                                   **{v: float(f"{x:.3g}") for v, x in worst.items()}},
            "same_instances_one_by_one": seq}


def run_batched_sequential(device, mix, nsteps, batched_states):
    """The batched workload's instances solved one after another as single
    grids (mixed precision, each with its own domain, the state resident,
    CUDA events around each instance's steps): the rate the same work reaches
    without batching, and whether every instance equals its batched result
    bit for bit."""
    import torch
    from hydro_b200 import Domain
    total_ms, cells, same = 0.0, 0, True
    for i, (H, u) in enumerate(mix):
        d = Domain(H, precision="mixed")
        d.upload(u)
        d.set_clock()
        d.synchronize()
        st = torch.cuda.ExternalStream(d.stream_ptr, device=device)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        d.launch_steps(nsteps)
        e1.record(st)
        e1.synchronize()
        total_ms += e0.elapsed_time(e1)
        cells += H.nx * H.ny
        same = same and bool(np.array_equal(d.download().view(np.uint64),
                                            batched_states[i].view(np.uint64)))
        d.close()
    return {"value": round(cells * nsteps / (total_ms / 1e3) / 1e6, 3),
            "unit": "Mcell-updates/s", "ms": round(total_ms, 3),
            "bitwise_equal_to_batched": same}


def serving_accuracy_requests():
    """A labelled mix for the served results' accuracy at large sides: four
    requests of side 1024..1536 and four of side 128..256 (tend 0.01, blast
    parameters drawn as in the stream), arriving within 50 ms, so that they
    are served together."""
    from hydro_b200.serve import Request, poisson_requests
    sides = [1024, 1536, 1280, 1088, 128, 192, 256, 136]
    base = poisson_requests(len(sides), 100.0, 20261205, 128, 256, 0.01, 0.01)
    return [Request(k, 0.00625 * k, sides[k], 0.01, r.bx, r.by, r.e0, r.rho)
            for k, r in enumerate(base)]


def solve_fp64(req):
    """A served request solved alone in FP64 until its tend."""
    from hydro_b200 import Batch
    from hydro_b200.batch import blast_spec, blast_state
    H, rho, e_bg, cell, eb = blast_spec(req.side, req.side, req.bx, req.by, req.e0, req.rho)
    b = Batch(H, capacity=1, arena_bytes=Batch.bytes_needed(H) + 4096, precision="fp64")
    s = b.add(H, blast_state(H, rho, e_bg, cell, eb), tend=req.tend)
    while b.status(s)["active"]:
        b.steps(64)
    u = b.download(s)
    b.close()
    return u


def run_serving_form(label, rate, n, side_lo, side_hi, tend_lo, tend_hi, wall_s, seed=20261204,
                     budget_bytes=None, priority_every=0, sample_small=6, requests=None):
    """The serving loop (continuous batching) on a Poisson request stream;
    arena = 80% of the free HBM unless budget_bytes is given; time-bounded.
    With priority_every = k, every k-th request has priority 1 (the others 0)
    and the server preempts: latencies are also reported per class."""
    import dataclasses
    import torch
    from hydro_b200 import make_params
    from hydro_b200.serve import BatchBackend, Server, poisson_requests
    free, total = torch.cuda.mem_get_info()
    budget = int(0.8 * free) if budget_bytes is None else int(budget_bytes)
    reqs = requests if requests is not None else poisson_requests(n, rate, seed, side_lo, side_hi,
                                                                  tend_lo, tend_hi)
    if priority_every:
        reqs = [dataclasses.replace(r, priority=1 if r.rid % priority_every == 0 else 0)
                for r in reqs]
    # Accuracy of what was served: the first few small requests are kept and
    # compared with their FP64 solves.
    sample = set([r.rid for r in reqs if r.side <= 256][:sample_small])
    if requests is not None:
        sample = set(r.rid for r in reqs)  # an explicit request list: every result is checked
    be = BatchBackend(make_params(128, 128), budget, capacity=4096, keep_results=sample)
    st = Server(be, preempt=bool(priority_every)).run(reqs, max_wall_s=wall_s)
    be.close()
    out = st.summary()
    if priority_every:
        prio = {r.rid: r.priority for r in reqs}
        for cls in (1, 0):
            lat = np.array([c[1] for c in st.completed if prio[c[0]] == cls])
            out[f"priority_{cls}"] = {
                "completed": int(lat.size),
                "p50_s": round(float(np.percentile(lat, 50)), 4) if lat.size else None,
                "p99_s": round(float(np.percentile(lat, 99)), 4) if lat.size else None}
    worst = {"rho": 0.0, "E": 0.0}
    by_id = {r.rid: r for r in reqs}
    for rid, u in be.results.items():
        err = field_errors(u, solve_fp64(by_id[rid]))
        for v in worst:
            worst[v] = max(worst[v], err[v]["l1_rel"])
    sides = sorted(by_id[rid].side for rid in be.results)
    out["l1_rel_vs_fp64_max"] = {"sample": f"{len(be.results)} completed requests, sides {sides}",
                                 **{v: float(f"{x:.3g}") for v, x in worst.items()}}
    out.update({"label": label, "lambda_per_s": rate, "requests_offered": n,
                "sides": [side_lo, side_hi], "tend": [tend_lo, tend_hi],
                "hbm_budget_gb": round(budget / 1e9, 1), "wall_limit_s": wall_s,
                "precision": "mixed"})
    return out


class quiet_stdout:
    """Route file descriptor 1 to /dev/null (the reference's C code prints
    set-up messages), so that the bench's stdout is its JSON line alone."""

    def __enter__(self):
        sys.stdout.flush()
        self.devnull = os.open(os.devnull, os.O_WRONLY)
        self.saved = os.dup(1)
        os.dup2(self.devnull, 1)
        return self

    def __exit__(self, *exc):
        os.dup2(self.saved, 1)
        os.close(self.saved)
        os.close(self.devnull)
        return False


def cpu_reference_sample(wl, budget_s, max_steps, warm=1):
    """The reference's own C99/OpenMP code (oracle/_ref) on the host cores,
    falling back to the C restatement (oracle/_build) where the reference was
    not compiled.  Runs whole time steps of the workload from its initial
    state until budget_s is spent (at least one timed step)."""
    from oracle import oracle as O
    p = O.make_param(wl["nx"], wl["ny"], boundary=(1, 1, 1, 1))
    cores = os.cpu_count() or 1
    O.oracle_lib().orc_set_threads(cores)
    if O.ref_available():
        kind = "reference"
        with quiet_stdout():
            r = O.RefState(p, wl["testcase"], nxystep=256)
            t0 = time.perf_counter()
            r.run(warm)
            tw = time.perf_counter() - t0
            nrun = max(1, min(max_steps, int(budget_s / max(tw / max(warm, 1), 1e-6))))
            n, dts, _, mcs_avg, el = r.run(warm + nrun)
            r.close()
        desc = (f"reference C99/OpenMP (oracle/_ref, gcc -O3 -fopenmp -mavx2) on "
                f"{wl['nx']}x{wl['ny']}: steps {warm}..{warm + n - 1} after {warm} warm-up "
                f"step(s), {cores} OpenMP threads")
    else:
        kind = "port"
        u = O.init_state(p, wl["testcase"])
        t0 = time.perf_counter()
        n, _, _ = O.run(p, u, max(1, min(max_steps, 2)))
        el = time.perf_counter() - t0
        desc = (f"C restatement (oracle/_build, OpenMP over lines) on {wl['nx']}x{wl['ny']}: "
                f"{n} steps, {cores} threads")
    mcs = wl["nx"] * wl["ny"] * n / el / 1e6
    return {"value": round(mcs, 3), "unit": "Mcell-updates/s", "cores": cores, "kind": kind,
            "sample": desc, "steps": n, "seconds": round(el, 3)}


NML_TEMPLATE = """&RUN
tend=1e9
nstepmax={nsteps}
noutput=0
/
&MESH
nx={nx}
ny={ny}
nxystep={nxystep}
dx={dx}
boundary_left=1
boundary_right=1
boundary_down=1
boundary_up=1
testcase={tc}
/
&HYDRO
courant_factor=0.8
niter_riemann=10
/
"""


def reference_binary_runs():
    """The reference application itself (oracle/_ref/hydro, main.c) on the host
    cores with OMP_NUM_THREADS = nproc and OMP_PROC_BIND = close: its own
    "Average MC/s" line (main.c:510-513, which leaves out steps <= 5) for the
    250x125 corner case (100 steps), the 4096^2 centred blast and a 6000^2
    centred blast as in the reference's 6000^2 input (dx 0.05), 12 steps each."""
    import re
    import shutil
    import subprocess
    import tempfile
    exe = os.path.join(ROOT, "oracle", "_ref", "hydro")
    if not os.path.exists(exe):
        return None
    cpu_model = ""
    try:
        with open("/proc/cpuinfo") as f:
            cpu_model = next((l.split(":", 1)[1].strip() for l in f if l.startswith("model name")),
                             "")
    except OSError:
        pass
    nproc = os.cpu_count() or 1
    env = dict(os.environ, OMP_NUM_THREADS=str(nproc), OMP_PROC_BIND="close")
    cases = [("250x125 corner blast, 100 steps", 250, 125, 125, 0.004, 1, 100),
             ("4096x4096 centred blast, 12 steps", 4096, 4096, 256, 1.0 / 4096, 0, 12),
             ("6000x6000 centred blast (dx 0.05), 12 steps", 6000, 6000, 1024, 0.05, 0, 12)]
    runs = []
    d = tempfile.mkdtemp(prefix="hb_ref_")
    try:
        for label, nx, ny, nxystep, dx, tc, nsteps in cases:
            nml = os.path.join(d, "in.nml")
            with open(nml, "w") as f:
                f.write(NML_TEMPLATE.format(nsteps=nsteps, nx=nx, ny=ny, nxystep=nxystep,
                                            dx=repr(dx), tc=tc))
            r = subprocess.run([exe, "-i", nml], cwd=d, env=env, capture_output=True,
                               text=True, timeout=600)
            m = re.search(r"Average MC/s:\s*([0-9.eE+-]+)", r.stdout)
            runs.append({"case": label, "average_mcs": float(m.group(1)) if m else None,
                         "rc": r.returncode})
    finally:
        shutil.rmtree(d, ignore_errors=True)
    return {"binary": "oracle/_ref/hydro (the reference application, gcc -O3 -fopenmp -mavx2)",
            "cpu_model": cpu_model, "nproc": nproc,
            "env": f"OMP_NUM_THREADS={nproc} OMP_PROC_BIND=close", "runs": runs}


def run_reference_arm(args, wl):
    world, rank, local, pg = dist_setup(False)
    if rank != 0:
        return 0
    budget = float(os.environ.get("HYDRO_BENCH_REF_BUDGET_S", "90"))
    cpu = cpu_reference_sample(wl, budget, args.steps, warm=max(1, min(args.warmup, 3)))
    line = {
        "impl": "reference", "metric": "Mcell-updates/s", "value": cpu["value"],
        "unit": "Mcell-updates/s", "n_gpus": 0, "steps": cpu["steps"], "warmup": args.warmup,
        "ms_per_step": round(cpu["seconds"] / max(cpu["steps"], 1) * 1e3, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (the workload's initial condition, generated in-process)",
        "config": {"workload": wl["name"], "nx": wl["nx"], "ny": wl["ny"],
                   "testcase": wl["testcase"], "steps_requested": args.steps,
                   "parallelism": f"OpenMP {cpu['cores']} threads"},
        "cpu_baseline": {k: cpu[k] for k in ("value", "unit", "cores", "kind", "sample")},
        "e2e": {"value": cpu["value"], "unit": "Mcell-updates/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default="centre_4096")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-mixed", action="store_true")
    ap.add_argument("--no-fma", action="store_true")
    ap.add_argument("--no-noalloc", action="store_true")
    ap.add_argument("--no-batched", action="store_true")
    ap.add_argument("--no-serving", action="store_true")
    ap.add_argument("--no-vtk", action="store_true")
    ap.add_argument("--no-noise", action="store_true")
    ap.add_argument("--no-corner8192", action="store_true")
    ap.add_argument("--serving-wall", type=float, default=20.0)
    ap.add_argument("--knee-wall", type=float, default=8.0)
    args = ap.parse_args()
    wl = WORKLOADS[args.workload]
    if args.warmup < 3:
        print("warning: --warmup < 3", file=sys.stderr)
    if args.impl == "reference":
        return run_reference_arm(args, wl)

    import torch
    world, rank, local, pg = dist_setup(True)
    torch.cuda.set_device(local)
    device = torch.device("cuda", local)

    import hydro_b200
    from hydro_b200 import Domain, HydroRun, init_state, make_params
    lib = hydro_b200.load()
    if lib.hydro_b200_set_device(local) != 0:
        hydro_b200._lib.check()

    nx, ny, K, W = wl["nx"], wl["ny"], args.steps, args.warmup
    H = make_params(nx, ny, testcase=wl["testcase"])
    u0 = init_state(H)
    state_bytes = u0.nbytes
    dom = Domain(H)
    stream = torch.cuda.ExternalStream(dom.stream_ptr, device=device)

    # Warm-up: W steps of the workload (module load, clocks), then back to step 0.
    dom.upload(u0)
    dom.set_clock()
    dom.launch_steps(W)
    dom.synchronize()
    dom.upload(u0)
    dom.set_clock()

    sampler = ClockSampler(local).start()
    time.sleep(0.3)
    barrier(pg, device)
    torch.cuda.synchronize(device)
    dom.synchronize()
    launches0 = dom.launch_count
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    tw0 = time.time()
    e0.record(stream)
    dom.launch_steps(K)
    e1.record(stream)
    e1.synchronize()
    tw1 = time.time()
    dom.synchronize()
    torch.cuda.synchronize(device)
    barrier(pg, device)
    ms = e0.elapsed_time(e1)
    gpu_launches = dom.launch_count - launches0
    sampler.stop()
    clocks = sampler.summary(tw0, tw1)
    ms_max = all_max(pg, ms, device)
    t_end, n_end, dt_end = dom.get_clock()
    assert n_end == K, (n_end, K)
    value = aggregate_mcs(world, nx * ny, K, ms_max)

    # Per-launch duration of the sweep kernel: the same K steps again with an
    # event pair around every sweep launch.
    dom.upload(u0)
    dom.set_clock()
    dom.profile(True)
    dom.profile_read(reset=True)
    dom.launch_steps(K)
    msx, msy, nxl, nyl = dom.profile_read(reset=True)
    dom.profile(False)
    sweep_ms = (msx + msy) / max(nxl + nyl, 1)
    kern = dom.kernels()
    alg_bytes = BYTES_PER_CELL_SWEEP * nx * ny
    achieved = alg_bytes / (sweep_ms / 1e3) / 1e9
    peak, peak_kind = measured_peak_hbm()
    dom.close()

    # The mixed-precision form on the same workload and steps, with its error
    # against the FP64 state.
    forms = {}
    ref_state = None
    if not (args.no_mixed and args.no_fma):
        dref = Domain(H)
        dref.upload(u0)
        dref.reserve_dts(K)
        dref.set_clock()
        dref.launch_steps(K)
        ref_state = dref.download()
        ref_dts = dref.get_dts(K)
        dref.close()
    if not args.no_fma:
        forms["fp64_fma"] = run_fma_form(H, u0, K, W, ref_state, ref_dts, pg, device, world)
    if not args.no_mixed:
        dm = Domain(H, precision="mixed")
        dm.upload(u0)
        dm.set_clock()
        dm.launch_steps(W)
        dm.synchronize()
        dm.upload(u0)
        dm.set_clock()
        sm = torch.cuda.ExternalStream(dm.stream_ptr, device=device)
        barrier(pg, device)
        g0, g1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        g0.record(sm)
        dm.launch_steps(K)
        g1.record(sm)
        g1.synchronize()
        mix_ms = all_max(pg, g0.elapsed_time(g1), device)
        mix_state = dm.download()
        mix_kernels = dm.kernels()
        dm.close()
        bulk = run_mixed_bulk_x(H, u0, K, W, pg, device, world, mix_state)
        err = field_errors(mix_state, ref_state)
        forms["mixed"] = {"value": round(world * nx * ny * K / (mix_ms / 1e3) / 1e6, 3),
                          "unit": "Mcell-updates/s", "ms_per_step": round(mix_ms / K, 4),
                          "speedup_vs_fp64": round(ms_max / mix_ms, 3),
                          "errors_vs_fp64": err,
                          "kernels": {"x": mix_kernels[0], "y": mix_kernels[1]},
                          # the same 128 B per cell-step of FP64 state as the plain path
                          "hbm_gbs_per_step": round(world * nx * ny * K * BYTES_PER_CELL_STEP
                                                    / (mix_ms / 1e3) / 1e9, 1),
                          "hbm_frac_of_measured_peak": round(
                              world * nx * ny * K * BYTES_PER_CELL_STEP / (mix_ms / 1e3) / 1e9
                              / measured_peak_hbm()[0], 4),
                          "x_bulk_copy_staging": bulk,
                          "precision": "FP32 stages; FP64 Newton p*, update, Courant"}
        if rank == 0 and world == 1:
            forms["mixed"]["beside_reference_fp32_build"] = mixed_beside_reference_fp32()
        del mix_state

    ref_state = None
    if not args.no_noise:
        forms["energy_noise"] = run_energy_noise_form(H, K, W, pg, device, world)
    if not args.no_mixed and not args.no_corner8192:
        forms["mixed_corner_8192"] = run_mixed_corner_8192(K, W, pg, device, world)
    if not args.no_noalloc and rank == 0 and world == 1:
        forms["noalloc"] = run_noalloc_form(device)
    if not args.no_vtk and rank == 0 and world == 1:
        forms["vtk_output"] = run_vtk_form(H, dom_state_after(H, u0, min(K, 20), "fp64"))
    if not args.no_batched and rank == 0:
        forms["batched"] = run_batched_form(device)
    if not args.no_serving and rank == 0:
        forms["serving"] = run_serving_form(
            "configured stream: lambda 200/s, sides 128..4096, tend 0.01..0.1 (time-bounded)",
            200.0, 10000, 128, 4096, 0.01, 0.1, args.serving_wall)
        # Arrival rates around the knee, where the offered load meets the
        # batch's throughput (labelled streams of smaller solves).
        forms["serving_knee"] = [run_serving_form(
            f"labelled stream: lambda {lam:g}/s, sides 128..512, tend 0.01..0.03",
            lam, int(lam * args.knee_wall * 1.5) + 10, 128, 512, 0.01, 0.03, args.knee_wall,
            sample_small=2) for lam in (20.0, 80.0, 160.0, 320.0, 640.0, 1280.0)]
        forms["serving_accuracy"] = run_serving_form(
            "labelled mix: sides 1024..1536 and 128..256, tend 0.01, arriving within 50 ms; "
            "every result against its FP64 solve", 0.0, 8, 128, 1536, 0.01, 0.01, 60.0,
            requests=serving_accuracy_requests())
        forms["serving_priority"] = run_serving_form(
            "priority mix (labelled): lambda 40/s, sides 128..768, tend 0.01..0.03, every 4th "
            "request priority 1 with preemption, 128 MB arena (memory-bound on purpose)",
            40.0, 1500, 128, 768, 0.01, 0.03, args.serving_wall, budget_bytes=128 << 20,
            priority_every=4)

    # End to end through the reference entry points on a pinned host array.
    e2e = None
    if not args.no_e2e:
        pinned = torch.empty(u0.shape, dtype=torch.float64, pin_memory=True)
        host = pinned.numpy()
        host[...] = u0
        run = HydroRun(H, host)
        est = torch.cuda.ExternalStream(run.stream_ptr, device=device)  # creates the mirror
        barrier(pg, device)
        f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        f0.record(est)
        run.sync_to_device()
        run.run_host_loop(K)
        run.sync_to_host()
        f1.record(est)
        f1.synchronize()
        e2e_ms = all_max(pg, f0.elapsed_time(f1), device)
        run.close()
        e2e = {"value": round(world * nx * ny * K / (e2e_ms / 1e3) / 1e6, 3),
               "unit": "Mcell-updates/s",
               "h2d_bytes_per_step": round(state_bytes / K, 1),
               "d2h_bytes_per_step": round((state_bytes + 16 * ((K + 1) // 2)) / K, 1),
               "path": "compute_deltat + hydro_godunov (reference ABI) on a pinned host uold; "
                       "upload, per-even-step Courant read-back and final download timed"}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        budget = float(os.environ.get("HYDRO_BENCH_CPU_BUDGET_S", "20"))
        cpu = cpu_reference_sample(wl, budget, 50, warm=1)
        cpu = {k: cpu[k] for k in ("value", "unit", "cores", "kind", "sample")}
        cpu["reference_application"] = reference_binary_runs()

    if pg is not None:
        barrier(pg, device)
        pg.destroy_process_group()
    if rank != 0:
        return 0
    # The committed ncu traffic figure is for the 4096^2 workload only.
    traffic = ncu_traffic_per_launch() if args.workload == "centre_4096" else None
    line = {
        "metric": "Mcell-updates/s", "value": round(value, 3), "unit": "Mcell-updates/s",
        "n_gpus": world, "steps": K, "warmup": W, "ms_per_step": round(ms_max / K, 4),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (the workload's initial condition, generated in-process)",
        "config": {"workload": wl["name"], "nx": nx, "ny": ny, "testcase": wl["testcase"],
                   "steps": f"0..{K - 1} of the {wl['run_steps']}-step run",
                   "precision": "fp64 (bitwise equal to the reference)",
                   "parallelism": "replicas" if world > 1 else "single GPU",
                   "l2": f"state {state_bytes / 1e6:.1f} MB per buffer > 126 MB L2; no flush"},
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak,
                     "unit": "GB/s", "frac": round(achieved / peak, 4),
                     "traffic": traffic,
                     "kernel": f"FP64 sweeps: x {kern[0]} window, y {kern[1]} "
                               f"({KERNEL_NAMES[kern[0]]} and {KERNEL_NAMES[kern[1]]})",
                     "alg_bytes_per_launch": alg_bytes, "launch_ms": round(sweep_ms, 4),
                     "fp64_pipe": ncu_fp64_pipe(),
                     "peak_kind": peak_kind},
        "gpu_launches": gpu_launches,
        "clocks": clocks,
        "e2e": e2e,
        "cpu_baseline": cpu,
        "forms": forms,
    }
    print(json.dumps(line), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())

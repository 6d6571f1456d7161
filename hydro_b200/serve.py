"""Serving loop: continuous batching of HydroC solve requests.

Requests (a square grid with a single blast and an end time) arrive by a
Poisson process.  The loop admits them first-come first-served into a batch
(hb_batch) while their resident state fits the HBM budget, advances every
admitted solve together -- each with its own dt -- in chunks of global steps,
and retires solves as their clocks pass tend, which frees slots and memory
for the queue.  Time to solution is measured from arrival (so it includes
queueing) to the poll that sees the solve finished.

With ``preempt`` on, requests carry a priority: when the head of the waiting
line cannot be admitted, running solves of lower priority are checkpointed to
host memory and removed (the reference's Continue.dump restart files,
CPP/Domain_Prot.cpp:284-411, held in memory) until it fits; they wait with
their checkpoint and resume bit for bit when memory frees up.  Waiting solves
are admitted by priority, then arrival.  A request larger than the whole
budget is rejected at arrival instead of blocking the line.

The loop talks to a backend (``BatchBackend`` for the GPU); the bookkeeping
is independent of it, so it is tested on the CPU with a simulated backend.
"""
from __future__ import annotations

import math
import time
from collections import deque
from dataclasses import dataclass, field

import numpy as np

from .batch import Batch, blast_spec, _u01
from .params import make_params


@dataclass
class Request:
    rid: int
    arrival: float   # seconds after the start of the stream
    side: int        # square grid side (nx = ny)
    tend: float
    bx: float
    by: float
    e0: float
    rho: float
    priority: int = 0

    @property
    def cells(self) -> int:
        return self.side * self.side


def poisson_requests(n: int, rate: float, seed: int, side_lo: int = 128, side_hi: int = 4096,
                     tend_lo: float = 0.01, tend_hi: float = 0.1) -> list:
    """n requests: exponential inter-arrival times of mean 1/rate; square side
    log-uniform in [side_lo, side_hi] rounded to a multiple of 8; tend
    uniform in [tend_lo, tend_hi]; blast as in the batched workload (cell
    uniform, E0 log-uniform in [0.1, 10]/dx^2, density uniform in [0.5, 2]).
    Draws are SplitMix64 of (seed, stream, request index)."""
    idx = np.arange(n, dtype=np.uint64)
    gaps = -np.log1p(-_u01(seed, 11, idx)) / rate
    arrivals = np.cumsum(gaps)
    lo, hi = math.log(side_lo), math.log(side_hi)
    sides = np.clip(np.rint(np.exp(lo + (hi - lo) * _u01(seed, 12, idx)) / 8) * 8, side_lo,
                    side_hi).astype(int)
    tends = tend_lo + (tend_hi - tend_lo) * _u01(seed, 13, idx)
    bx, by = _u01(seed, 14, idx), _u01(seed, 15, idx)
    e0 = np.exp(math.log(0.1) + (math.log(10.0) - math.log(0.1)) * _u01(seed, 16, idx))
    rho = 0.5 + 1.5 * _u01(seed, 17, idx)
    return [Request(int(k), float(arrivals[k]), int(sides[k]), float(tends[k]), float(bx[k]),
                    float(by[k]), float(e0[k]), float(rho[k])) for k in range(n)]


class BatchBackend:
    """GPU backend: one hb_batch whose arena is the HBM budget."""

    def __init__(self, H, budget_bytes: int, capacity: int = 1024, precision: str = "mixed",
                 keep_results=False):
        """keep_results: True to keep every finished state (host memory), or a
        set of request ids to keep only those."""
        self.batch = Batch(H, capacity, budget_bytes, precision=precision)
        self.budget = budget_bytes
        self.capacity = capacity
        self.keep_results = keep_results
        self.results = {}

    def try_admit(self, req: Request) -> int:
        H, rho, e_bg, cell, e_blast = blast_spec(req.side, req.side, req.bx, req.by, req.e0,
                                                 req.rho)
        return self.batch.try_add_blast(H, rho, e_bg, cell, e_blast, tend=req.tend)

    def steps(self, k: int) -> None:
        self.batch.steps(k)

    def table(self):
        return self.batch.table()

    def can_ever_fit(self, req: Request) -> bool:
        """Whether the request fits the arena at all (an empty one)."""
        return Batch.bytes_needed(make_params(req.side, req.side)) <= self.budget

    def checkpoint(self, slot: int) -> dict:
        return self.batch.checkpoint(slot)

    def fits_after(self, req: Request, ckpt, slots: list) -> bool:
        """Whether `req` (or its checkpoint) would fit once `slots` are
        evicted, by free bytes (the arena's first fit may still find it
        fragmented)."""
        nx, ny = (req.side, req.side) if ckpt is None else (ckpt["nx"], ckpt["ny"])
        need = Batch.bytes_needed(make_params(nx, ny))
        freed = sum(Batch.bytes_needed(self.batch.params[s]) for s in slots)
        return need <= self.batch.arena_free + freed

    def try_resume(self, ckpt: dict) -> int:
        return self.batch.resume(ckpt)

    def evict(self, slot: int) -> None:
        self.batch.remove(slot)

    def release(self, slot: int, req: Request) -> None:
        keep = self.keep_results
        if keep is True or (keep and req.rid in keep):
            self.results[req.rid] = self.batch.download(slot)
        self.batch.remove(slot)

    def close(self) -> None:
        self.batch.close()


# Side buckets of the latency breakdown: (label, lowest side, highest side).
SIDE_BUCKETS = (("side<=256", 0, 256), ("256<side<=1024", 257, 1024), ("side>1024", 1025, 1 << 30))


def _pct(x, q):
    return round(float(np.percentile(x, q)), 4) if len(x) else None


@dataclass
class ServeStats:
    completed: list = field(default_factory=list)   # (rid, latency s, steps, cells)
    # Requests still queued or running when the loop stopped: (rid, age s at
    # the cutoff, "queued" | "running", cells).  Their time to solution is
    # unknown but at least their age.
    censored: list = field(default_factory=list)
    admitted: int = 0
    arrived: int = 0
    wall_s: float = 0.0
    cell_steps: float = 0.0
    queue_samples: list = field(default_factory=list)  # (time s, queued, running)
    chunks: int = 0
    unfinished: int = 0
    preemptions: int = 0
    rejected: int = 0

    def summary(self) -> dict:
        lat = np.array([c[1] for c in self.completed]) if self.completed else np.zeros(0)
        ages = np.array([c[1] for c in self.censored]) if self.censored else np.zeros(0)
        q = [s[1] for s in self.queue_samples]
        # Every request that arrived and was not rejected: completed ones at
        # their time to solution, censored ones at their age.  Percentiles of
        # this set are lower bounds on the true percentiles of the stream.
        both = np.concatenate([lat, ages])
        by_side = {}
        for label, lo, hi in SIDE_BUCKETS:
            cl = [c[1] for c in self.completed if lo <= math.isqrt(c[3]) <= hi]
            ce = [c[1] for c in self.censored if lo <= math.isqrt(c[3]) <= hi]
            by_side[label] = {"completed": len(cl), "p50_s": _pct(cl, 50), "p99_s": _pct(cl, 99),
                              "censored": len(ce),
                              "censored_age_max_s": round(max(ce), 4) if ce else None,
                              "p50_lower_bound_s": _pct(cl + ce, 50),
                              "p99_lower_bound_s": _pct(cl + ce, 99)}
        return {
            "arrived": self.arrived, "admitted": self.admitted,
            "completed": len(self.completed),
            "wall_s": round(self.wall_s, 3),
            "mcell_updates_per_s": round(self.cell_steps / max(self.wall_s, 1e-9) / 1e6, 3),
            "p50_s": _pct(lat, 50),
            "p99_s": _pct(lat, 99),
            "latency_note": "p50_s/p99_s cover completed requests only; *_lower_bound_s also "
                            "count every censored request (queued or running at the cutoff) "
                            "at its age, a lower bound on its time to solution",
            "censored": {"count": len(self.censored),
                         "queued": sum(1 for c in self.censored if c[2] == "queued"),
                         "running": sum(1 for c in self.censored if c[2] == "running"),
                         "age_p50_s": _pct(ages, 50), "age_p99_s": _pct(ages, 99),
                         "age_max_s": round(float(ages.max()), 4) if ages.size else None},
            "p50_lower_bound_s": _pct(both, 50),
            "p99_lower_bound_s": _pct(both, 99),
            "by_side": by_side,
            "queue_max": max(q) if q else 0,
            "queue_end": q[-1] if q else 0,
            "running_end": self.unfinished,
            "chunks": self.chunks,
            "preemptions": self.preemptions,
            "rejected": self.rejected,
        }


class Server:
    """Continuous batching over a backend: first-come first-served, or by
    priority with preemption (``preempt``)."""

    def __init__(self, backend, chunk_target_s: float = 0.01, max_chunk: int = 256,
                 clock=time.perf_counter, sleep=time.sleep, preempt: bool = False):
        self.backend = backend
        self.chunk_target_s = chunk_target_s
        self.max_chunk = max_chunk
        self.clock = clock
        self.sleep = sleep
        self.preempt = preempt

    def _place(self, req: Request, ckpt) -> int:
        return self.backend.try_admit(req) if ckpt is None else self.backend.try_resume(ckpt)

    def _admit(self, st, waiting: list, running: dict) -> None:
        """Admit from the head of `waiting` (entries [request, checkpoint or
        None, steps counted]) while memory allows.  With preemption, when the
        head does not fit, evict running solves of lower priority (lowest
        first, latest arrival first among equals) -- only if evicting them
        makes room by the backend's estimate."""
        while waiting:
            head = waiting[0]
            req, ckpt, counted = head
            slot = self._place(req, ckpt)
            if slot < 0 and self.preempt:
                victims = sorted((s for s, (r, _) in running.items() if r.priority < req.priority),
                                 key=lambda s: (running[s][0].priority, -running[s][0].arrival))
                chosen = []
                for v in victims:
                    chosen.append(v)
                    if self.backend.fits_after(req, ckpt, chosen):
                        break
                else:
                    chosen = []
                for v in chosen:
                    vreq, vcounted = running.pop(v)
                    vck = self.backend.checkpoint(v)
                    self.backend.evict(v)
                    st.preemptions += 1
                    waiting.append([vreq, vck, vcounted])
                if chosen:
                    slot = self._place(req, ckpt)
                    waiting.sort(key=lambda w: (-w[0].priority, w[0].arrival))
            if slot < 0:
                break
            del waiting[next(i for i, w in enumerate(waiting) if w is head)]
            running[slot] = (req, counted)
            if ckpt is None:
                st.admitted += 1

    def run(self, requests: list, max_wall_s: float) -> ServeStats:
        st = ServeStats()
        pending = deque(sorted(requests, key=lambda r: r.arrival))
        waiting: list = []     # [request, checkpoint or None, steps counted]
        running = {}           # slot -> (request, steps already counted)
        k = 1
        t0 = self.clock()
        while True:
            now = self.clock() - t0
            if now >= max_wall_s or not (pending or waiting or running):
                break
            arrived = False
            while pending and pending[0].arrival <= now:
                req = pending.popleft()
                st.arrived += 1
                if not self.backend.can_ever_fit(req):
                    st.rejected += 1  # larger than the whole budget: it would block the line
                    continue
                waiting.append([req, None, 0])
                arrived = True
            if arrived and self.preempt:
                waiting.sort(key=lambda w: (-w[0].priority, w[0].arrival))
            self._admit(st, waiting, running)
            st.queue_samples.append((now, len(waiting), len(running)))
            if not running:
                if pending:
                    self.sleep(max(0.0, min(pending[0].arrival - now, max_wall_s - now)))
                    continue
                break  # nothing runs, nothing can be admitted, nothing arrives
            c0 = self.clock()
            self.backend.steps(k)
            active, nstep, _ = self.backend.table()
            dtc = self.clock() - c0
            st.chunks += 1
            done_time = self.clock() - t0
            for slot in list(running):
                req, counted = running[slot]
                n = int(nstep[slot])
                st.cell_steps += float(req.cells) * (n - counted)
                running[slot] = (req, n)
                if not active[slot]:
                    st.completed.append((req.rid, done_time - req.arrival, n, req.cells))
                    self.backend.release(slot, req)
                    del running[slot]
            # Next chunk: about chunk_target_s of device work.
            if dtc > 0:
                k = int(max(1, min(self.max_chunk, round(k * self.chunk_target_s / dtc))))
        st.wall_s = self.clock() - t0
        late = [r for r in pending if r.arrival <= st.wall_s]  # arrived, never looked at
        arrived_waiting = len(waiting) + len(late)
        st.arrived += len(late)
        st.queue_samples.append((st.wall_s, arrived_waiting, len(running)))
        st.unfinished = len(running)
        # Censored requests: their age at the cutoff bounds their time to
        # solution.  Arrivals not yet looked at get the arrival rule (rejected
        # when larger than the whole budget).
        fit = [r for r in late if self.backend.can_ever_fit(r)]
        st.rejected += len(late) - len(fit)
        for req in [w[0] for w in waiting] + fit:
            st.censored.append((req.rid, st.wall_s - req.arrival, "queued", req.cells))
        for req, _ in running.values():
            st.censored.append((req.rid, st.wall_s - req.arrival, "running", req.cells))
        return st

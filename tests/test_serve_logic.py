"""Serving-loop bookkeeping on the CPU: a simulated backend with a memory
budget, per-request step counts and a per-cell-step cost, driven by a fake
clock.  Checks FIFO admission under the budget, completion and latency
accounting, work accounting, and queue growth under overload."""
import math

import pytest

from hydro_b200.serve import Request, Server, poisson_requests


class FakeClock:
    def __init__(self):
        self.t = 0.0

    def __call__(self):
        return self.t

    def sleep(self, dt):
        self.t += max(dt, 1e-6)


class SimBackend:
    """Slots with a byte budget (64 B per cell); a request needs
    steps(side, tend) steps; a global step costs sum(cells) * cost s."""

    def __init__(self, clock, budget_cells, cost=1e-9, capacity=64):
        self.clock = clock
        self.budget = budget_cells
        self.cost = cost
        self.capacity = capacity
        self.slots = {}
        self.admitted_order = []
        self.resumed = []
        self.peak = 0

    @staticmethod
    def steps_needed(req):
        return max(1, int(req.side * req.tend * 4))

    def used(self):
        return sum(r.cells for r, _ in self.slots.values())

    def try_admit(self, req):
        if len(self.slots) >= self.capacity or self.used() + req.cells > self.budget:
            return -1
        slot = min(set(range(self.capacity)) - set(self.slots))
        self.slots[slot] = (req, 0)
        self.admitted_order.append(req.rid)
        self.peak = max(self.peak, self.used())
        return slot

    def steps(self, k):
        for _ in range(k):
            cells = 0
            for s, (r, n) in list(self.slots.items()):
                if n < self.steps_needed(r):
                    self.slots[s] = (r, n + 1)
                    cells += r.cells
            self.clock.t += cells * self.cost

    def table(self):
        active = [0] * self.capacity
        nstep = [0] * self.capacity
        for s, (r, n) in self.slots.items():
            active[s] = int(n < self.steps_needed(r))
            nstep[s] = n
        return active, nstep, [0.0] * self.capacity

    def release(self, slot, req):
        del self.slots[slot]

    # preemption: a checkpoint is the request and its step count
    def checkpoint(self, slot):
        req, n = self.slots[slot]
        return {"req": req, "n": n, "nx": req.side, "ny": req.side}

    def evict(self, slot):
        del self.slots[slot]

    def try_resume(self, ck):
        slot = self.try_admit(ck["req"])
        if slot >= 0:
            self.slots[slot] = (ck["req"], ck["n"])
            self.resumed.append(ck["req"].rid)
        return slot

    def can_ever_fit(self, req):
        return req.cells <= self.budget

    def fits_after(self, req, ck, slots):
        freed = sum(self.slots[s][0].cells for s in slots)
        return self.used() - freed + req.cells <= self.budget


def test_poisson_requests_are_seeded_and_in_range():
    a = poisson_requests(2000, 200.0, seed=4)
    b = poisson_requests(2000, 200.0, seed=4)
    assert [r.__dict__ for r in a] == [r.__dict__ for r in b]
    assert all(128 <= r.side <= 4096 and r.side % 8 == 0 for r in a)
    assert all(0.01 <= r.tend <= 0.1 for r in a)
    gaps = [a[i + 1].arrival - a[i].arrival for i in range(len(a) - 1)]
    mean = sum(gaps) / len(gaps)
    assert abs(mean - 1 / 200.0) < 0.1 / 200.0
    logs = [math.log(r.side) for r in a]
    assert abs(sum(logs) / len(logs) - (math.log(128) + math.log(4096)) / 2) < 0.1


def test_light_load_completes_everything_fifo():
    clk = FakeClock()
    be = SimBackend(clk, budget_cells=10**6)
    reqs = poisson_requests(40, 5.0, seed=1, side_lo=32, side_hi=128)
    st = Server(be, clock=clk, sleep=clk.sleep).run(reqs, max_wall_s=1e6)
    assert len(st.completed) == 40 and st.admitted == 40
    assert be.admitted_order == sorted(be.admitted_order)
    by_id = {r.rid: r for r in reqs}
    work = sum(r.cells * SimBackend.steps_needed(r) for r in reqs)
    assert st.cell_steps == work
    for rid, lat, n, cells in st.completed:
        assert n == SimBackend.steps_needed(by_id[rid]) and lat > 0
    s = st.summary()
    assert s["completed"] == 40 and s["p50_s"] <= s["p99_s"]


def test_budget_is_never_exceeded_and_overload_queues():
    clk = FakeClock()
    budget = 3 * 128 * 128
    be = SimBackend(clk, budget_cells=budget, cost=1e-7)
    reqs = poisson_requests(300, 500.0, seed=2, side_lo=64, side_hi=128)
    st = Server(be, clock=clk, sleep=clk.sleep).run(reqs, max_wall_s=0.5)
    assert be.peak <= budget
    s = st.summary()
    assert s["queue_end"] > 0 and s["completed"] < 300
    assert st.admitted == s["completed"] + s["running_end"]


def test_head_of_line_waits_for_memory():
    """A request larger than the free budget waits; later small ones do not
    overtake it (first-come first-served)."""
    clk = FakeClock()
    be = SimBackend(clk, budget_cells=2 * 100 * 100, cost=1e-6)
    reqs = [Request(1, 0.0, 100, 0.05, .5, .5, 1., 1.),      # fits
            Request(3, 0.0005, 120, 0.05, .5, .5, 1., 1.),   # must wait for memory
            Request(2, 0.001, 8, 0.01, .5, .5, 1., 1.)]      # small, arrives last
    st = Server(be, clock=clk, sleep=clk.sleep).run(reqs, max_wall_s=1e3)
    assert be.admitted_order == [1, 3, 2]
    assert len(st.completed) == 3


def test_preemption_by_priority_loses_no_work():
    """Two low-priority solves fill the budget; a high-priority request arrives,
    evicts the latest low-priority one, finishes first, and the evicted solve
    resumes from its checkpoint: every solve completes with exactly its own
    step count and the work adds up."""
    clk = FakeClock()
    be = SimBackend(clk, budget_cells=2 * 100 * 100, cost=1e-6)
    reqs = [Request(1, 0.0, 100, 0.5, .5, .5, 1., 1., priority=0),
            Request(2, 0.001, 100, 0.5, .5, .5, 1., 1., priority=0),
            Request(3, 0.02, 100, 0.1, .5, .5, 1., 1., priority=5)]
    st = Server(be, clock=clk, sleep=clk.sleep, preempt=True, chunk_target_s=0.01).run(
        reqs, max_wall_s=1e3)
    assert st.preemptions == 1 and be.resumed == [2]
    assert be.peak <= be.budget
    done = {rid: n for rid, _, n, _ in st.completed}
    assert done == {r.rid: SimBackend.steps_needed(r) for r in reqs}
    order = [rid for rid, *_ in st.completed]
    assert order.index(3) < order.index(2)
    assert st.cell_steps == sum(r.cells * SimBackend.steps_needed(r) for r in reqs)


def test_no_preemption_without_priority_or_room():
    """Equal priorities never preempt; nor does a request that would not fit
    even after evicting every lower-priority solve."""
    clk = FakeClock()
    be = SimBackend(clk, budget_cells=2 * 100 * 100, cost=1e-6)
    reqs = [Request(1, 0.0, 100, 0.3, .5, .5, 1., 1.),
            Request(2, 0.0, 100, 0.3, .5, .5, 1., 1.),
            Request(3, 0.01, 100, 0.1, .5, .5, 1., 1.)]
    st = Server(be, clock=clk, sleep=clk.sleep, preempt=True).run(reqs, max_wall_s=1e3)
    assert st.preemptions == 0 and be.admitted_order == [1, 2, 3]
    clk = FakeClock()
    be = SimBackend(clk, budget_cells=2 * 100 * 100, cost=1e-6)
    reqs = [Request(1, 0.0, 100, 0.3, .5, .5, 1., 1., priority=1),
            Request(2, 0.0, 100, 0.3, .5, .5, 1., 1., priority=0),
            Request(3, 0.01, 150, 0.1, .5, .5, 1., 1., priority=9)]
    st = Server(be, clock=clk, sleep=clk.sleep, preempt=True).run(reqs, max_wall_s=1e3)
    assert st.preemptions == 0 and len(st.completed) == 2


def test_request_larger_than_the_budget_is_rejected_not_blocking():
    clk = FakeClock()
    be = SimBackend(clk, budget_cells=100 * 100, cost=1e-6)
    reqs = [Request(1, 0.0, 200, 0.05, .5, .5, 1., 1.),   # 4x the budget
            Request(2, 0.001, 64, 0.05, .5, .5, 1., 1.)]
    st = Server(be, clock=clk, sleep=clk.sleep).run(reqs, max_wall_s=1e3)
    assert st.rejected == 1 and [c[0] for c in st.completed] == [2]
    assert st.summary()["rejected"] == 1


def test_overload_reports_censored_requests_and_side_buckets():
    """Under overload the stream is cut off with requests still queued and
    running.  Every arrived, admissible request is either completed or
    censored (with its age at the cutoff as a lower bound on its time to
    solution), the lower-bound percentiles are at least the completed ones'
    order statistics allow, and the side buckets partition both sets."""
    clk = FakeClock()
    be = SimBackend(clk, budget_cells=3 * 128 * 128, cost=1e-7)
    reqs = poisson_requests(400, 500.0, seed=3, side_lo=64, side_hi=2048)
    st = Server(be, clock=clk, sleep=clk.sleep).run(reqs, max_wall_s=0.5)
    s = st.summary()
    assert s["censored"]["count"] > 0 and s["censored"]["queued"] > 0
    assert s["completed"] + s["censored"]["count"] + s["rejected"] == s["arrived"]
    assert s["censored"]["running"] == s["running_end"]
    for rid, age, state, cells in st.censored:
        r = next(q for q in reqs if q.rid == rid)
        assert abs(age - (st.wall_s - r.arrival)) < 1e-9 and state in ("queued", "running")
    assert s["p50_lower_bound_s"] >= min(c[1] for c in st.completed)
    assert s["censored"]["age_max_s"] <= st.wall_s
    buckets = s["by_side"]
    assert sum(b["completed"] for b in buckets.values()) == s["completed"]
    assert sum(b["censored"] for b in buckets.values()) == s["censored"]["count"]


def test_light_load_has_nothing_censored():
    clk = FakeClock()
    be = SimBackend(clk, budget_cells=10**6)
    reqs = poisson_requests(20, 5.0, seed=5, side_lo=32, side_hi=128)
    s = Server(be, clock=clk, sleep=clk.sleep).run(reqs, max_wall_s=1e6).summary()
    assert s["censored"]["count"] == 0 and s["p50_lower_bound_s"] == s["p50_s"]
    assert s["by_side"]["side<=256"]["completed"] == 20

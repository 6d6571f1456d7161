"""The serving loop on the GPU: requests arriving while others run are
admitted as memory frees up, run overlapped in one batch, and each result is
the same as the request solved alone (bitwise: the per-cell arithmetic does
not depend on the company or the tiling)."""
import numpy as np
import pytest

from hydro_b200 import Batch, make_params
from hydro_b200.batch import blast_spec, blast_state
from hydro_b200.serve import BatchBackend, Server, poisson_requests
from _helpers import bitwise_equal

pytestmark = pytest.mark.gpu


def solve_alone(req):
    H, rho, e_bg, cell, eb = blast_spec(req.side, req.side, req.bx, req.by, req.e0, req.rho)
    b = Batch(H, capacity=1, arena_bytes=Batch.bytes_needed(H) + 4096, precision="mixed")
    s = b.add(H, blast_state(H, rho, e_bg, cell, eb), tend=req.tend)
    while b.status(s)["active"]:
        b.steps(16)
    u = b.download(s)
    b.close()
    return u


def test_served_results_equal_alone(product_lib):
    # Near-simultaneous arrivals and a budget for two of the largest requests:
    # most requests queue and are admitted as earlier ones finish.
    reqs = poisson_requests(24, 1e4, seed=9, side_lo=32, side_hi=160, tend_lo=0.002,
                            tend_hi=0.006)
    H = make_params(64, 64)
    budget = 2 * Batch.bytes_needed(make_params(160, 160))
    be = BatchBackend(H, budget, capacity=32, keep_results=True)
    st = Server(be, chunk_target_s=0.002).run(reqs, max_wall_s=120.0)
    be.close()
    s = st.summary()
    assert s["completed"] == len(reqs), s
    assert max(q for _, q, _ in st.queue_samples) > 0  # some requests had to wait
    for req in reqs:
        assert bitwise_equal(be.results[req.rid], solve_alone(req)), req.rid


def test_preempted_solves_resume_bit_for_bit(product_lib):
    """A budget for two mid-size solves; high-priority requests arriving later
    evict low-priority ones (checkpoint to the host, removal), which resume
    when memory frees up.  Every result equals the request solved alone."""
    import dataclasses
    base = poisson_requests(6, 1e4, seed=21, side_lo=96, side_hi=128, tend_lo=0.004,
                            tend_hi=0.006)
    # low priority: long solves (about 250 steps) from t = 0; high priority:
    # short ones arriving 2 ms later, while the first ones run
    reqs = [dataclasses.replace(r, arrival=0.0, tend=0.05, priority=0) for r in base[:3]]
    reqs += [dataclasses.replace(r, arrival=0.002, priority=3) for r in base[3:]]
    budget = 2 * Batch.bytes_needed(make_params(128, 128)) + 4096
    be = BatchBackend(make_params(64, 64), budget, capacity=8, keep_results=True)
    st = Server(be, chunk_target_s=0.002, preempt=True).run(reqs, max_wall_s=120.0)
    be.close()
    s = st.summary()
    assert s["completed"] == len(reqs), s
    assert s["preemptions"] >= 1, s
    for req in reqs:
        assert bitwise_equal(be.results[req.rid], solve_alone(req)), req.rid

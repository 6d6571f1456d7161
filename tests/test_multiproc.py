"""The multi-process path of bench.py on the CPU: two ranks over gloo (the
GPU run uses NCCL with the same calls).  Each rank advances its own replica
(here the C restatement on a small grid, standing in for the device work),
the ranks meet at barriers, the time is the max over ranks and the value is
the whole-job aggregate; the reference arm runs on rank 0 only."""
import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

WORKER = r"""
import json, os, sys, time
sys.path.insert(0, sys.argv[1])
import bench
world, rank, local, pg = bench.dist_setup(False)
from oracle import oracle as O
p = O.make_param(48 + 16 * rank, 40, boundary=(1, 1, 1, 1))
u = O.init_state(p, 0)
bench.barrier(pg, "cpu")
t0 = time.perf_counter()
n, dts, _ = O.run(p, u, 6 + 2 * rank)
ms = (time.perf_counter() - t0) * 1e3 + 5.0 * rank
ms_max = bench.all_max(pg, ms, "cpu")
value = bench.aggregate_mcs(world, 48 * 40, 6, ms_max)
bench.barrier(pg, "cpu")
print(json.dumps({"rank": rank, "world": world, "ms": ms, "ms_max": ms_max, "value": value,
                  "steps": n}))
pg.destroy_process_group()
"""


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def run_ranks(code, world=2, extra_args=()):
    port = free_port()
    procs = []
    for r in range(world):
        env = dict(os.environ, RANK=str(r), LOCAL_RANK=str(r), WORLD_SIZE=str(world),
                   MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), OMP_NUM_THREADS="1")
        procs.append(subprocess.Popen([sys.executable, "-c", code, ROOT, *extra_args], env=env,
                                      stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True))
    outs = []
    for p in procs:
        out, err = p.communicate(timeout=180)
        assert p.returncode == 0, err[-2000:]
        outs.append(out)
    return outs


def test_two_ranks_max_over_ranks_and_aggregate():
    outs = run_ranks(WORKER)
    res = [json.loads(o.strip().splitlines()[-1]) for o in outs]
    assert {r["rank"] for r in res} == {0, 1} and all(r["world"] == 2 for r in res)
    ms_max = max(r["ms"] for r in res)
    assert all(abs(r["ms_max"] - ms_max) < 1e-9 for r in res)
    assert all(abs(r["value"] - 2 * 48 * 40 * 6 / (ms_max / 1e3) / 1e6) < 1e-9 for r in res)
    assert [r["steps"] for r in sorted(res, key=lambda r: r["rank"])] == [6, 8]


REF_ARM = r"""
import sys
sys.path.insert(0, sys.argv[1])
sys.argv = ["bench.py", "--impl", "reference", "--steps", "2", "--warmup", "1",
            "--workload", "corner_250x125"]
import bench
import os
os.environ["HYDRO_BENCH_REF_BUDGET_S"] = "1"
sys.exit(bench.main())
"""


def test_reference_arm_prints_on_rank_zero_only():
    outs = run_ranks(REF_ARM)
    lines = [[l for l in o.splitlines() if l.startswith("{")] for o in outs]
    assert len(lines[0]) == 1 and lines[1] == []
    line = json.loads(lines[0][0])
    assert line["impl"] == "reference" and line["value"] > 0
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["cpu_baseline"]["cores"] >= 1

"""Domain split on the CPU: the decomposition against the reference's own
SplitSurface.c, and the split driver (halo exchange, dt min-reduction, sweep
order) over oracle-computed subdomains -- in one process and as gloo ranks --
against the single-grid oracle run, bit for bit."""
import ctypes as C
import json
import os

import numpy as np
import pytest

from hydro_b200 import init_state, make_params
from hydro_b200.split import (Box, LocalComm, SplitRun, calc_sub_surface, decompose,
                              gather_into, local_params, process_grid, scatter_state)
from oracle import oracle as O
from _split_oracle import OracleSubdomain, orc_param_of
from test_multiproc import ROOT, run_ranks

REF_SPLIT = os.path.join(ROOT, "oracle", "_ref", "libsplit.so")


@pytest.mark.parametrize("nproc,grid", [(1, (1, 1)), (2, (2, 1)), (3, (3, 1)), (4, (2, 2)),
                                        (6, (3, 2)), (8, (4, 2)), (9, (3, 3)), (10, (5, 2)),
                                        (12, (4, 3)), (16, (4, 4)), (18, (6, 3))])
def test_process_grid(nproc, grid):
    assert process_grid(nproc) == grid


@pytest.mark.parametrize("nproc", [5, 7, 11])
def test_process_grid_rejects_what_the_reference_rejects(nproc):
    with pytest.raises(ValueError):
        process_grid(nproc)


@pytest.mark.skipif(not os.path.exists(REF_SPLIT), reason="reference SplitSurface.c not built")
@pytest.mark.parametrize("gx,gy", [(250, 125), (37, 29), (4096, 4096), (1000, 3)])
@pytest.mark.parametrize("nproc", [1, 2, 3, 4, 6, 8, 9, 12])
def test_boxes_match_reference_split_surface(gx, gy, nproc):
    lib = C.CDLL(REF_SPLIT)
    lib.CalcSubSurface.argtypes = [C.c_int] * 7 + [C.POINTER(C.c_int), C.c_int, C.c_int]
    for r in range(nproc):
        box = (C.c_int * 8)(*([0] * 4 + [-1] * 4))
        # parametres.c:290-292: the two passes of the reference
        lib.CalcSubSurface(0, gx, 0, gy, 0, nproc - 1, 0, box, r, 0)
        lib.CalcSubSurface(0, gx, 0, gy, 0, nproc - 1, 0, box, r, 1)
        b = calc_sub_surface(gx, gy, nproc, r)
        assert list(box) == [b.x0, b.x1, b.y0, b.y1, b.up, b.down, b.left, b.right], (r, list(box))


@pytest.mark.parametrize("gx,gy,nproc", [(37, 29, 4), (250, 125, 6), (64, 64, 9), (33, 70, 8)])
def test_boxes_tile_the_grid(gx, gy, nproc):
    boxes = decompose(gx, gy, nproc)
    owner = np.full((gy, gx), -1)
    for r, b in enumerate(boxes):
        assert (owner[b.y0:b.y1, b.x0:b.x1] == -1).all()
        owner[b.y0:b.y1, b.x0:b.x1] = r
        for idim in (1, 2):
            for side in (0, 1):
                nb = b.neighbour(idim, side)
                if nb < 0:
                    continue
                o = boxes[nb]
                assert o.neighbour(idim, 1 - side) == r
                if idim == 1:
                    assert (o.y0, o.y1) == (b.y0, b.y1)
                    assert (o.x1 == b.x0) if side == 0 else (o.x0 == b.x1)
                else:
                    assert (o.x0, o.x1) == (b.x0, b.x1)
                    assert (o.y1 == b.y0) if side == 0 else (o.y0 == b.y1)
    assert (owner >= 0).all()


def test_too_many_ranks_for_the_grid_raises():
    with pytest.raises(ValueError):
        decompose(2, 40, 3)


def test_local_params_open_inner_sides():
    Hg = make_params(100, 60, boundary=(1, 2, 1, 2))
    boxes = decompose(100, 60, 4)
    H = local_params(Hg, boxes[0], 0, 4)
    assert (H.nx, H.ny, H.dx) == (50, 30, Hg.dx)
    assert (H.boundary_left, H.boundary_right, H.boundary_down, H.boundary_up) == (1, 0, 1, 0)
    H3 = local_params(Hg, boxes[3], 3, 4)
    assert (H3.boundary_left, H3.boundary_right, H3.boundary_down, H3.boundary_up) == (0, 2, 0, 2)
    assert (H3.globnx, H3.globny, H3.nproc, H3.mype) == (100, 60, 4, 3)


def single_run(Hg, u0, nsteps):
    p = orc_param_of(Hg)
    u = u0.copy()
    n, dts, t = O.run(p, u, nsteps)
    return u, dts, t


def outer_mask(Hg):
    """Cells a split reproduces: the interior and the ghost lines of the
    physical sides, without the corners."""
    m = np.zeros((Hg.ny + 4, Hg.nx + 4), dtype=bool)
    m[2:-2, :] = True
    m[:, 2:-2] = True
    return m


@pytest.mark.parametrize("gx,gy,tc,nproc,bnd", [
    (37, 29, 0, 4, (1, 1, 1, 1)),
    (40, 24, 1, 2, (1, 1, 1, 1)),
    (31, 45, 2, 6, (1, 1, 1, 1)),
    (48, 36, 0, 9, (2, 2, 2, 2)),
    (50, 30, 0, 3, (1, 2, 2, 1)),
])
@pytest.mark.parametrize("overlap", [False, True])
def test_local_split_equals_single_grid(gx, gy, tc, nproc, bnd, overlap):
    """With overlap, each sweep is issued as its ghost-free part before the
    halo exchange and its edge part after the unpack."""
    Hg = make_params(gx, gy, testcase=tc, boundary=bnd)
    u0 = init_state(Hg, tc)
    want, dts, t = single_run(Hg, u0, 24)
    boxes = decompose(gx, gy, nproc)
    subs = [OracleSubdomain(local_params(Hg, b, r, nproc), b, r, scatter_state(u0, b))
            for r, b in enumerate(boxes)]
    run = SplitRun(Hg, subs, LocalComm(), overlap=overlap)
    assert run.run(24) == 24
    if overlap:
        assert all(len(s.parts) == 2 * 2 * 24 for s in subs)
    got = np.zeros_like(want)
    for s in subs:
        gather_into(got, s.download(), s.box)
    m = outer_mask(Hg)
    assert np.array_equal(got[:, m], want[:, m])
    assert run.dts == list(dts[:24]) and run.t == t


WORKER = r"""
import json, os, sys
sys.path.insert(0, sys.argv[1]); sys.path.insert(0, os.path.join(sys.argv[1], "tests"))
import numpy as np, torch, torch.distributed as dist
from hydro_b200 import init_state, make_params
from hydro_b200.split import DistComm, SplitRun, decompose, gather_into, local_params, scatter_state
from _split_oracle import OracleSubdomain
gx, gy, tc, nsteps, overlap = (int(a) for a in sys.argv[2:7])
dist.init_process_group("gloo", init_method="env://")
rank, world = dist.get_rank(), dist.get_world_size()
Hg = make_params(gx, gy, testcase=tc)
u0 = init_state(Hg, tc)
boxes = decompose(gx, gy, world)
sub = OracleSubdomain(local_params(Hg, boxes[rank], rank, world), boxes[rank], rank,
                      scatter_state(u0, boxes[rank]))
run = SplitRun(Hg, [sub], DistComm(), overlap=bool(overlap))
run.run(nsteps)
assert not overlap or len(sub.parts) == 4 * nsteps
parts = [None] * world
dist.all_gather_object(parts, sub.download())
if rank == 0:
    g = np.zeros_like(u0)
    for r, ul in enumerate(parts):
        gather_into(g, ul, boxes[r])
    np.save(sys.argv[7], g)
    print(json.dumps({"t": run.t, "dts": run.dts}))
dist.destroy_process_group()
"""


@pytest.mark.parametrize("world,gx,gy,tc,overlap", [(2, 41, 27, 0, 0), (3, 50, 23, 2, 0),
                                                    (4, 36, 30, 1, 0), (2, 41, 27, 0, 1),
                                                    (4, 36, 30, 1, 1)])
def test_gloo_ranks_split_equals_single_grid(tmp_path, world, gx, gy, tc, overlap):
    out = str(tmp_path / "g.npy")
    outs = run_ranks(WORKER, world=world,
                     extra_args=(str(gx), str(gy), str(tc), "16", str(overlap), out))
    rec = json.loads(outs[0].strip().splitlines()[-1])
    Hg = make_params(gx, gy, testcase=tc)
    want, dts, t = single_run(Hg, init_state(Hg, tc), 16)
    got = np.load(out)
    m = outer_mask(Hg)
    assert np.array_equal(got[:, m], want[:, m])
    assert rec["dts"] == list(dts[:16]) and rec["t"] == t

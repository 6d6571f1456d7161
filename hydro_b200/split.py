"""Domain split: one grid over several subdomains (GPUs or ranks).

This is the reference's MPI build of the same variant, on the library's
sweeps:

* decomposition -- ``calc_sub_surface`` restates the simple (non k-d tree)
  ``CalcSubSurface`` of SplitSurface.c:102-185, which the default build uses
  (WITHKDTREE is not defined): a px x py process grid close to square, boxes
  of ceil(n / p) cells, ranks row-major from the lower left;
* boundaries -- a side that faces a neighbour gets boundary type 0
  (parametres.c:317-330), so make_boundary leaves its ghosts alone;
* halos -- before each sweep every subdomain sends the two interior lines next
  to each inner side of that sweep's direction and receives the neighbour's
  into its ghost cells (mpileftright / mpiupdown, mpibounds.c:165-310, called
  from make_boundary.c:48-52 and :125-129).  The library packs and unpacks the
  strips on the device (hydro_b200_domain_halo_pack / _unpack); the transport
  is torch.distributed point-to-point (NCCL between GPUs, gloo on the CPU) or,
  for subdomains in one process, a device copy;
* time step -- dt on even steps is the minimum over subdomains of
  courant_factor*dx / MAX(cournox, MAX(cournoy, smallc)) (compute_deltat.c:74,
  MPI_Allreduce MIN of main.c:361-372), halved at step 0; the sweep order
  alternates as in main.c:394-400.

Each cell's arithmetic is the single grid's, on the same inputs, so the split
result equals the single-grid run bit for bit.  With a periodic boundary
(type > 2) on a split axis each subdomain wraps onto itself, as the reference's
MPI build does; that is not the single grid's periodic problem.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

from .params import make_params, state_shape

# Box slots of parametres.h:19-28 / SplitSurface.h:4.
XMIN, XMAX, YMIN, YMAX, UP, DOWN, LEFT, RIGHT = range(8)


@dataclass
class Box:
    x0: int
    x1: int
    y0: int
    y1: int
    up: int
    down: int
    left: int
    right: int

    @property
    def nx(self) -> int:
        return self.x1 - self.x0

    @property
    def ny(self) -> int:
        return self.y1 - self.y0

    def neighbour(self, idim: int, side: int) -> int:
        """Rank across `side` (0 = left/down, 1 = right/up) of direction idim, or -1."""
        if idim == 1:
            return self.left if side == 0 else self.right
        return self.down if side == 0 else self.up


def process_grid(nproc: int) -> tuple:
    """(px, py) of SplitSurface.c:106-151; raises when nproc has no factor
    pair the reference accepts."""
    ny = int(math.sqrt(nproc))
    res = (nproc - ny * ny) // ny
    nx = ny + res
    if nx * ny != nproc:
        divider, last = 2, 1
        while divider < int(math.sqrt(nproc)):
            if nproc % divider == 0:
                last = divider
            divider += 1
        if last == 1:
            raise ValueError(f"{nproc} subdomains can't be divided evenly in x and y "
                             f"(closest {nx * ny})")
        ny = last
        res = (nproc - ny * ny) // ny
        nx = ny + res
    return nx, ny


def calc_sub_surface(globnx: int, globny: int, nproc: int, mype: int) -> Box:
    """Box and neighbours of rank `mype` (SplitSurface.c:102-185, called as
    CalcSubSurface(0, globnx, 0, globny, 0, nproc-1, ...), parametres.c:290)."""
    xmin, xmax, ymin, ymax = 0, globnx, 0, globny
    px, py = process_grid(nproc)
    pex, pey = mype % px, mype // px
    incx = (xmax - xmin + 1) // px
    incy = (ymax - ymin + 1) // py
    if incx * px + xmin < xmax:
        incx += 1
    if incy * py + ymin < ymax:
        incy += 1
    x0 = max(pex * incx + xmin, 0)
    x1 = min((pex + 1) * incx + xmin, xmax)
    y0 = max(pey * incy + ymin, 0)
    y1 = min((pey + 1) * incy + ymin, ymax)
    up = mype + px if mype + px < nproc else -1
    down = mype - px if mype - px >= 0 else -1
    left = mype - 1 if pex != 0 else -1
    right = mype + 1 if pex + 1 < px else -1
    return Box(x0, x1, y0, y1, up, down, left, right)


def decompose(globnx: int, globny: int, nproc: int) -> list:
    """Boxes of all ranks; raises (as parametres.c:301-312 aborts) when a box
    is empty."""
    boxes = [calc_sub_surface(globnx, globny, nproc, r) for r in range(nproc)]
    for r, b in enumerate(boxes):
        if b.nx <= 0 or b.ny <= 0:
            raise ValueError(f"decomposition of {globnx}x{globny} over {nproc} leaves rank {r} "
                             f"an empty box ({b.nx}x{b.ny})")
    return boxes


def local_params(Hg, box: Box, rank: int, nproc: int):
    """The subdomain's parameter record: its nx, ny, the global dx and
    constants, boundary type 0 on sides with a neighbour (parametres.c:317-330)."""
    bnd = (0 if box.left >= 0 else Hg.boundary_left, 0 if box.right >= 0 else Hg.boundary_right,
           0 if box.down >= 0 else Hg.boundary_down, 0 if box.up >= 0 else Hg.boundary_up)
    H = make_params(box.nx, box.ny, dx=Hg.dx, tend=Hg.tend, nstepmax=Hg.nstepmax,
                    courant_factor=Hg.courant_factor, niter_riemann=Hg.niter_riemann,
                    iorder=Hg.iorder, slope_type=Hg.slope_type, scheme=Hg.scheme, boundary=bnd,
                    testcase=Hg.testCase, gamma=Hg.gamma, smallr=Hg.smallr, smallc=Hg.smallc)
    H.nproc, H.mype = nproc, rank
    H.globnx, H.globny = Hg.nx, Hg.ny
    H.box[XMIN], H.box[XMAX], H.box[YMIN], H.box[YMAX] = box.x0, box.x1, box.y0, box.y1
    H.box[UP], H.box[DOWN], H.box[LEFT], H.box[RIGHT] = box.up, box.down, box.left, box.right
    return H


def scatter_state(u_global: np.ndarray, box: Box) -> np.ndarray:
    """The subdomain's padded block of a global padded state (its interior
    and the two ghost/halo lines around it)."""
    return np.ascontiguousarray(u_global[:, box.y0:box.y1 + 4, box.x0:box.x1 + 4])


def gather_into(u_global: np.ndarray, u_local: np.ndarray, box: Box) -> None:
    """Write a subdomain's interior, and its ghost lines on physical sides
    (not the corners), into the global padded state."""
    nx, ny = box.nx, box.ny
    u_global[:, box.y0 + 2:box.y1 + 2, box.x0 + 2:box.x1 + 2] = u_local[:, 2:ny + 2, 2:nx + 2]
    if box.left < 0:
        u_global[:, box.y0 + 2:box.y1 + 2, 0:2] = u_local[:, 2:ny + 2, 0:2]
    if box.right < 0:
        u_global[:, box.y0 + 2:box.y1 + 2, box.x1 + 2:box.x1 + 4] = u_local[:, 2:ny + 2,
                                                                            nx + 2:nx + 4]
    if box.down < 0:
        u_global[:, 0:2, box.x0 + 2:box.x1 + 2] = u_local[:, 0:2, 2:nx + 2]
    if box.up < 0:
        u_global[:, box.y1 + 2:box.y1 + 4, box.x0 + 2:box.x1 + 2] = u_local[:, ny + 2:ny + 4,
                                                                            2:nx + 2]


def compute_dt(courant_factor: float, dx: float, smallc: float, cx: float, cy: float) -> float:
    """compute_deltat.c:74 with utils.h's MAX (x > y ? x : y)."""
    m = cy if cy > smallc else smallc
    m = cx if cx > m else m
    return courant_factor * dx / m


# --------------------------------------------------------------------------
# Subdomain on the GPU


class GpuSubdomain:
    """A subdomain held by the library (hb_domain) with device halo buffers."""

    def __init__(self, H, box: Box, rank: int, device, precision: str = "fp64", kernels=None):
        import torch

        from .solver import Domain

        self.H, self.box, self.rank = H, box, rank
        self.device = torch.device(device)
        with torch.cuda.device(self.device):
            self.dom = Domain(H, precision=precision, kernels=kernels)
            self.comm_stream = None  # DistComm's transfer stream (created on first use)
            self.stream = torch.cuda.ExternalStream(self.dom.stream_ptr, device=self.device)
            self.send = {}
            self.recv = {}
            for idim in (1, 2):
                n = self.dom.halo_count(idim)
                for side in (0, 1):
                    if box.neighbour(idim, side) >= 0:
                        self.send[idim, side] = torch.empty(n, dtype=torch.float64,
                                                            device=self.device)
                        self.recv[idim, side] = torch.empty(n, dtype=torch.float64,
                                                            device=self.device)

    def upload(self, u_local: np.ndarray) -> None:
        self.dom.upload(u_local)

    def download(self) -> np.ndarray:
        return self.dom.download()

    def courant(self):
        return self.dom.courant()

    def sweep(self, stage: int, idim: int, dt: float, fuse: bool, part: int = 0) -> None:
        self.dom.sweep(stage, idim, dt, fuse, part)

    def pack(self, stage: int, idim: int, side: int) -> None:
        self.dom.halo_pack(stage, idim, side, self.send[idim, side].data_ptr())

    def unpack(self, idim: int, side: int) -> None:
        self.dom.halo_unpack(idim, side, self.recv[idim, side].data_ptr())

    def synchronize(self) -> None:
        self.dom.synchronize()

    def close(self) -> None:
        self.dom.close()


# --------------------------------------------------------------------------
# Transports


class DistComm:
    """torch.distributed: one subdomain per rank.  With NCCL the transfers
    run on the subdomain's stream, ordered after its pack kernels and before
    its unpack kernels without a host wait."""

    def __init__(self, group=None):
        import torch.distributed as dist

        self.dist = dist
        self.group = group

    def _ops(self, sub, idim: int) -> list:
        ops = []
        for side in (0, 1):
            nb = sub.box.neighbour(idim, side)
            if nb >= 0:
                ops.append(self.dist.P2POp(self.dist.isend, sub.send[idim, side], nb, self.group))
                ops.append(self.dist.P2POp(self.dist.irecv, sub.recv[idim, side], nb, self.group))
        return ops

    def exchange(self, subs: list, idim: int) -> None:
        self.exchange_finish(subs, self.exchange_start(subs, idim))

    def exchange_start(self, subs: list, idim: int):
        """Start the transfers of direction idim after the packs already
        issued on the subdomain's stream.  On a GPU they run on a stream of
        their own, so that work issued on the subdomain's stream afterwards
        (the sweep's ghost-free windows) overlaps them."""
        import torch

        (sub,) = subs
        ops = self._ops(sub, idim)
        if not ops:
            return None
        stream = getattr(sub, "stream", None)
        if stream is None:
            return self.dist.batch_isend_irecv(ops)
        if getattr(sub, "comm_stream", None) is None:
            sub.comm_stream = torch.cuda.Stream(device=sub.device)
        packed = torch.cuda.Event()
        packed.record(stream)
        with torch.cuda.stream(sub.comm_stream):
            sub.comm_stream.wait_event(packed)
            return self.dist.batch_isend_irecv(ops)

    def exchange_finish(self, subs: list, works) -> None:
        """Order the subdomain's stream after the transfers (no host wait on a
        GPU): work issued on it afterwards (the unpacks) sees the strips."""
        import torch

        if not works:
            return
        (sub,) = subs
        stream = getattr(sub, "stream", None)
        if stream is None:
            for w in works:
                w.wait()
            return
        with torch.cuda.stream(stream):
            for w in works:
                w.wait()

    def min(self, subs: list, x: float) -> float:
        import torch

        (sub,) = subs
        stream = getattr(sub, "stream", None)
        if stream is None:
            t = torch.tensor([x], dtype=torch.float64)
            self.dist.all_reduce(t, op=self.dist.ReduceOp.MIN, group=self.group)
            return float(t.item())
        # Upload, reduce and read back on the subdomain's stream.
        with torch.cuda.stream(stream):
            t = torch.tensor([x], dtype=torch.float64, device=sub.device)
            self.dist.all_reduce(t, op=self.dist.ReduceOp.MIN, group=self.group)
            return float(t.item())


class LocalComm:
    """All subdomains in this process: strips move by a copy once every
    subdomain's pack has completed."""

    def exchange(self, subs: list, idim: int) -> None:
        by_rank = {s.rank: s for s in subs}
        for s in subs:
            s.synchronize()
        for s in subs:
            for side in (0, 1):
                nb = s.box.neighbour(idim, side)
                if nb >= 0:
                    s.recv[idim, side].copy_(by_rank[nb].send[idim, 1 - side])
        _sync_torch(subs)

    def exchange_start(self, subs: list, idim: int):
        return idim

    def exchange_finish(self, subs: list, idim) -> None:
        self.exchange(subs, idim)

    def min(self, subs: list, x: float) -> float:
        return x


def _sync_torch(subs) -> None:
    import torch

    for s in subs:
        dev = getattr(s, "device", None)
        if dev is not None and dev.type == "cuda":
            torch.cuda.synchronize(dev)


# --------------------------------------------------------------------------
# Driver


class SplitRun:
    """main.c:344-408 over subdomains.  `subs` are the subdomains this
    process owns (one per rank with DistComm; all of them with LocalComm).

    With ``overlap`` each sweep is issued in two parts around its halo
    exchange: pack the strips, start the transfers, sweep the windows that
    read no ghost cell (hydro_b200_domain_sweep_part, part 1) while the strips
    travel, then finish the transfers, unpack, and sweep the windows next to
    the ghosts (part 2).  The results are the same bits as without it."""

    def __init__(self, Hg, subs: list, comm, overlap: bool = False):
        self.Hg = Hg
        self.subs = subs
        self.comm = comm
        self.overlap = overlap
        self.t = 0.0
        self.nstep = 0
        self.dt = 0.0
        self.dts = []

    def _exchange(self, stage: int, idim: int) -> None:
        for s in self.subs:
            for side in (0, 1):
                if s.box.neighbour(idim, side) >= 0:
                    s.pack(stage, idim, side)
        self.comm.exchange(self.subs, idim)
        for s in self.subs:
            for side in (0, 1):
                if s.box.neighbour(idim, side) >= 0:
                    s.unpack(idim, side)

    def _sweep_stage(self, stage: int, idim: int, fuse: bool) -> None:
        if not self.overlap:
            self._exchange(stage, idim)
            for s in self.subs:
                s.sweep(stage, idim, self.dt, fuse)
            return
        for s in self.subs:
            for side in (0, 1):
                if s.box.neighbour(idim, side) >= 0:
                    s.pack(stage, idim, side)
        pending = self.comm.exchange_start(self.subs, idim)
        for s in self.subs:
            s.sweep(stage, idim, self.dt, fuse, 1)
        self.comm.exchange_finish(self.subs, pending)
        for s in self.subs:
            for side in (0, 1):
                if s.box.neighbour(idim, side) >= 0:
                    s.unpack(idim, side)
        for s in self.subs:
            s.sweep(stage, idim, self.dt, fuse, 2)

    def step(self) -> float:
        Hg = self.Hg
        if self.nstep % 2 == 0:
            dt = math.inf
            for s in self.subs:
                cx, cy = s.courant()
                d = compute_dt(Hg.courant_factor, Hg.dx, Hg.smallc, cx, cy)
                dt = d if d < dt else dt
            dt = self.comm.min(self.subs, dt)
            if self.nstep == 0:
                dt = dt / 2.0
            self.dt = dt
        first = 1 if self.nstep % 2 == 0 else 2
        second = 3 - first
        # The Courant maxima of the state after an odd step feed the next dt.
        fuse = self.nstep % 2 == 1
        self._sweep_stage(0, first, False)
        self._sweep_stage(1, second, fuse)
        self.dts.append(self.dt)
        self.nstep += 1
        self.t += self.dt
        return self.dt

    def run(self, nstepmax: int, tend: float = 1e300) -> int:
        n0 = self.nstep
        while self.t < tend and self.nstep < nstepmax:
            self.step()
        return self.nstep - n0


def split_gpu_local(Hg, u_global: np.ndarray, nparts: int, devices=None,
                    precision: str = "fp64", overlap: bool = False, kernels=None):
    """All subdomains of an `nparts` split in this process, subdomain r on
    devices[r % len(devices)] (default: cuda:0).  Returns the SplitRun."""
    boxes = decompose(Hg.nx, Hg.ny, nparts)
    devices = devices or ["cuda:0"]
    subs = []
    for r, b in enumerate(boxes):
        H = local_params(Hg, b, r, nparts)
        s = GpuSubdomain(H, b, r, devices[r % len(devices)], precision, kernels)
        s.upload(scatter_state(u_global, b))
        subs.append(s)
    return SplitRun(Hg, subs, LocalComm(), overlap=overlap)


def gather_global(Hg, subs: list, out: np.ndarray | None = None) -> np.ndarray:
    """The global state assembled from subdomains held in this process."""
    u = np.zeros(state_shape(Hg), dtype=np.float64) if out is None else out
    for s in subs:
        gather_into(u, s.download(), s.box)
    return u

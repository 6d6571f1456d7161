"""A subdomain computed by the oracle (the CPU restatement), with the same
halo-strip layout as the library's pack/unpack kernels.  Used to check the
split driver's protocol (decomposition, halo exchange, dt reduction) on the
CPU, where the library's sweeps cannot run."""
import numpy as np
import torch

from oracle import oracle as O


def orc_param_of(H):
    return O.make_param(H.nx, H.ny, dx=H.dx,
                        boundary=(H.boundary_left, H.boundary_right, H.boundary_down,
                                  H.boundary_up),
                        iorder=H.iorder, scheme=H.scheme, niter_riemann=H.niter_riemann,
                        slope_type=H.slope_type, gamma=H.gamma, smallr=H.smallr,
                        smallc=H.smallc, courant_factor=H.courant_factor)


def strip_index(u_shape, idim, side, ghost):
    """(rows, cols) index arrays of a strip in the [var][line][2] (idim 1) or
    [var][2][line] (idim 2) order of the library's halo kernel."""
    _, nyt, nxt = u_shape
    nx, ny = nxt - 4, nyt - 4
    nl = nx if idim == 1 else ny
    ks = [side * (nl + 2) + c for c in (0, 1)] if ghost else [2 + c if side == 0 else nl + c
                                                              for c in (0, 1)]
    if idim == 1:
        rows = np.arange(2, ny + 2)[:, None].repeat(2, 1)
        cols = np.array(ks)[None, :].repeat(ny, 0)
    else:
        rows = np.array(ks)[:, None].repeat(nx, 1)
        cols = np.arange(2, nx + 2)[None, :].repeat(2, 0)
    return rows, cols


class OracleSubdomain:
    def __init__(self, H, box, rank, u_local):
        self.H, self.box, self.rank = H, box, rank
        self.p = orc_param_of(H)
        self.u = np.ascontiguousarray(u_local, dtype=np.float64).copy()
        self.send, self.recv = {}, {}
        self.parts = []
        for idim in (1, 2):
            n = 8 * (H.ny if idim == 1 else H.nx)
            for side in (0, 1):
                if box.neighbour(idim, side) >= 0:
                    self.send[idim, side] = torch.zeros(n, dtype=torch.float64)
                    self.recv[idim, side] = torch.zeros(n, dtype=torch.float64)

    def courant(self):
        _, cx, cy = O.courant(self.p, self.u)
        return cx, cy

    def sweep(self, stage, idim, dt, fuse, part=0):
        """part 0: the sweep.  The oracle sweeps whole lines, so the two parts
        of an overlapped sweep are: part 1, which must run before the unpack,
        records its place; part 2, after the unpack, sweeps."""
        if part == 1:
            self.parts.append((idim, "ghost-free"))
            return
        if part == 2:
            assert self.parts and self.parts[-1] == (idim, "ghost-free")
            self.parts.append((idim, "edges"))
        O.sweep(self.p, idim, dt, self.u)

    def pack(self, stage, idim, side):
        r, c = strip_index(self.u.shape, idim, side, ghost=False)
        self.send[idim, side].copy_(torch.from_numpy(self.u[:, r, c].reshape(-1).copy()))

    def unpack(self, idim, side):
        r, c = strip_index(self.u.shape, idim, side, ghost=True)
        self.u[:, r, c] = self.recv[idim, side].numpy().reshape((4,) + r.shape)

    def synchronize(self):
        pass

    def download(self):
        return self.u.copy()

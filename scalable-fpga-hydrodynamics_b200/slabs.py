"""The reference's X-slab decomposition over ranks (hydro2d/main.cxx:621-636, --sdx N
--sdy 1; hydro3d likewise), one process per GPU.

Rank r of N owns a contiguous range of global X rows (2D) or planes (3D). Every step:
  1. each rank sends its first interior row to the rank on its left and its last to the
     rank on its right, which store them in their ghost rows NB_X+1 and 0 (periodic across
     ranks: rank 0's left neighbour is rank N-1), as the reference's host exchange does
     (hydro2d/main.cxx:381-424);
  2. each rank steps its slab with the X ghost rows read from memory (X_GHOSTS_FROM_MEMORY);
  3. the next Dt is the MIN of the ranks' Dt (main.cxx:781) and t advances by it.
The update of a cell depends only on its neighbours, so the state after n steps is
bit-identical to the whole domain stepped on one device. The exchange is the only
collective on the data path: two rows per rank per step, plus one scalar MIN.
"""
from __future__ import annotations

import numpy as np

from . import (KERNEL_AUTO, HydroError, Physics, _torch, alloc_state, init_blast_at, mass, step)
from .batch import Blast
from .replicas import Replicas


def slab_rows(nb_x: int, world: int, rank: int):
    """Global interior rows (1-based, inclusive) of `rank`: an even split, the first
    nb_x % world ranks one row longer."""
    if nb_x < world:
        raise HydroError(-1, f"{nb_x} rows cannot be split over {world} ranks")
    base, extra = divmod(nb_x, world)
    lo = 1 + rank * base + min(rank, extra)
    return lo, lo + base + (1 if rank < extra else 0) - 1


class XSlabRun:
    """One rank's slab of the reference blast (2D or 3D), stepped in lock step with the
    other ranks of `reps` (Replicas: torch.distributed over NCCL on GPUs, or gloo, which
    stages the exchanged rows through host memory)."""

    def __init__(self, nb, dtype, reps: Replicas, kernel=KERNEL_AUTO, stream=None):
        torch = _torch()
        self.torch, self.reps = torch, reps
        self.nb = tuple(int(n) for n in nb)
        self.T = dtype
        self.kernel, self.stream = kernel, stream
        self.lo, self.hi = slab_rows(self.nb[0], reps.world, reps.rank)
        self.nb_local = (self.hi - self.lo + 1,) + self.nb[1:]
        # constants of the whole domain (DX, C_min), not of the slab
        self.phys = Physics(dtype, self.nb)
        self.phys_local = Physics(dtype, self.nb_local)
        for f in ("D", "min_spacing", "Cc", "C_min"):
            setattr(self.phys_local, f, getattr(self.phys, f))
        self.cur = alloc_state(self.nb_local, dtype)
        self.nxt = alloc_state(self.nb_local, dtype)
        tdt = torch.float64 if dtype is np.float64 else torch.float32
        self.dt_dev = torch.zeros(1, dtype=tdt, device="cuda")
        # the reference blast of the whole domain, seen from this slab's rows
        g = Blast(nb=self.nb, rho_in=1.0, rho_out=1.2, p_in=10.0, p_out=0.1)
        local = Blast(nb=self.nb_local, centre=(g.centre[0] - (self.lo - 1),) + tuple(g.centre[1:]), radius=g.radius,
                      rho_in=1.0, rho_out=1.2, p_in=10.0, p_out=0.1)
        first = init_blast_at(self.cur, self.phys_local, local, stream=stream)
        first = self._min(first)
        big = dtype(1e20)
        self.dt = first if first < big else big
        self.t, self.it = 0.0, 0
        self.row = int(np.prod([n + 2 for n in self.nb[1:]]))  # cells per X row (plane)

    # -- collectives ----------------------------------------------------------------
    def _min(self, x):
        if self.reps.world == 1:
            return x
        torch = self.torch
        dev = "cuda" if self.reps.backend == "nccl" else "cpu"
        t = torch.tensor([float(x)], dtype=torch.float64 if self.T is np.float64 else torch.float32, device=dev)
        self.reps.dist.all_reduce(t, op=self.reps.dist.ReduceOp.MIN)
        return self.T(t.item())

    def _rows(self, a, i):
        """View of X row (plane) i of one state array (both components of the cell)."""
        nv = a.numel() // ((self.nb_local[0] + 2) * self.row)
        return a[i * self.row * nv:(i + 1) * self.row * nv]

    def exchange(self):
        """Fill the ghost rows 0 and NB_X_local+1 of the current state from the
        neighbouring ranks' edge rows (periodic across ranks)."""
        n = self.nb_local[0]
        if self.reps.world == 1:
            for a in self.cur:
                self._rows(a, 0).copy_(self._rows(a, n))
                self._rows(a, n + 1).copy_(self._rows(a, 1))
            return
        dist, torch = self.reps.dist, self.torch
        left = (self.reps.rank - 1) % self.reps.world
        right = (self.reps.rank + 1) % self.reps.world
        staged = self.reps.backend != "nccl"
        for a in self.cur:
            first, last = self._rows(a, 1), self._rows(a, n)
            send_l = first.cpu() if staged else first.contiguous()
            send_r = last.cpu() if staged else last.contiguous()
            recv_lo = torch.empty_like(send_l)
            recv_hi = torch.empty_like(send_r)
            # the rightward message (last row -> right neighbour's ghost row 0) first, then the
            # leftward one: with two ranks both neighbours are the same peer and messages
            # between a pair of ranks match in issue order (NCCL has no tags)
            ops = [dist.P2POp(dist.isend, send_r, right, tag=1), dist.P2POp(dist.isend, send_l, left, tag=2),
                   dist.P2POp(dist.irecv, recv_lo, left, tag=1), dist.P2POp(dist.irecv, recv_hi, right, tag=2)]
            for r in dist.batch_isend_irecv(ops):
                r.wait()
            self._rows(a, 0).copy_(recv_lo)       # left neighbour's last row
            self._rows(a, n + 1).copy_(recv_hi)   # right neighbour's first row

    def step(self):
        self.exchange()
        dtd = self.phys.dtd(self.dt)
        step(self.cur, self.nxt, self.dt_dev, self.phys_local, dtd, kernel=self.kernel, sync=True,
             stream=self.stream, x_ghosts=True)
        self.cur, self.nxt = self.nxt, self.cur
        dtn = self._min(self.T(self.dt_dev.item()))
        big = self.T(1e20)
        self.dt = dtn if dtn < big else big
        self.it += 1
        self.t += float(self.dt)

    def run(self, max_t: float, max_it: int):
        while self.t < max_t and self.it < max_it:
            self.step()
        return self

    def mass(self) -> float:
        """Total density of the whole domain (sum over ranks of each slab's compensated sum)."""
        m = mass(self.cur[0], self.nb_local, self.stream)
        return self.reps.sum_over_ranks(m) if self.reps.world > 1 else m

    def interior(self):
        """This slab's interior as host arrays (rhoE, uvx), shaped (rows, ..., comps)."""
        shape = tuple(n + 2 for n in self.nb_local)
        inner = tuple(slice(1, n + 1) for n in self.nb_local)
        out = []
        for a, nv in zip(self.cur, (2, len(self.nb))):
            out.append(a.cpu().numpy().reshape(shape + (nv,))[inner])
        return out

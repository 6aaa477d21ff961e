"""The reference's X-slab decomposition over ranks (hydro2d/main.cxx:621-636, --sdx N
--sdy 1; hydro3d likewise), one process per GPU.

Rank r of N owns a contiguous range of global X rows (2D) or planes (3D). The update of a
cell depends only on its neighbours, so the state after n steps is bit-identical to the
whole domain stepped on one device. The exchange is the only collective on the data path:
two rows per rank per step, plus one scalar MIN of Dt (main.cxx:781).

Each step overlaps the exchange with the bulk of the update:
  1. the two edge rows (1 and n) of the slab are updated first; they read the ghost rows 0
     and n+1 that the previous step's exchange filled;
  2. the new edge rows are sent to the neighbouring ranks (rank 0's left neighbour is rank
     N-1), which receive them into the ghost rows of their new state, as the reference's
     host exchange does (hydro2d/main.cxx:381-424), while
  3. the interior rows 2 .. n-1 are updated (they read rows 1 .. n only);
  4. the exchange is completed, the three partial Dt are combined (the minimum of
     C_min / max over parts is C_min / the max over the slab: division by a positive
     maximum is monotone) and the MIN over ranks is taken on the device; one scalar comes
     back to the host for the next step's DtDx, as in the reference's loop.
Every update of a part of the slab is one step call on a view of the state whose first row
is the part's lower X neighbour, with the X neighbours read from memory.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import (KERNEL_AUTO, HydroError, Physics, StepInfo, _check, alloc_state, init_blast_at, lib, mass, step)
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


def _gpu_stepper(stream, kernel, arith):
    """Step function of the GPU library: (state_in, state_out, dt_out, phys, dtd, sync)."""

    def run(cur, nxt, dt_out, phys, dtd, sync):
        _, info = step(cur, nxt, dt_out, phys, dtd, kernel=kernel, sync=sync, stream=stream, x_ghosts=True,
                       arith=arith)
        return info

    return run


class XSlabRun:
    """One rank's slab of the reference blast (2D or 3D), stepped in lock step with the
    other ranks of `reps` (Replicas: torch.distributed over NCCL on GPUs, or gloo, which
    stages the exchanged rows through host memory).

    `stepper` and `state` replace the GPU library for a run on the host (the schedule and
    the exchange are the same): stepper(state_in, state_out, dt_out, phys, dtd, sync) steps
    the rows of views whose first and last rows are X ghosts, and `state` gives the slab's
    initial (rhoE, uvx) arrays (torch tensors with ghost rows) and first Dt."""

    def __init__(self, nb, dtype, reps: Replicas, kernel=KERNEL_AUTO, stream=None, arith=None, overlap=True,
                 stepper=None, state=None):
        import torch

        self.torch, self.reps = torch, reps
        self.nb = tuple(int(n) for n in nb)
        self.T = dtype
        self.overlap = overlap
        self.lo, self.hi = slab_rows(self.nb[0], reps.world, reps.rank)
        self.nb_local = (self.hi - self.lo + 1,) + self.nb[1:]
        self.nv = len(self.nb)
        self.row = int(np.prod([n + 2 for n in self.nb[1:]]))  # cells per X row (plane)
        # constants of the whole domain (DX, C_min), not of the slab
        self.phys = Physics(dtype, self.nb)
        self.stream = stream
        self.stepper = stepper or _gpu_stepper(stream, kernel, arith)
        tdt = torch.float64 if dtype is np.float64 else torch.float32
        if state is None:
            self.device = "cuda"
            self.cur = alloc_state(self.nb_local, dtype)
            self.nxt = alloc_state(self.nb_local, dtype)
            # the reference blast of the whole domain, seen from this slab's rows
            g = Blast(nb=self.nb, rho_in=1.0, rho_out=1.2, p_in=10.0, p_out=0.1)
            local = Blast(nb=self.nb_local, centre=(g.centre[0] - (self.lo - 1),) + tuple(g.centre[1:]),
                          radius=g.radius, rho_in=1.0, rho_out=1.2, p_in=10.0, p_out=0.1)
            first = init_blast_at(self.cur, self._phys_rows(self.nb_local[0]), local, stream=stream)
        else:
            (self.cur, first) = state
            self.device = self.cur[0].device.type
            self.nxt = tuple(torch.zeros_like(a) for a in self.cur)
        # one Dt scalar per updated part (edges, interior) and their minimum
        self.dt_parts = torch.zeros(3, dtype=tdt, device=self.device)
        self.dt_min = torch.zeros(1, dtype=tdt, device=self.device)
        first = self._min_host(first)
        big = dtype(1e20)
        self.dt = first if first < big else big
        self.t, self.it = 0.0, 0
        self.infos = []
        self._exchange_blocking(self.cur)

    # -- views and parts ----------------------------------------------------------------
    def _phys_rows(self, nrows):
        p = Physics(self.T, (nrows,) + self.nb[1:])
        for f in ("D", "min_spacing", "Cc", "C_min"):
            setattr(p, f, getattr(self.phys, f))
        return p

    def _rows(self, a, i, j=None):
        """View of X rows i .. j-1 (default: row i) of one state array."""
        nv = a.numel() // ((self.nb_local[0] + 2) * self.row)
        j = i + 1 if j is None else j
        return a[i * self.row * nv:j * self.row * nv]

    def _part(self, state, first, nrows):
        """The state seen from row `first`: a view of rows first .. first+nrows+1, where the
        step updates rows first+1 .. first+nrows from their neighbours."""
        return tuple(self._rows(a, first, first + nrows + 2) for a in state)

    def _update(self, first, nrows, k, sync):
        phys = self._phys_rows(nrows)
        info = self.stepper(self._part(self.cur, first, nrows), self._part(self.nxt, first, nrows),
                            self.dt_parts[k:k + 1], phys, self.phys.dtd(self.dt), sync)
        return info

    # -- collectives ----------------------------------------------------------------------
    def _min_host(self, x):
        if self.reps.world == 1:
            return x
        torch = self.torch
        t = torch.tensor([float(x)], dtype=torch.float64 if self.T is np.float64 else torch.float32,
                         device=self.reps.device)
        self.reps.dist.all_reduce(t, op=self.reps.dist.ReduceOp.MIN)
        return self.T(t.item())

    def _start_exchange(self, state):
        """Start sending `state`'s edge rows to the neighbours and receiving theirs into
        the ghost rows; returns the pending works and the copies that finish it."""
        n = self.nb_local[0]
        if self.reps.world == 1:
            for a in state:
                self._rows(a, 0).copy_(self._rows(a, n))
                self._rows(a, n + 1).copy_(self._rows(a, 1))
            return [], []
        dist, torch = self.reps.dist, self.torch
        left = (self.reps.rank - 1) % self.reps.world
        right = (self.reps.rank + 1) % self.reps.world
        staged = self.reps.backend != "nccl" and state[0].device.type == "cuda"
        ops, finish = [], []
        for a in state:
            first, last = self._rows(a, 1), self._rows(a, n)
            send_l = first.cpu() if staged else first.contiguous()
            send_r = last.cpu() if staged else last.contiguous()
            recv_lo = torch.empty_like(send_l)
            recv_hi = torch.empty_like(send_r)
            # the rightward message (last row -> right neighbour's ghost row 0) first, then the
            # leftward one: with two ranks both neighbours are the same peer and messages
            # between a pair of ranks match in issue order (NCCL has no tags)
            ops += [dist.P2POp(dist.isend, send_r, right, tag=1), dist.P2POp(dist.isend, send_l, left, tag=2),
                    dist.P2POp(dist.irecv, recv_lo, left, tag=1), dist.P2POp(dist.irecv, recv_hi, right, tag=2)]
            finish.append((self._rows(a, 0), recv_lo))       # left neighbour's last row
            finish.append((self._rows(a, n + 1), recv_hi))   # right neighbour's first row
        return dist.batch_isend_irecv(ops), finish

    @staticmethod
    def _finish_exchange(works, finish):
        for w in works:
            w.wait()
        for dst, src in finish:
            dst.copy_(src)

    def _exchange_blocking(self, state):
        self._finish_exchange(*self._start_exchange(state))

    def exchange(self):
        """Fill the ghost rows 0 and NB_X_local+1 of the current state from the
        neighbouring ranks' edge rows (periodic across ranks)."""
        self._exchange_blocking(self.cur)

    # -- the step -------------------------------------------------------------------------
    def step(self):
        n = self.nb_local[0]
        self.dt_parts.fill_(float("inf"))
        self.infos = []
        if not self.overlap or n <= 2:
            # the whole slab in one update, then the exchange for the next step
            self.infos.append(self._update(0, n, 0, True))
            self._exchange_blocking(self.nxt)
        else:
            # edge rows first, their exchange in flight while the interior is updated
            self.infos.append(self._update(0, 1, 0, True))
            self.infos.append(self._update(n - 1, 1, 1, True))
            pending = self._start_exchange(self.nxt)
            self.infos.append(self._update(1, n - 2, 2, False))
            self._finish_exchange(*pending)
        torch = self.torch
        torch.amin(self.dt_parts, dim=0, keepdim=True, out=self.dt_min)
        if self.reps.world > 1:
            dt = self.dt_min
            if self.reps.backend != "nccl" and dt.device.type == "cuda":
                dt = dt.cpu()
            self.reps.dist.all_reduce(dt, op=self.reps.dist.ReduceOp.MIN)
            dtn = self.T(dt.item())
        else:
            dtn = self.T(self.dt_min.item())
        if self.overlap and n > 2 and self.device == "cuda":
            # the interior update was enqueued without waiting: its status, now complete
            info = StepInfo()
            _check(lib().hydro_last_step_info(ctypes.byref(info)))
            self.infos[-1] = info
        self.cur, self.nxt = self.nxt, self.cur
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

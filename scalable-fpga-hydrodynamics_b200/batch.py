"""Batched step over many blast instances (C ABI `hydro_batch_*`).

One persistent kernel per step advances every admitted instance with its own Dt, FP64
simulated time and end condition; `run(n)` replays n steps as one CUDA graph.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from . import HydroError, _check, _torch, last_error, lib

_c = ctypes


class BlastSpec(_c.Structure):
    """hydro_blast_t"""

    _fields_ = [("nb", _c.c_size_t * 3), ("centre", _c.c_double * 3), ("radius", _c.c_double),
                ("rho_in", _c.c_double), ("rho_out", _c.c_double), ("p_in", _c.c_double), ("p_out", _c.c_double),
                ("gamma", _c.c_double), ("K", _c.c_double), ("C", _c.c_double), ("t_end", _c.c_double),
                ("max_steps", _c.c_longlong)]


class BatchStatus(_c.Structure):
    """hydro_batch_status_t"""

    _fields_ = [("t", _c.c_double), ("dt", _c.c_double), ("mass", _c.c_double), ("mom", _c.c_double * 3),
                ("energy", _c.c_double), ("max_speed", _c.c_double), ("steps", _c.c_longlong),
                ("active", _c.c_int), ("err", _c.c_uint), ("exact_passes", _c.c_longlong)]


@dataclass
class Blast:
    """A blast problem in the reference's cell-index coordinates (interior cells 1..NB)."""

    nb: tuple
    centre: tuple = None
    radius: float = None
    rho_in: float = 1.0
    rho_out: float = 1.2
    p_in: float = 10.0
    p_out: float = 0.1
    gamma: float = 1.4
    K: float = 1.1
    C: float = None
    t_end: float = float("inf")
    max_steps: int = 2 ** 62

    def __post_init__(self):
        self.nb = tuple(int(n) for n in self.nb)
        c = tuple((n + 1) / 2.0 for n in self.nb)
        if self.centre is None:
            self.centre = c  # the reference's circle (hydro2d/main.cxx:290-292)
        if self.radius is None:
            self.radius = min(c) / 3
        if self.C is None:
            self.C = 0.4 if len(self.nb) == 3 else 0.5

    def spec(self) -> BlastSpec:
        s = BlastSpec()
        for i, n in enumerate(self.nb):
            s.nb[i] = n
            s.centre[i] = self.centre[i]
        s.radius, s.rho_in, s.rho_out, s.p_in, s.p_out = self.radius, self.rho_in, self.rho_out, self.p_in, self.p_out
        s.gamma, s.K, s.C, s.t_end = self.gamma, self.K, self.C, self.t_end
        s.max_steps = int(min(self.max_steps, 2 ** 62))
        return s


def _declare(L):
    if getattr(L, "_batch_declared", False):
        return L
    vp = _c.c_void_p
    L.hydro_batch_create.argtypes = [_c.c_int, _c.c_int, _c.c_int, _c.c_int, vp]
    L.hydro_batch_create.restype = vp
    L.hydro_batch_add.argtypes = [vp, _c.POINTER(BlastSpec)]
    L.hydro_batch_add.restype = _c.c_int
    L.hydro_batch_bytes.argtypes = [vp, _c.POINTER(BlastSpec)]
    L.hydro_batch_bytes.restype = _c.c_longlong
    L.hydro_batch_remove.argtypes = [vp, _c.c_int]
    L.hydro_batch_remove.restype = _c.c_int
    L.hydro_batch_run.argtypes = [vp, _c.c_int, _c.c_int]
    L.hydro_batch_run.restype = _c.c_int
    L.hydro_batch_status.argtypes = [vp, _c.c_int, _c.POINTER(BatchStatus)]
    L.hydro_batch_status.restype = _c.c_int
    L.hydro_batch_copy_state.argtypes = [vp, _c.c_int, vp, vp, _c.c_int]
    L.hydro_batch_copy_state.restype = _c.c_int
    L.hydro_batch_destroy.argtypes = [vp]
    L.hydro_batch_destroy.restype = None
    L.hydro_batch_sync.argtypes = [vp]
    L.hydro_batch_sync.restype = _c.c_int
    L.hydro_batch_prepare.argtypes = [vp, _c.c_int]
    L.hydro_batch_prepare.restype = _c.c_int
    L.hydro_batch_set_skip_fraction.argtypes = [vp, _c.c_double]
    L.hydro_batch_set_skip_fraction.restype = _c.c_int
    L.hydro_batch_set_arith.argtypes = [vp, _c.c_int]
    L.hydro_batch_set_arith.restype = _c.c_int
    L._batch_declared = True
    return L


class Batch:
    """A set of blast instances advanced together (2D; FP32 or FP64)."""

    def __init__(self, dim: int = 2, dtype=np.float32, chunk: int = 0, capacity: int = 1024, stream=None,
                 arith=None):
        """arith: "strict", "fused" or None (the library default)."""
        torch = _torch()
        self.L = _declare(lib())
        self.dim, self.T = dim, dtype
        self.stream = stream
        h = stream.cuda_stream if stream is not None else None
        self.h = self.L.hydro_batch_create(dim, np.dtype(dtype).itemsize, chunk, capacity, h)
        if not self.h:
            raise HydroError(*last_error())
        self.blasts = {}
        if arith is not None:
            from . import _ARITH_BITS

            _check(self.L.hydro_batch_set_arith(self.h, _ARITH_BITS[arith]))

    def close(self):
        if self.h:
            self.L.hydro_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def bytes(self, blast: Blast) -> int:
        return int(self.L.hydro_batch_bytes(self.h, _c.byref(blast.spec())))

    def add(self, blast: Blast) -> int:
        slot = self.L.hydro_batch_add(self.h, _c.byref(blast.spec()))
        if slot < 0:
            raise HydroError(slot, last_error()[1])
        self.blasts[slot] = blast
        return slot

    def remove(self, slot: int):
        _check(self.L.hydro_batch_remove(self.h, slot))
        self.blasts.pop(slot, None)

    def run(self, nsteps: int, sync: bool = True):
        _check(self.L.hydro_batch_run(self.h, nsteps, 1 if sync else 0))

    def sync(self):
        _check(self.L.hydro_batch_sync(self.h))

    def prepare(self, nsteps: int):
        """Build the graph of `nsteps` steps now (the next run(nsteps) only launches)."""
        _check(self.L.hydro_batch_prepare(self.h, nsteps))

    def set_skip_fraction(self, frac: float):
        """Signal-speed skip threshold as a fraction of the previous step's max (default
        0.9; 0: every cell exact; above 1: every step takes the exact pass)."""
        _check(self.L.hydro_batch_set_skip_fraction(self.h, float(frac)))

    def status(self, slot: int) -> dict:
        s = BatchStatus()
        _check(self.L.hydro_batch_status(self.h, slot, _c.byref(s)))
        return dict(t=s.t, dt=s.dt, mass=s.mass, mom=tuple(s.mom), energy=s.energy, max_speed=s.max_speed,
                    steps=s.steps, active=bool(s.active), err=s.err, exact_passes=s.exact_passes)

    def state(self, slot: int):
        """(rhoE, uvx) numpy arrays in the reference layout."""
        b = self.blasts[slot]
        ncell = int(np.prod([n + 2 for n in b.nb]))
        rhoE = np.zeros(2 * ncell, self.T)
        uvx = np.zeros((3 if self.dim == 3 else 2) * ncell, self.T)
        _check(self.L.hydro_batch_copy_state(self.h, slot, rhoE.ctypes.data_as(_c.c_void_p),
                                             uvx.ctypes.data_as(_c.c_void_p), 1))
        return rhoE, uvx

"""The allocation-free 2D FP64 step (hydro2d_step_f64_noalloc), through the C ABI.

It exists for callers that cannot allocate: programs whose GPU memory is owned by their own
pool or caching allocator, stepping loops that must not run cudaMalloc/cudaFree (which can
synchronise the whole device), and programs built to allocate nothing after start-up. Its
scratch is a fixed array inside the library instead of memory allocated on first use.

Checked here: two calls in a row, each against the regular entry point (hydro2d_step_f64)
on the same inputs, bit for bit (the tolerance of every FP64 test in this suite); the
Dt_next and the step results (mass, max speed) agree; a grid beyond the fixed scratch is
rejected. The file is named to be collected last, and passes alone in a fresh process too.
"""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

from conftest import load_pkg

hb = load_pkg()
pytestmark = pytest.mark.gpu


def _declare(L):
    d = ctypes.c_double
    fn = L.hydro2d_step_f64_noalloc
    fn.argtypes = [ctypes.c_void_p] * 5 + [d] * 5 + [ctypes.c_size_t] * 2 + [d] * 2 + [
        ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(hb.StepInfo)]
    fn.restype = ctypes.c_int
    return fn


def _state(cuda, nb, seed):
    rng = np.random.default_rng(seed)
    ncell = (nb[0] + 2) * (nb[1] + 2)
    rho = rng.uniform(0.5, 2.0, ncell)
    vel = rng.uniform(-0.5, 0.5, (ncell, 2))
    p = rng.uniform(0.05, 10.0, ncell)
    E = p / 0.4 + 0.5 * rho * (vel ** 2).sum(1)
    rhoE = np.stack([rho, E], 1).reshape(-1)
    uv = (vel * rho[:, None]).reshape(-1)
    return cuda.from_numpy(rhoE).cuda(), cuda.from_numpy(uv).cuda()


@pytest.mark.parametrize("nb", [(60, 60), (257, 301), (33, 7)])
def test_noalloc_step_matches_regular_step_twice(cuda, nb):
    L = hb.lib()
    noalloc = _declare(L)
    phys = hb.Physics(np.float64, nb)
    stream = hb._stream_handle()
    cur_a = _state(cuda, nb, 11)
    cur_b = tuple(a.clone() for a in cur_a)
    dt_a = cuda.zeros(1, dtype=cuda.float64, device="cuda")
    dt_b = cuda.zeros(1, dtype=cuda.float64, device="cuda")
    dt = np.float64(0.05) * phys.min_spacing / np.float64(6)
    for call in range(2):
        dtd = phys.dtd(dt)
        nxt_a = tuple(cuda.zeros_like(a) for a in cur_a)
        nxt_b = tuple(cuda.zeros_like(a) for a in cur_b)
        ia, ib = hb.StepInfo(), hb.StepInfo()
        rc = L.hydro2d_step_f64(hb._ptr(cur_a[0]), hb._ptr(cur_a[1]), hb._ptr(nxt_a[0]), hb._ptr(nxt_a[1]),
                                hb._ptr(dt_a), phys.C_min, phys.g, phys.gm1, phys.divgamma, phys.k, nb[0], nb[1],
                                dtd[0], dtd[1], stream, 0, 1, ctypes.byref(ia))
        assert rc == 0, hb.last_error()
        rc = noalloc(hb._ptr(cur_b[0]), hb._ptr(cur_b[1]), hb._ptr(nxt_b[0]), hb._ptr(nxt_b[1]), hb._ptr(dt_b),
                     phys.C_min, phys.g, phys.gm1, phys.divgamma, phys.k, nb[0], nb[1], dtd[0], dtd[1], stream, 1,
                     ctypes.byref(ib))
        assert rc == 0, hb.last_error()
        cuda.cuda.synchronize()
        assert cuda.equal(nxt_a[0], nxt_b[0]), f"call {call}: rho/E differ"
        assert cuda.equal(nxt_a[1], nxt_b[1]), f"call {call}: momenta differ"
        assert dt_a.item() == dt_b.item(), f"call {call}: Dt_next differs"
        assert ia.max_speed == ib.max_speed and ia.err == ib.err == 0
        assert abs(ia.mass - ib.mass) <= 1e-14 * abs(ia.mass)
        cur_a, cur_b = nxt_a, nxt_b
        dt = np.float64(dt_a.item())


def test_noalloc_rejects_grids_beyond_its_scratch(cuda):
    L = hb.lib()
    noalloc = _declare(L)
    one = cuda.zeros(4, dtype=cuda.float64, device="cuda")
    p = hb._ptr(one)
    rc = noalloc(p, p, p, p, p, 0.1, 1.4, 0.4, 2.5, 1.1, 4, 10_000_000, 1e-3, 1e-3, hb._stream_handle(), 1, None)
    assert rc == hb.HYDRO_ERR_ARG
    code, msg = hb.last_error()
    assert code == hb.HYDRO_ERR_ARG and "exceeds the fixed scratch" in msg

"""The allocation-free 2D FP64 step (hydro2d_step_f64_noalloc), through the C ABI.

It exists for callers that cannot allocate: programs whose GPU memory is owned by their own
pool or caching allocator, stepping loops that must not run cudaMalloc/cudaFree (which can
synchronise the whole device), and programs built to allocate nothing after start-up. Its
scratch is a fixed array inside the library instead of memory allocated on first use.

Checked here, bit for bit (the tolerance of every FP64 test in this suite):
* two calls in a row, each against the regular entry point (hydro2d_step_f64) on the same
  inputs; the Dt_next and the step results (mass, max speed) agree;
* one call against the oracle directly;
* arrays offset by 8 bytes, which the strip kernel's 16-byte staging rejects: the step
  falls back to the direct kernel and matches hydro2d_step_f64 with the direct kernel;
* an asynchronous call (sync = 0) on a state with a negative density: its results and
  its error code come back through hydro2d_noalloc_last_info, and the next good call
  clears them;
* in a fresh process that calls only the allocation-free entry points, the library
  creates none of the per-device contexts the regular entry points allocate;
* a grid beyond the fixed scratch is rejected.
The file is named to be collected last, and passes alone in a fresh process too.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
import sys
import textwrap

import numpy as np
import pytest

from conftest import ROOT, load_pkg

hb = load_pkg()
pytestmark = pytest.mark.gpu


def _declare(L):
    d = ctypes.c_double
    fn = L.hydro2d_step_f64_noalloc
    fn.argtypes = [ctypes.c_void_p] * 5 + [d] * 5 + [ctypes.c_size_t] * 2 + [d] * 2 + [
        ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(hb.StepInfo)]
    fn.restype = ctypes.c_int
    L.hydro2d_noalloc_last_info.argtypes = [ctypes.c_void_p, ctypes.POINTER(hb.StepInfo)]
    L.hydro2d_noalloc_last_info.restype = ctypes.c_int
    return fn


def _call(fn, cur, nxt, dt, phys, nb, dtd, sync, info=None):
    return fn(hb._ptr(cur[0]), hb._ptr(cur[1]), hb._ptr(nxt[0]), hb._ptr(nxt[1]), hb._ptr(dt), phys.C_min, phys.g,
              phys.gm1, phys.divgamma, phys.k, nb[0], nb[1], dtd[0], dtd[1], hb._stream_handle(), sync,
              ctypes.byref(info) if info is not None else None)


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
                                dtd[0], dtd[1], stream, hb.ARITH_STRICT, 1, ctypes.byref(ia))
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


def test_noalloc_matches_oracle(cuda, oracle):
    nb = (61, 130)
    phys = hb.Physics(np.float64, nb)
    fn = _declare(hb.lib())
    st = tuple(a.cpu().numpy() for a in _state(cuda, nb, 5))
    oracle.ghost_x(st, nb)  # the oracle reads the X ghost rows, the kernel wraps in-kernel
    ref = (np.zeros_like(st[0]), np.zeros_like(st[1]))
    dtd = phys.dtd(np.float64(0.05) * phys.min_spacing / np.float64(6))
    dref = oracle.step(st, ref, phys, dtd)
    cur = tuple(cuda.from_numpy(a.copy()).cuda() for a in st)
    nxt = tuple(cuda.zeros_like(a) for a in cur)
    dt = cuda.zeros(1, dtype=cuda.float64, device="cuda")
    info = hb.StepInfo()
    assert _call(fn, cur, nxt, dt, phys, nb, dtd, 1, info) == 0, hb.last_error()
    assert info.kernel == hb.KERNEL_STRIP
    assert nxt[0].cpu().numpy().tobytes() == ref[0].tobytes()
    assert nxt[1].cpu().numpy().tobytes() == ref[1].tobytes()
    assert np.float64(dt.item()).tobytes() == dref.tobytes()


def test_noalloc_direct_fallback_on_misaligned_arrays(cuda):
    """Arrays that start 8 bytes past a 16-byte boundary: the step runs the direct kernel
    and matches hydro2d_step_f64 forced to the direct kernel, twice in a row."""
    nb = (40, 77)
    phys = hb.Physics(np.float64, nb)
    L = hb.lib()
    fn = _declare(L)

    def shifted(a):
        buf = cuda.zeros(a.numel() + 1, dtype=a.dtype, device="cuda")
        v = buf[1:]
        v.copy_(a)
        assert v.data_ptr() % 16 == 8
        return v

    src = _state(cuda, nb, 9)
    cur_a = tuple(shifted(a) for a in src)
    cur_b = tuple(shifted(a) for a in src)
    dt_a = cuda.zeros(1, dtype=cuda.float64, device="cuda")
    dt_b = cuda.zeros(1, dtype=cuda.float64, device="cuda")
    dt = np.float64(0.05) * phys.min_spacing / np.float64(6)
    for call in range(2):
        dtd = phys.dtd(dt)
        nxt_a = tuple(shifted(cuda.zeros_like(a)) for a in src)
        nxt_b = tuple(shifted(cuda.zeros_like(a)) for a in src)
        ia, ib = hb.StepInfo(), hb.StepInfo()
        rc = L.hydro2d_step_f64(hb._ptr(cur_a[0]), hb._ptr(cur_a[1]), hb._ptr(nxt_a[0]), hb._ptr(nxt_a[1]),
                                hb._ptr(dt_a), phys.C_min, phys.g, phys.gm1, phys.divgamma, phys.k, nb[0], nb[1],
                                dtd[0], dtd[1], hb._stream_handle(), hb.KERNEL_DIRECT, 1, ctypes.byref(ia))
        assert rc == 0, hb.last_error()
        assert _call(fn, cur_b, nxt_b, dt_b, phys, nb, dtd, 1, ib) == 0, hb.last_error()
        assert ib.kernel == hb.KERNEL_DIRECT
        assert cuda.equal(nxt_a[0], nxt_b[0]) and cuda.equal(nxt_a[1], nxt_b[1]), f"call {call}"
        assert dt_a.item() == dt_b.item() and ia.max_speed == ib.max_speed
        cur_a, cur_b = nxt_a, nxt_b
        dt = np.float64(dt_a.item())


def test_noalloc_async_results_and_errors(cuda):
    """sync = 0 only enqueues; hydro2d_noalloc_last_info reads the step's record from the
    fixed array: a negative density is reported, and a following good step clears it."""
    nb = (50, 64)
    phys = hb.Physics(np.float64, nb)
    L = hb.lib()
    fn = _declare(L)
    dtd = phys.dtd(np.float64(0.05) * phys.min_spacing / np.float64(6))
    good = _state(cuda, nb, 3)
    bad = tuple(a.clone() for a in good)
    c = 20 * (nb[1] + 2) + 30
    bad[0][2 * c] = -1.0  # one interior cell with rho < 0
    nxt = tuple(cuda.zeros_like(a) for a in good)
    dt = cuda.zeros(1, dtype=cuda.float64, device="cuda")
    info = hb.StepInfo()
    assert _call(fn, bad, nxt, dt, phys, nb, dtd, 0) == 0, hb.last_error()
    rc = L.hydro2d_noalloc_last_info(hb._stream_handle(), ctypes.byref(info))
    assert rc == hb.HYDRO_ERR_NONPHYSICAL
    assert info.err & 1 and info.kernel == hb.KERNEL_STRIP
    ref = hb.StepInfo()
    assert _call(fn, good, nxt, dt, phys, nb, dtd, 1, ref) == 0, hb.last_error()
    assert _call(fn, good, nxt, dt, phys, nb, dtd, 0) == 0, hb.last_error()
    rc = L.hydro2d_noalloc_last_info(hb._stream_handle(), ctypes.byref(info))
    assert rc == hb.HYDRO_OK and info.err == 0
    assert info.max_speed == ref.max_speed and info.mass == ref.mass


def test_noalloc_allocates_no_context(cuda):
    """A fresh process that steps only through the allocation-free entry points: the
    library creates none of the per-device contexts (scratch words, partials, pinned
    status record) that the regular entry points allocate on first use."""
    code = textwrap.dedent(f"""
        import ctypes, sys
        import numpy as np
        sys.path.insert(0, {str(ROOT / 'tests')!r})
        from conftest import load_pkg
        import torch
        hb = load_pkg()
        L = hb.lib()
        d = ctypes.c_double
        fn = L.hydro2d_step_f64_noalloc
        fn.argtypes = [ctypes.c_void_p] * 5 + [d] * 5 + [ctypes.c_size_t] * 2 + [d] * 2 + [
            ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(hb.StepInfo)]
        fn.restype = ctypes.c_int
        nb = (30, 40)
        phys = hb.Physics(np.float64, nb)
        n = (nb[0] + 2) * (nb[1] + 2)
        rhoE = torch.tensor([1.0, 2.5] * n, dtype=torch.float64, device="cuda")
        uv = torch.zeros(2 * n, dtype=torch.float64, device="cuda")
        out = (torch.zeros_like(rhoE), torch.zeros_like(uv))
        dt = torch.zeros(1, dtype=torch.float64, device="cuda")
        dtd = phys.dtd(np.float64(1e-3))
        info = hb.StepInfo()
        for _ in range(2):
            rc = fn(hb._ptr(rhoE), hb._ptr(uv), hb._ptr(out[0]), hb._ptr(out[1]), hb._ptr(dt), phys.C_min, phys.g,
                    phys.gm1, phys.divgamma, phys.k, nb[0], nb[1], dtd[0], dtd[1], None, 1, ctypes.byref(info))
            assert rc == 0, hb.last_error()
        L.hydro_device_contexts.restype = ctypes.c_int
        print("contexts", L.hydro_device_contexts())
    """)
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=600,
                       env=dict(os.environ))
    assert r.returncode == 0, r.stderr[-2000:]
    assert "contexts 0" in r.stdout, r.stdout

"""Parity at the full sizes of the large plain-path configurations: the 2D 40000 x 20000 and
the 3D 512^3 blast, FP64 and FP32, three steps from the blast initial condition on the GPU,
each step checked against the oracle restatement on the host.

The whole grid does not fit the host as the reference program holds it (51.2 GB of state in
2D FP64), and the reference program itself cannot run 512^3 (its line-buffer size check
exits, hydro3d/main.cxx:550-563). So each step is checked slab by slab: the GPU's input
state of the step is copied to the host a slab of rows (planes) at a time, with the X
neighbours of the first and last interior rows wrapped periodically as the kernels do, the
oracle steps the slab (it reads the two rows around it as its X ghost rows), and its output
rows are compared byte for byte with the GPU's output rows. A chain of steps that are each
bit-identical from identical inputs is bit-identical as a whole. The step's Dt_next is the
minimum of the slabs' C_min / max_speed: division by a positive maximum is monotone, so the
slab minimum is the global value, compared bit for bit. Slabs run on all host cores (the
oracle call releases the GIL).

Also checked: the device initial condition's total mass and first Dt against the oracle's
cell-by-cell statistics of the same blast, and the fused mass of each step against the
oracle's sums of the slabs (1e-13 relative: the two sums group the cells differently).
"""
from __future__ import annotations

import hashlib
import os
from concurrent.futures import ThreadPoolExecutor

import numpy as np
import pytest

from conftest import load_pkg

hb = load_pkg()
pytestmark = [pytest.mark.gpu, pytest.mark.slow]


def _threads():
    try:
        return max(1, len(os.sched_getaffinity(0)))
    except Exception:
        return os.cpu_count() or 1


def _rows(t, row_elems, a, b):
    """Rows a..b-1 of a flat device array with `row_elems` elements per row, on the host."""
    return t[row_elems * a:row_elems * b].cpu().numpy()


def _slab_input(state, nb, nv, i0, i1):
    """Rows (planes) i0-1 .. i1+1 of `state`, the X ghosts wrapped periodically."""
    plane = int(np.prod([n + 2 for n in nb[1:]]))
    out = []
    for t, w in ((state[0], 2), (state[1], nv)):
        re = plane * w
        parts = []
        lo = i0 - 1
        if lo == 0:
            parts.append(_rows(t, re, nb[0], nb[0] + 1))
            lo = 1
        hi = i1 + 1
        top = None
        if hi == nb[0] + 1:
            top = _rows(t, re, 1, 2)
            hi = nb[0]
        parts.append(_rows(t, re, lo, hi + 1))
        if top is not None:
            parts.append(top)
        out.append(np.ascontiguousarray(np.concatenate(parts)))
    return tuple(out)


def _check_step(oracle, phys, dtd, nb, before, after, dt_dev, info, slab_rows):
    """The GPU step before -> after against the oracle, slab by slab; returns the digests."""
    nv = len(nb)
    T = phys.dtype
    plane = int(np.prod([n + 2 for n in nb[1:]]))
    slabs = [(i0, min(nb[0], i0 + slab_rows - 1)) for i0 in range(1, nb[0] + 1, slab_rows)]

    def work(s):
        i0, i1 = s
        inp = _slab_input(before, nb, nv, i0, i1)
        ref = (np.zeros_like(inp[0]), np.zeros_like(inp[1]))
        sp = hb.Physics(T, nb)
        sp.nb = (i1 - i0 + 1,) + tuple(nb[1:])  # the slab: its rows with the two around it as ghosts
        dref = oracle.step(inp, ref, sp, dtd)
        got = (_rows(after[0], plane * 2, i0, i1 + 1), _rows(after[1], plane * nv, i0, i1 + 1))
        want = (ref[0][plane * 2:-plane * 2], ref[1][plane * nv:-plane * nv])
        inner = tuple(slice(1, n + 1) for n in nb[1:])
        g = [a.reshape((i1 - i0 + 1,) + tuple(n + 2 for n in nb[1:]) + (w,))[(slice(None),) + inner]
             for a, w in zip(got, (2, nv))]
        r = [a.reshape((i1 - i0 + 1,) + tuple(n + 2 for n in nb[1:]) + (w,))[(slice(None),) + inner]
             for a, w in zip(want, (2, nv))]
        dg, dr = hashlib.sha256(), hashlib.sha256()
        for x, y in zip(g, r):
            dg.update(np.ascontiguousarray(x).tobytes())
            dr.update(np.ascontiguousarray(y).tobytes())
        m = oracle.mass(ref[0], sp.nb)
        return i0, dg.digest() == dr.digest(), dref, m, dg.digest(), dr.digest()

    # a digest of the slabs' digests, in row order, on each side
    hg, hr = hashlib.sha256(), hashlib.sha256()
    dmin, mass, bad = None, 0.0, []
    with ThreadPoolExecutor(_threads()) as ex:
        for i0, same, dref, m, dg, dr in ex.map(work, slabs):
            if not same:
                bad.append(i0)
            hg.update(dg)
            hr.update(dr)
            dmin = dref if dmin is None or dref < dmin else dmin
            mass += m
    assert not bad, f"slabs starting at rows {bad[:5]} differ from the oracle"
    assert hg.hexdigest() == hr.hexdigest()
    assert T(dt_dev).tobytes() == T(dmin).tobytes(), (dt_dev, dmin)
    assert abs(info.mass - mass) <= 1e-13 * abs(mass)
    return hg.hexdigest()


@pytest.mark.parametrize("T", [np.float64, np.float32])
@pytest.mark.parametrize("nb,slab_rows", [((40000, 20000), 200), ((512, 512, 512), 16)])
def test_large_grid_steps_match_oracle(cuda, oracle, nb, slab_rows, T):
    run = hb.BlastRun(nb, T, arith="strict")
    phys = run.phys
    # the device initial condition: mass and first Dt against the oracle's statistics
    m0, dt0 = oracle.blast_stats(nb, phys)
    assert T(run.first_dt).tobytes() == T(dt0).tobytes()
    assert abs(run.mass0 - m0) <= 1e-13 * abs(m0)
    for _ in range(3):
        dtd = phys.dtd(run.dt)
        run.step()
        # after the swap: run.nxt holds the step's input, run.cur its output
        _check_step(oracle, phys, dtd, nb, run.nxt, run.cur, run.dt_dev.item(), run.last_info, slab_rows)
    if T is np.float64:
        # total mass conserved to 1e-13 relative (FP32 states round each update in FP32)
        m1 = run.mass()
        assert abs(m1 - run.mass0) <= 1e-13 * abs(run.mass0)
    del run
    cuda.cuda.empty_cache()

"""The reference's X-slab decomposition (--sdx N): ranks exchange edge rows between steps
and step their slabs with the X ghost rows read from memory; the result is bit-identical
to the whole domain stepped on one device. Two ranks share one GPU here (gloo, rows staged
through host memory): no kernel waits on another rank, the exchange happens between
steps on the host."""
from __future__ import annotations

import os
import socket

import numpy as np
import pytest

from conftest import ROOT, load_pkg

hb = load_pkg()
pytestmark = pytest.mark.gpu


def interior(state, nb):
    shape = tuple(n + 2 for n in nb)
    inner = tuple(slice(1, n + 1) for n in nb)
    return [a.reshape(shape + (nv,))[inner] for a, nv in zip(state, (2, len(nb)))]


@pytest.mark.parametrize("nb,T", [((60, 60), np.float64), ((64, 50), np.float32), ((20, 18, 16), np.float64)])
def test_single_rank_slab_equals_whole_domain(cuda, nb, T):
    from hydro_b200.replicas import Replicas
    from hydro_b200.slabs import XSlabRun

    steps = 20
    whole = hb.BlastRun(nb, T).run(1e9, steps)
    slab = XSlabRun(nb, T, Replicas("gloo", env={})).run(1e9, steps)
    assert slab.t == whole.t and np.float64(slab.dt) == np.float64(whole.dt)
    a, b = slab.interior(), interior(whole.host_state(), nb)
    assert a[0].tobytes() == b[0].tobytes() and a[1].tobytes() == b[1].tobytes()
    assert abs(slab.mass() - whole.mass()) <= 1e-13 * whole.mass()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, nb, dtname, steps, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK="0")
    try:
        import sys

        sys.path.insert(0, str(ROOT / "tests"))
        from conftest import load_pkg as lp

        lp()
        import torch
        from hydro_b200.replicas import Replicas
        from hydro_b200.slabs import XSlabRun

        torch.cuda.set_device(0)
        reps = Replicas("gloo", timeout_s=120)
        run = XSlabRun(nb, np.dtype(dtname).type, reps).run(1e9, steps)
        inner = run.interior()
        m = run.mass()
        q.put((rank, run.lo, run.hi, run.t, float(run.dt), m, inner[0].copy(), inner[1].copy()))
        reps.close()
    except Exception as e:  # reported to the parent
        import traceback

        q.put((rank, None, None, None, None, None, repr(e) + traceback.format_exc(), None))


@pytest.mark.parametrize("world,nb,T", [(2, (64, 50), np.float64), (3, (31, 40), np.float32),
                                        (2, (18, 12, 34), np.float64)])
def test_ranks_on_one_gpu_equal_whole_domain(cuda, world, nb, T):
    import multiprocessing as mp

    steps = 15
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, nb, np.dtype(T).name, steps, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = sorted((q.get(timeout=300) for _ in procs), key=lambda o: o[0])
    for p in procs:
        p.join(timeout=120)
    for o in out:
        assert o[1] is not None, o[6]
    whole = hb.BlastRun(nb, T).run(1e9, steps)
    ref = interior(whole.host_state(), nb)
    for rank, lo, hi, t, dt, m, r, u in out:
        assert t == whole.t and dt == float(whole.dt), rank
        assert r.tobytes() == np.ascontiguousarray(ref[0][lo - 1:hi]).tobytes(), rank
        assert u.tobytes() == np.ascontiguousarray(ref[1][lo - 1:hi]).tobytes(), rank
        assert abs(m - whole.mass()) <= 1e-13 * whole.mass()
    assert [o[1] for o in out][0] == 1 and out[-1][2] == nb[0]

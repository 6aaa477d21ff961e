"""Host-side logic without a GPU: the seeded workloads, the serving summary, and the
replica bookkeeping and the X-slab ghost exchange over worlds of two and three gloo ranks
on CPU."""
from __future__ import annotations

import math
import os
import socket
import time

import numpy as np
import pytest

from conftest import load_pkg

hb = load_pkg()


def test_request_stream_needs_a_bound():
    from hydro_b200.workloads import request_stream

    with pytest.raises(ValueError):
        request_stream(10.0)
    a = request_stream(10.0, seed=4, count=12)
    assert len(a) == 12 and all(x.arrival < y.arrival for x, y in zip(a, a[1:]))
    b = request_stream(10.0, duration=a[5].arrival + 1e-9, seed=4)
    assert [r.rid for r in b] == list(range(6))
    assert [r.blast.nb for r in b] == [r.blast.nb for r in a[:6]]


def test_request_stream_distribution():
    """Sides, dimensionality, precision and t_end follow the serving workload's ranges."""
    from hydro_b200.workloads import request_stream, sound_crossing_time

    reqs = request_stream(1000.0, seed=1, count=2000)
    tc = sound_crossing_time()
    n3 = sum(len(r.blast.nb) == 3 for r in reqs)
    assert 0.25 < n3 / len(reqs) < 0.35
    assert 0.45 < sum(r.dtype is np.float64 for r in reqs) / len(reqs) < 0.55
    for r in reqs:
        lo, hi = (32, 256) if len(r.blast.nb) == 3 else (64, 4096)
        assert all(lo <= n <= hi for n in r.blast.nb), r.blast.nb
        assert 0.05 * tc <= r.blast.t_end <= 0.5 * tc
        ratio = r.blast.p_in / r.blast.p_out
        assert 10 - 1e-9 <= ratio <= 1000 + 1e-9
    gaps = np.diff([0.0] + [r.arrival for r in reqs])
    assert abs(gaps.mean() - 1e-3) < 1e-4  # Poisson arrivals at the requested rate


def test_batch_blasts_distribution():
    from hydro_b200.workloads import batch_blasts

    bl = batch_blasts(512, seed=2, steps=200)
    for b in bl:
        lo, hi = sorted(b.nb)
        assert 32 <= lo and hi <= 2048 and hi / lo <= 2.0 + 1e-6
        assert 0.05 * lo - 1e-9 <= b.radius <= 0.2 * lo + 1e-9
        assert b.max_steps == 200 and b.rho_in == b.rho_out == 1.0 and b.gamma == 1.4
        for c, n in zip(b.centre, b.nb):
            assert 1 + 0.25 * (n - 1) - 1e-9 <= c <= 1 + 0.75 * (n - 1) + 1e-9


def test_summarize_counts_partial_work():
    from hydro_b200.serving import Record, summarize

    recs = [Record(0, 0.0, done=1.0, steps=10, cells=100), Record(1, 0.5, done=3.5, steps=20, cells=50),
            Record(2, 1.0, steps=7, cells=1000)]  # unfinished: counts as work, not latency
    s = summarize(recs, wall=4.0)
    assert s["completed"] == 2 and s["requests"] == 3
    assert s["cell_updates"] == 10 * 100 + 20 * 50 + 7 * 1000
    assert math.isclose(s["p50_s"], 2.0) and s["p99_s"] <= 3.0 + 1e-12
    assert math.isclose(s["gcell_s"], 9000 / 4.0 / 1e9)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    try:
        import importlib.util
        import sys

        from conftest import ROOT

        spec = importlib.util.spec_from_file_location(
            "hydro_b200_replicas", ROOT / "scalable-fpga-hydrodynamics_b200" / "replicas.py")
        mod = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(mod)
        reps = mod.Replicas("gloo", timeout_s=60)
        reps.barrier()
        mx = reps.max_over_ranks(10.0 * (rank + 1))
        sm = reps.sum_over_ranks(rank + 1)
        share = reps.share(range(11))
        reps.barrier()
        reps.close()
        q.put((rank, mx, sm, share))
    except Exception as e:  # reported to the parent
        q.put((rank, repr(e), None, None))


def test_replicas_gloo_two_ranks():
    """Two ranks on CPU: max-over-ranks timing, the sum of work, and disjoint complete
    shares of a request stream."""
    import multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [o[1] for o in out] == [20.0, 20.0], out
    assert [o[2] for o in out] == [3.0, 3.0]
    shares = [o[3] for o in out]
    assert sorted(shares[0] + shares[1]) == list(range(11)) and not set(shares[0]) & set(shares[1])


def test_replicas_single_process_is_identity():
    from hydro_b200.replicas import Replicas

    r = Replicas("gloo", env={})
    assert (r.rank, r.world) == (0, 1)
    assert r.max_over_ranks(3.5) == 3.5 and r.share([1, 2, 3]) == [1, 2, 3]
    r.barrier()
    r.close()


def test_slab_rows_partition():
    from hydro_b200.slabs import slab_rows

    for nb_x in (1, 7, 40000):
        for world in range(1, min(nb_x, 9) + 1):
            rows = [slab_rows(nb_x, world, r) for r in range(world)]
            assert rows[0][0] == 1 and rows[-1][1] == nb_x
            assert all(b[0] == a[1] + 1 for a, b in zip(rows, rows[1:]))
            sizes = [hi - lo + 1 for lo, hi in rows]
            assert max(sizes) - min(sizes) <= 1 and min(sizes) >= 1
    with pytest.raises(hb.HydroError):
        slab_rows(2, 3, 0)


def _slab_rank_main(rank, world, port, nb, q):
    """One gloo rank: fill its slab with values naming (global row, column, component),
    exchange the X ghost rows and report what landed in them, plus the MIN of Dt."""
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    try:
        import torch

        from conftest import load_pkg as _load

        _load()
        from hydro_b200.replicas import Replicas
        from hydro_b200.slabs import XSlabRun, slab_rows

        reps = Replicas("gloo", timeout_s=60)
        run = XSlabRun.__new__(XSlabRun)  # the exchange and Dt logic only: no device state
        run.torch, run.reps, run.nb, run.T = torch, reps, tuple(nb), np.float64
        run.lo, run.hi = slab_rows(nb[0], world, rank)
        n = run.hi - run.lo + 1
        run.nb_local = (n,) + tuple(nb[1:])
        run.row = int(np.prod([m + 2 for m in nb[1:]]))
        arrays = []
        for nv in (2, len(nb)):
            a = np.full((n + 2, run.row, nv), -1.0)
            for i in range(1, n + 1):
                g = run.lo + i - 1
                a[i] = g * 1e4 + np.arange(run.row)[:, None] * 10 + np.arange(nv)[None, :]
            arrays.append(torch.from_numpy(a.reshape(-1).copy()))
        run.cur = tuple(arrays)
        run.exchange()
        ghosts = [(a.numpy().reshape(n + 2, run.row, -1)[0].copy(), a.numpy().reshape(n + 2, run.row, -1)[n + 1].copy())
                  for a in run.cur]
        dt = run._min_host(0.25 + rank)
        reps.barrier()
        reps.close()
        q.put((rank, run.lo, run.hi, ghosts, float(dt)))
    except Exception as e:  # reported to the parent
        q.put((rank, repr(e), None, None, None))


@pytest.mark.parametrize("world,nb", [(2, (6, 5)), (3, (7, 4)), (2, (4, 3, 2)), (3, (5, 2, 3))])
def test_slab_exchange_gloo(world, nb):
    """The X-slab ghost exchange across gloo ranks on CPU: ghost row 0 of each rank holds
    the last interior row of the rank on its left and ghost row NB+1 the first row of the
    rank on its right, periodically (with two ranks both neighbours are the same peer);
    the next Dt is the MIN over ranks."""
    import multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_slab_rank_main, args=(r, world, port, nb, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = sorted((q.get(timeout=120) for _ in procs), key=lambda o: o[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    row = int(np.prod([m + 2 for m in nb[1:]]))
    for rank, lo, hi, ghosts, dt in out:
        assert ghosts is not None, lo
        assert dt == 0.25
        left = lo - 1 if lo > 1 else nb[0]    # global row below this slab (periodic)
        right = hi + 1 if hi < nb[0] else 1   # global row above it
        for (g0, g1), nv in zip(ghosts, (2, len(nb))):
            cols = np.arange(row)[:, None] * 10 + np.arange(nv)[None, :]
            np.testing.assert_array_equal(g0, left * 1e4 + cols)
            np.testing.assert_array_equal(g1, right * 1e4 + cols)


class _FakeEngine:
    """Stands in for a batch engine: each instance needs `max_steps` steps, occupies
    100 bytes per cell, and `run(n)` advances every active instance by up to n steps (the
    engine's device-side end condition stops an instance at exactly its need)."""

    def __init__(self, log):
        self.log, self.slots, self.next = log, {}, 0

    def bytes(self, blast):
        return 100 * int(np.prod(blast.nb))

    def add(self, blast):
        self.next += 1
        self.slots[self.next] = [blast, 0]
        self.log.append(("add", id(self), self.next, self.bytes(blast)))
        return self.next

    def run(self, n, sync=True):
        time.sleep(0.001)  # a tick takes time, so later arrivals meet running work
        for s in self.slots.values():
            s[1] = min(s[1] + n, s[0].max_steps)

    def sync(self):
        pass

    def status(self, slot):
        b, steps = self.slots[slot]
        return {"active": steps < b.max_steps, "steps": steps, "err": 0}

    def remove(self, slot):
        self.log.append(("remove", id(self), slot, self.bytes(self.slots[slot][0])))
        del self.slots[slot]

    def state(self, slot):
        return None

    def close(self):
        pass


def test_server_admission_on_cpu():
    """The continuous-batching loop with fake engines: first-come first-served admission,
    the memory budget never exceeded, a request that can never fit rejected, requests that
    arrive while others run admitted at once when room allows, and every admitted request
    retired after exactly the steps it needs."""
    from hydro_b200.batch import Blast
    from hydro_b200.serving import Server
    from hydro_b200.workloads import Request

    log = []
    srv = Server.__new__(Server)  # the scheduling loop only: no device
    srv.budget, srv.steps_per_tick, srv.engines, srv.streams = 100 * 10_000.0, 4, {}, {}

    def engine(dim, dtype):
        key = (dim, np.dtype(dtype).name)
        if key not in srv.engines:
            srv.engines[key] = _FakeEngine(log)
        return srv.engines[key]

    srv.engine = engine
    sizes = [(60, 60), (50, 40), (90, 90), (20, 30, 10), (200, 200), (10, 10), (40, 40, 4)]
    need = [9, 30, 13, 5, 3, 21, 7]
    reqs = [Request(rid=i, arrival=0.0005 * i, blast=Blast(nb=nb, max_steps=n),
                    dtype=np.float32 if i % 2 else np.float64)
            for i, (nb, n) in enumerate(zip(sizes, need))]
    recs, wall = srv.serve(reqs, max_wall=30.0)
    recs = {r.rid: r for r in recs}
    # (200, 200) needs 4 MB against a 1 MB budget: rejected, never admitted
    assert recs[4].err == -1 and recs[4].admit is None and recs[4].done is None
    for r in reqs:
        if r.rid != 4:
            assert recs[r.rid].done is not None and recs[r.rid].steps == r.blast.max_steps, r.rid
    # memory in use never above the budget
    used = peak = 0
    for ev, _eng, _slot, nbytes in log:
        used += nbytes if ev == "add" else -nbytes
        peak = max(peak, used)
    assert peak <= srv.budget and used == 0
    # admission in arrival order
    admitted = [rid for rid in sorted(recs, key=lambda k: recs[k].admit or 1e30) if recs[rid].admit is not None]
    assert admitted == sorted(admitted)
    # continuous batching: the second request joined while the first was still running
    assert recs[1].admit < recs[0].done


def _oracle_slab_rank(rank, world, port, nb, steps, overlap, q):
    """One gloo rank stepping its slab with the oracle on the host through XSlabRun's
    schedule (edge rows, their exchange, interior rows, Dt MIN); reports its interior,
    t and Dt."""
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    try:
        import torch

        from conftest import load_pkg as _load

        _load()
        import oracle as orc
        from hydro_b200 import Physics
        from hydro_b200.replicas import Replicas
        from hydro_b200.slabs import XSlabRun, slab_rows

        o = orc.Oracle()
        T = np.float64
        phys = Physics(T, nb)
        full = tuple(np.zeros(int(np.prod([n + 2 for n in nb])) * k, T) for k in (2, len(nb)))
        first = o.init(full, phys)
        lo, hi = slab_rows(nb[0], world, rank)
        row = int(np.prod([n + 2 for n in nb[1:]]))
        state = tuple(torch.from_numpy(a[(lo - 1) * row * k:(hi + 2) * row * k].copy())
                      for a, k in zip(full, (2, len(nb))))

        def stepper(cur, nxt, dt_out, p, dtd, sync):
            d = o.step(tuple(a.numpy() for a in cur), tuple(a.numpy() for a in nxt), p, dtd)
            dt_out.fill_(float(d))
            return None

        reps = Replicas("gloo", timeout_s=60)
        run = XSlabRun(nb, T, reps, overlap=overlap, stepper=stepper, state=(state, first)).run(1e9, steps)
        out = run.interior()
        reps.barrier()
        reps.close()
        q.put((rank, lo, hi, [a.copy() for a in out], run.t, float(run.dt)))
    except Exception as e:  # reported to the parent
        import traceback

        q.put((rank, traceback.format_exc(), None, None, None, None))


@pytest.mark.parametrize("overlap", [True, False])
@pytest.mark.parametrize("world,nb", [(2, (13, 9)), (3, (11, 6)), (2, (9, 6, 5)), (3, (8, 5, 4))])
def test_slab_schedule_gloo_matches_whole_domain(world, nb, overlap):
    """XSlabRun's step schedule across gloo ranks on CPU, with the oracle as the step: the
    edge rows first, their exchange in flight while the interior rows are updated, then
    the Dt MIN over ranks (overlap), or the whole slab then the exchange. After six steps
    the gathered slabs are bit-identical to the whole domain stepped by the oracle with
    periodic X ghosts, with the same t and Dt."""
    import multiprocessing as mp

    import oracle as orc
    from hydro_b200 import Physics

    steps = 6
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_oracle_slab_rank, args=(r, world, port, nb, steps, overlap, q))
             for r in range(world)]
    for p in procs:
        p.start()
    out = sorted((q.get(timeout=180) for _ in procs), key=lambda o: o[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, lo, *_ in out:
        assert out[rank][3] is not None, lo
    o = orc.Oracle()
    T = np.float64
    phys = Physics(T, nb)
    full = tuple(np.zeros(int(np.prod([n + 2 for n in nb])) * k, T) for k in (2, len(nb)))
    first = o.init(full, phys)
    ref, t_log, dt_log = orc.host_loop(o.step, full, phys, first, 1e9, steps)
    want = orc.interior(ref, nb)
    for k in range(2):
        got = np.concatenate([r[3][k] for r in out], axis=0)
        assert got.tobytes() == np.ascontiguousarray(want[k]).tobytes()
    for rank, lo, hi, _, t, dt in out:
        assert t == t_log[-1] + float(dt_log[-1]) and dt == float(dt_log[-1])


def test_serving_stream_matches_saved_trace():
    """The serving workload's seeded request stream (the one the serving sweep ran) is
    regenerated exactly: grids, blast parameters, end times, precisions and arrivals of
    the saved trace, and the streams at other rates are the same requests with scaled
    arrivals."""
    import json

    from conftest import GOLDEN

    load_pkg()
    from hydro_b200.workloads import request_stream

    saved = json.loads((GOLDEN / "serving_trace.json").read_text())
    reqs = request_stream(saved["rate"], seed=saved["seed"], count=saved["count"])
    assert len(reqs) == len(saved["requests"])
    for r, s in zip(reqs, saved["requests"]):
        assert r.rid == s["rid"] and list(r.blast.nb) == s["nb"] and np.dtype(r.dtype).name == s["dtype"]
        for a, b in ((r.arrival, s["arrival"]), (r.blast.radius, s["radius"]), (r.blast.p_in, s["p_in"]),
                     (r.blast.t_end, s["t_end"])):
            assert abs(a - b) <= 1e-8 * max(1.0, abs(b))
        assert all(abs(a - b) <= 1e-8 * max(1.0, abs(b)) for a, b in zip(r.blast.centre, s["centre"]))
    slow = request_stream(10.0, seed=saved["seed"], count=saved["count"])
    for a, b in zip(slow, reqs):
        assert a.blast.nb == b.blast.nb and abs(a.arrival - 10.0 * b.arrival) <= 1e-9 * max(1.0, a.arrival)

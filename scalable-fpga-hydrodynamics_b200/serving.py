"""Continuous-batching server for blast requests, and the one-at-a-time plain-path baseline.

The server admits requests as they arrive while their state fits a device-memory budget,
keeps every admitted request's state on the device inside one batch engine per
(dimensionality, precision), advances all engines concurrently a few steps per tick (one
CUDA graph per engine per tick, each on its own stream), retires each request the tick its
device-side end condition (t >= t_end) is reached, frees its memory and admits waiting
requests into the freed room. A request's time-to-solution is retirement time minus arrival.

The baseline serves the same stream first-come first-served, one request at a time,
through the plain path: the reference's host loop (one launcher call, one host Dt read-back
per step) on the drop-in kernels in the request's precision.
"""
from __future__ import annotations

import time
from collections import deque
from dataclasses import dataclass, field

import numpy as np

from . import BlastRun, _torch
from .batch import Batch


@dataclass
class Record:
    rid: int
    arrival: float
    admit: float = None
    done: float = None
    steps: int = 0
    cells: int = 0
    dim: int = 2
    precision: str = "f32"
    err: int = 0
    status: dict = field(default_factory=dict)

    @property
    def tts(self):
        return None if self.done is None else self.done - self.arrival


def summarize(records, wall):
    """Latency percentiles over the completed requests; throughput over all the work done
    within the wall time (steps of unfinished requests included)."""
    done = [r for r in records if r.done is not None]
    tts = np.array([r.tts for r in done]) if done else np.array([np.nan])
    work = sum(r.steps * r.cells for r in records)
    return dict(requests=len(records), completed=len(done), p50_s=float(np.percentile(tts, 50)),
                p99_s=float(np.percentile(tts, 99)), mean_s=float(np.mean(tts)), wall_s=wall,
                cell_updates=int(work), gcell_s=work / wall / 1e9 if wall > 0 else 0.0,
                errors=sum(1 for r in done if r.err))


class Server:
    """Continuous batching over batch engines keyed by (dim, precision)."""

    def __init__(self, hbm_budget: float = 150e9, steps_per_tick: int = 8, chunk2d: int = 0, chunk3d: int = 0,
                 capacity: int = 4096, arith: dict = None):
        """arith: the arithmetic of the engines per precision, e.g. {np.float32: "fused"}
        (missing precisions: the library default)."""
        self.torch = _torch()
        self.budget = float(hbm_budget)
        self.steps_per_tick = int(steps_per_tick)
        self.chunks = {2: chunk2d, 3: chunk3d}
        self.capacity = capacity
        self.engines = {}
        self.streams = {}
        self.stats = {}
        self.arith = {np.dtype(k).name: v for k, v in (arith or {}).items()}

    def engine(self, dim, dtype) -> Batch:
        key = (dim, np.dtype(dtype).name)
        if key not in self.engines:
            s = self.torch.cuda.Stream()
            self.streams[key] = s
            self.engines[key] = Batch(dim, dtype, chunk=self.chunks[dim], capacity=self.capacity, stream=s,
                                      arith=self.arith.get(np.dtype(dtype).name))
        return self.engines[key]

    def close(self):
        for e in self.engines.values():
            e.close()
        self.engines.clear()

    def serve(self, requests, max_wall: float = None, keep_results: bool = False, dtype=None):
        """Serve `requests` (workloads.Request) as they arrive, each in its own precision or
        all in `dtype`; returns (records, wall seconds). keep_results copies each retired
        request's final state to the host (Record.status['state'])."""
        reqs = sorted(requests, key=lambda r: r.arrival)
        prec = lambda r: dtype or r.dtype
        recs = {r.rid: Record(r.rid, r.arrival, dim=len(r.blast.nb), precision=np.dtype(prec(r)).name,
                              cells=int(np.prod(r.blast.nb))) for r in reqs}
        pending = deque()
        active = {}  # (key, slot) -> (request, bytes)
        used = 0.0
        nxt = 0
        # budget statistics: the most bytes held at once, the longest queue of arrived
        # requests waiting, and the ticks on which a waiting request did not fit
        self.stats = dict(budget_bytes=self.budget, peak_bytes=0.0, max_waiting=0, ticks_budget_bound=0, ticks=0)
        t0 = time.perf_counter()
        clock = lambda: time.perf_counter() - t0
        while True:
            now = clock()
            while nxt < len(reqs) and reqs[nxt].arrival <= now:
                pending.append(reqs[nxt])
                nxt += 1
            # admission, first come first served, while the state fits the budget
            while pending:
                r = pending[0]
                eng = self.engine(len(r.blast.nb), prec(r))
                need = eng.bytes(r.blast)
                if need > self.budget:
                    pending.popleft()
                    recs[r.rid].err = -1  # can never fit
                    continue
                if used + need > self.budget:
                    break
                slot = eng.add(r.blast)
                used += need
                active[((len(r.blast.nb), np.dtype(prec(r)).name), slot)] = (r, need)
                recs[r.rid].admit = clock()
                pending.popleft()
            self.stats["peak_bytes"] = max(self.stats["peak_bytes"], used)
            self.stats["max_waiting"] = max(self.stats["max_waiting"], len(pending))
            if pending:
                self.stats["ticks_budget_bound"] += 1
            if not active:
                if nxt >= len(reqs) and not pending:
                    break
                if nxt < len(reqs):
                    time.sleep(max(0.0, min(0.002, reqs[nxt].arrival - clock())))
                continue
            self.stats["ticks"] += 1
            busy = {k for (k, _s) in active}
            for k in busy:
                self.engines[k].run(self.steps_per_tick, sync=False)
            for k in busy:
                self.engines[k].sync()
            now = clock()
            for (k, slot), (r, need) in list(active.items()):
                st = self.engines[k].status(slot)
                if not st["active"]:
                    rec = recs[r.rid]
                    rec.done, rec.steps, rec.err, rec.status = now, st["steps"], st["err"], st
                    if keep_results:
                        st["state"] = self.engines[k].state(slot)
                    self.engines[k].remove(slot)
                    used -= need
                    del active[(k, slot)]
            if max_wall is not None and clock() > max_wall:
                for (k, slot), (r, _need) in active.items():  # work done so far, unfinished
                    recs[r.rid].steps = self.engines[k].status(slot)["steps"]
                break
        wall = clock()
        return list(recs.values()), wall


def serve_plain(requests, max_wall: float = None, dtype=None):
    """First-come first-served, one request at a time through the plain path (in each
    request's precision, or in `dtype` for all of them)."""
    torch = _torch()
    reqs = sorted(requests, key=lambda r: r.arrival)
    recs = []
    t0 = time.perf_counter()
    clock = lambda: time.perf_counter() - t0
    for r in reqs:
        T = dtype or r.dtype
        rec = Record(r.rid, r.arrival, dim=len(r.blast.nb), precision=np.dtype(T).name,
                     cells=int(np.prod(r.blast.nb)))
        recs.append(rec)
        if max_wall is not None and clock() > max_wall:
            continue
        wait = r.arrival - clock()
        if wait > 0:
            time.sleep(wait)
        rec.admit = clock()
        run = BlastRun(r.blast.nb, T, blast=r.blast)
        while run.t < r.blast.t_end and run.it < r.blast.max_steps:
            run.step()
            if max_wall is not None and clock() > max_wall:
                break
        torch.cuda.synchronize()
        if run.t >= r.blast.t_end or run.it >= r.blast.max_steps:
            rec.done = clock()
        rec.steps = run.it
        del run
    return recs, clock()

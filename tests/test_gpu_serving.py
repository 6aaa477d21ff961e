"""Serving: continuous batching admits requests as slots and memory free up, their work
overlaps on the device, and each request's result is the same alone and in the mix."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import load_pkg

hb = load_pkg()
pytestmark = pytest.mark.gpu


def small_stream(n=10, seed=5):
    from hydro_b200.workloads import request_stream

    reqs = request_stream(rate=400.0, duration=n / 400.0 * 3, seed=seed, sides_2d=(64, 160), sides_3d=(16, 40),
                          t_end_frac=(0.01, 0.03))
    return reqs[:n]


def test_serving_result_same_alone_and_in_mix(cuda):
    from hydro_b200.serving import Server, summarize

    reqs = small_stream()
    assert {len(r.blast.nb) for r in reqs} == {2, 3} and {np.dtype(r.dtype).name for r in reqs} == {"float32",
                                                                                                    "float64"}
    srv = Server(hbm_budget=2e9, steps_per_tick=4)
    recs, wall = srv.serve(reqs, keep_results=True)
    srv.close()
    s = summarize(recs, wall)
    assert s["completed"] == len(reqs) and s["errors"] == 0
    overlapped = sum(1 for a in recs for b in recs if a.rid < b.rid and b.admit < a.done and a.admit < b.done)
    assert overlapped > 0  # requests shared the device
    for r in reqs[:4]:
        alone = Server(hbm_budget=2e9, steps_per_tick=4)
        r0 = type(r)(r.rid, 0.0, r.blast, r.dtype)
        ra, _ = alone.serve([r0], keep_results=True)
        alone.close()
        mix = next(x for x in recs if x.rid == r.rid)
        a, m = ra[0].status, mix.status
        assert a["steps"] == m["steps"] and a["t"] == m["t"] and a["mass"] == m["mass"], r.rid
        assert a["state"][0].tobytes() == m["state"][0].tobytes(), r.rid
        assert a["state"][1].tobytes() == m["state"][1].tobytes(), r.rid


def test_served_result_equals_plain_path(cuda):
    """A served request (batched, device-side time stepping) and the same problem through
    the plain path's host loop: identical step count, t and interior bits."""
    import oracle as orc
    from hydro_b200.serving import Server

    reqs = small_stream(6, seed=9)
    srv = Server(hbm_budget=2e9, steps_per_tick=4)
    recs, _ = srv.serve(reqs, keep_results=True)
    srv.close()
    for r in reqs:
        rec = next(x for x in recs if x.rid == r.rid)
        run = hb.BlastRun(r.blast.nb, r.dtype, blast=r.blast)
        while run.t < r.blast.t_end:
            run.step()
        assert rec.status["steps"] == run.it and rec.status["t"] == run.t, r.rid
        ours = orc.interior(rec.status["state"], r.blast.nb)
        ref = orc.interior(run.host_state(), r.blast.nb)
        assert ours[0].tobytes() == ref[0].tobytes() and ours[1].tobytes() == ref[1].tobytes(), r.rid


def test_admission_respects_budget(cuda):
    """With room for one request at a time the server serialises them, and a request
    larger than the whole budget is rejected."""
    from hydro_b200.batch import Blast
    from hydro_b200.serving import Server
    from hydro_b200.workloads import Request

    big = [Request(i, 0.0, Blast(nb=(200, 200), rho_out=1.0, t_end=0.002), np.float32) for i in range(3)]
    huge = Request(3, 0.0, Blast(nb=(4000, 4000), t_end=0.001), np.float64)
    srv = Server(hbm_budget=1.5 * 2 * 4 * 4 * 202 * 202, steps_per_tick=2)
    recs, _ = srv.serve(big + [huge])
    srv.close()
    done = sorted((r for r in recs if r.done is not None), key=lambda r: r.admit)
    assert len(done) == 3
    for a, b in zip(done, done[1:]):
        assert b.admit >= a.done - 1e-6  # no overlap: the budget holds one at a time
    assert next(r for r in recs if r.rid == 3).err == -1

"""Batched step: bit-identical to the plain path per instance, independent of the mix,
FP32 within the stated tolerance of the FP64 oracle, conservation sums reported."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import load_pkg

hb = load_pkg()
pytestmark = pytest.mark.gpu


def interior(st, nb):
    import oracle as orc

    return orc.interior(st, nb)


@pytest.mark.parametrize("arith", ["strict", "fused"])
@pytest.mark.parametrize("T", [np.float64, np.float32])
def test_batch_instance_equals_plain_path(cuda, T, arith):
    """The reference blast through the batch (with other instances around it) and through
    the plain path in the same arithmetic: same Dt sequence end, same t, same interior bits."""
    from hydro_b200.batch import Batch, Blast

    nb = (300, 250) if T is np.float64 else (300, 252)
    steps = 40
    plain = hb.BlastRun(nb, T, arith=arith).run(1e9, steps)
    b = Batch(2, T, capacity=8, arith=arith)
    others = [b.add(Blast(nb=(97, 131), max_steps=steps + 5)), b.add(Blast(nb=(64, 500), max_steps=3))]
    slot = b.add(Blast(nb=nb, max_steps=steps))
    b.run(steps + 5)
    st = b.status(slot)
    assert st["steps"] == steps and not st["active"]
    assert st["t"] == plain.t
    assert np.float64(st["dt"]) == np.float64(plain.dt)
    ours = interior(b.state(slot), nb)
    ref = interior(plain.host_state(), nb)
    assert ours[0].tobytes() == ref[0].tobytes() and ours[1].tobytes() == ref[1].tobytes()
    assert abs(st["mass"] - plain.mass()) <= 1e-13 * st["mass"]
    assert b.status(others[1])["steps"] == 3
    b.close()


def test_batch_result_independent_of_mix(cuda):
    """Each instance alone and in a mix of 24 uneven instances: identical bits, identical
    conservation sums (the per-instance reduction order does not depend on the mix)."""
    from hydro_b200.batch import Batch
    from hydro_b200.workloads import batch_blasts

    blasts = batch_blasts(24, seed=3, steps=30)
    for bl in blasts:  # keep the test quick: shrink the largest instances
        bl.nb = tuple(min(n, 400) for n in bl.nb)
        bl.centre = tuple(min(c, n) for c, n in zip(bl.centre, bl.nb))
        bl.radius = min(bl.radius, 0.2 * min(bl.nb))
    mix = Batch(2, np.float32, capacity=64)
    slots = [mix.add(bl) for bl in blasts]
    mix.run(30)
    for k in (0, 7, 23):
        alone = Batch(2, np.float32, capacity=4)
        s = alone.add(blasts[k])
        alone.run(30)
        a, m = alone.status(s), mix.status(slots[k])
        assert a == m, (k, a, m)
        sa, sm = alone.state(s), mix.state(slots[k])
        assert sa[0].tobytes() == sm[0].tobytes() and sa[1].tobytes() == sm[1].tobytes()
        alone.close()
    mix.close()


def test_batch_fp32_accuracy_vs_fp64_oracle(cuda, oracle):
    """The reference 60x60 blast through the FP32 batch against the FP64 oracle after
    200 steps: relative L1 on rho <= 1e-5."""
    from hydro_b200.batch import Batch, Blast

    nb = (60, 60)
    r64 = oracle.run(nb, np.float64, 2.0, 200)
    b = Batch(2, np.float32, capacity=2)
    s = b.add(Blast(nb=nb, t_end=2.0, max_steps=200))
    b.run(200)
    st = b.status(s)
    assert st["steps"] == r64["it"]
    a = interior(b.state(s), nb)[0][..., 0].astype(np.float64)
    r = interior(r64["state"], nb)[0][..., 0]
    l1 = np.abs(a - r).sum() / np.abs(r).sum()
    linf = np.abs(a - r).max() / np.abs(r).max()
    print(f"batched FP32 vs FP64 oracle: rho rel L1 {l1:.2e}, rel Linf {linf:.2e}")
    assert l1 <= 1e-5
    assert abs(st["mass"] - r64["mass1"]) <= 1e-5 * r64["mass1"]
    b.close()


def test_batch_retire_remove_reuse(cuda):
    """Instances retire at t_end, slots are reused, the graph is rebuilt on change."""
    from hydro_b200.batch import Batch, Blast

    b = Batch(2, np.float32, capacity=2)
    s0 = b.add(Blast(nb=(64, 64), t_end=0.01))
    s1 = b.add(Blast(nb=(80, 48), max_steps=10))
    b.run(50)
    st0, st1 = b.status(s0), b.status(s1)
    assert not st0["active"] and st0["t"] >= 0.01 and st0["steps"] < 50
    assert st1["steps"] == 10
    b.remove(s0)
    s2 = b.add(Blast(nb=(70, 70), max_steps=5))
    assert s2 == s0
    b.run(10)
    assert b.status(s2)["steps"] == 5
    with pytest.raises(hb.HydroError):
        b.add(Blast(nb=(10, 10)))  # both slots in use
    b.close()


@pytest.mark.parametrize("arith", ["strict", "fused"])
@pytest.mark.parametrize("T", [np.float64, np.float32])
def test_batch3d_instance_equals_plain_path(cuda, T, arith):
    """A 3D blast through the 3D batch (beside two other instances) and through the plain
    3D path in the same arithmetic: same t, same Dt, same interior bits (the plain FP64
    path stages its planes by tensor maps here, the batch by per-lane copies)."""
    from hydro_b200.batch import Batch, Blast

    nb = (40, 36, 30)
    steps = 25
    bl = Blast(nb=nb, max_steps=steps)
    plain = hb.BlastRun(nb, T, blast=bl, arith=arith).run(1e9, steps)
    b = Batch(3, T, capacity=4, arith=arith)
    b.add(Blast(nb=(20, 50, 17), max_steps=steps + 3))
    b.add(Blast(nb=(33, 12, 40), max_steps=4))
    slot = b.add(bl)
    b.run(steps + 3)
    st = b.status(slot)
    assert st["steps"] == steps and not st["active"]
    assert st["t"] == plain.t
    assert np.float64(st["dt"]) == np.float64(plain.dt)
    ours = interior(b.state(slot), nb)
    ref = interior(plain.host_state(), nb)
    assert ours[0].tobytes() == ref[0].tobytes() and ours[1].tobytes() == ref[1].tobytes()
    b.close()


def test_batch3d_fp32_accuracy_vs_fp64_oracle(cuda, oracle):
    """The reference 3D blast (24^3) through the FP32 3D batch against the FP64 oracle:
    relative L1 on rho <= 1e-5."""
    from hydro_b200.batch import Batch, Blast

    nb = (24, 24, 24)
    r64 = oracle.run(nb, np.float64, 2.0, 60)
    b = Batch(3, np.float32, capacity=2)
    s = b.add(Blast(nb=nb, t_end=2.0, max_steps=60))
    b.run(60)
    assert b.status(s)["steps"] == r64["it"]
    a = interior(b.state(s), nb)[0][..., 0].astype(np.float64)
    r = interior(r64["state"], nb)[0][..., 0]
    l1 = np.abs(a - r).sum() / np.abs(r).sum()
    print(f"batched 3D FP32 vs FP64 oracle: rho rel L1 {l1:.2e}")
    assert l1 <= 1e-5
    b.close()


def test_autotune_picks_a_candidate(cuda, tmp_path, monkeypatch):
    """The autotuner times every candidate chunk, caches the fastest per (GPU, dim,
    precision) and `best_chunk` reads it back; an untuned key gives the default (0)."""
    import json

    import hydro_b200.autotune as at

    monkeypatch.setattr(at, "CACHE", tmp_path / "tune.json")
    assert at.best_chunk(2, np.float32) == 0
    c = at.tune(2, np.float32, candidates=(64, 256), n=6, steps=3)
    assert c in (64, 256)
    assert at.best_chunk(2, np.float32) == c
    entry = next(iter(json.loads((tmp_path / "tune.json").read_text()).values()))
    assert set(entry["gcell_s"]) == {"64", "256"} and all(v > 0 for v in entry["gcell_s"].values())
    c3 = at.tune(3, np.float64, candidates=(32, 64), n=4, steps=2)
    assert c3 in (32, 64) and at.best_chunk(3, np.float64) == c3


@pytest.mark.parametrize("dim", [2, 3])
@pytest.mark.parametrize("T", [np.float32, np.float64])
def test_batch_speed_skip_never_changes_results(cuda, dim, T):
    """The signal-speed skip is exact: with the skip off (fraction 0), at its default, and
    with every cell skipping (every step after the first then takes the exact pass over
    the instance), times, Dt, conservation sums and states are identical."""
    from hydro_b200.batch import Batch
    from hydro_b200.workloads import _blast, _sides

    rng = np.random.default_rng(21 + dim)
    lo, hi = (64, 200) if dim == 2 else (12, 40)
    blasts = [_blast(rng, _sides(rng, lo, hi, dim), max_steps=12) for _ in range(5)]
    steps = 12
    runs = []
    for frac in (0.0, 0.9, 1e30):
        b = Batch(dim, T, capacity=8)
        b.set_skip_fraction(frac)
        slots = [b.add(bl) for bl in blasts]
        b.run(steps)
        runs.append(([b.status(s) for s in slots], [b.state(s) for s in slots]))
        b.close()
    for st_a, st_b in zip(runs[0][0], runs[2][0]):
        assert st_a["exact_passes"] == 0 and st_b["exact_passes"] == steps - 1
    for (stats, states) in runs[1:]:
        for a, b2 in zip(runs[0][0], stats):
            a, b2 = dict(a), dict(b2)
            a.pop("exact_passes"), b2.pop("exact_passes")
            assert a == b2
        for (ra, ua), (rb, ub) in zip(runs[0][1], states):
            assert ra.tobytes() == rb.tobytes() and ua.tobytes() == ub.tobytes()
    with pytest.raises(hb.HydroError):
        Batch(dim, T, capacity=1).set_skip_fraction(-1.0)

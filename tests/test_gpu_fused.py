"""The fused arithmetic (HYDRO_ARITH_FUSED): products feeding sums contracted into one
rounding, reciprocal and square roots from the hardware approximations refined by one
third-order step. Not bit-identical to the reference, so it is held to tolerances:

* the refined reciprocal and square root against the correctly rounded values (numpy's
  IEEE division and square root) over many binades: within 2 ulp;
* one step on seeded states against the strict oracle: density and pressure within 1e-13
  (FP64) / 1e-5 (FP32) max pointwise relative error, the denominator floored at 1e-12 /
  1e-6 x max |field|; the velocities within the same bound relative to the field's
  largest magnitude (max |a - b| / max |b|);
* whole runs (60x60 and 60^3 x 200 iterations from the blast, 37x23 x 120) against the
  strict oracle: the same iteration count, t and Dt within 1e-12 relative, density and
  pressure within 1e-12 max pointwise relative error, velocities within 1e-12 of their
  largest magnitude;
* the mass conserved to 1e-13 relative.
A velocity component is a quotient of a small momentum by the density near the wave front
and at rest, where the fused and strict results differ by a few units in the last place of
the momenta's scale: pointwise relative to the component itself that reaches 1e-3 in cells
whose velocity is 1e-12 of the largest (measured), so velocities are held to their scale.
"""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

from conftest import load_pkg
from test_gpu_parity import primitives, to_dev
from test_oracle import SHAPES_2D, SHAPES_3D, cfl_dt, seeded_state

hb = load_pkg()
pytestmark = pytest.mark.gpu


def ulps(a, b):
    """Distance in units in the last place between same-signed finite values."""
    it = np.int64 if a.dtype == np.float64 else np.int32
    return np.abs(a.view(it).astype(np.int64) - b.view(it).astype(np.int64))


@pytest.mark.parametrize("T", [np.float64, np.float32])
def test_fused_reciprocal_and_sqrt_within_2_ulp(cuda, T):
    rng = np.random.default_rng(1)
    lo, hi = (-990, 990) if T is np.float64 else (-120, 120)
    n = 1 << 21
    x = (rng.uniform(1, 2, n) * np.exp2(rng.integers(lo, hi, n).astype(np.float64))).astype(T)
    x[: n // 4] *= -1  # negative reciprocals
    specials = np.array([1, 2, 0.5, 3, 1e-30, 1e30, np.finfo(T).tiny, np.finfo(T).max], dtype=T)
    x = np.concatenate([x, specials])
    d = cuda.from_numpy(x).cuda()
    r, s = cuda.empty_like(d), cuda.empty_like(d)
    L = hb.lib()
    fn = L.hydro_fused_math_f64 if T is np.float64 else L.hydro_fused_math_f32
    fn.argtypes = [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    fn.restype = ctypes.c_int
    assert fn(hb._ptr(d), d.numel(), hb._ptr(r), hb._ptr(s), None) == 0
    want_r = (T(1) / x).astype(T)
    pos = x > 0
    want_s = np.sqrt(x[pos]).astype(T)
    got_r, got_s = r.cpu().numpy(), s.cpu().numpy()[pos]
    fin = np.isfinite(want_r) & (want_r != 0)
    assert ulps(got_r[fin], want_r[fin]).max() <= 2
    assert ulps(got_s, want_s).max() <= 2


def max_rel(a, b, floor):
    """Density and pressure: max pointwise relative error, denominators floored at
    floor x max |field|; velocities: max absolute error over the field's max magnitude."""
    out = {}
    for k in b:
        top = np.abs(b[k]).max()
        if k in ("rho", "p"):
            den = np.maximum(np.abs(b[k]), floor * top)
            den[den == 0] = 1.0
            out[k] = float((np.abs(a[k] - b[k]) / den).max())
        else:
            out[k] = float(np.abs(a[k] - b[k]).max() / top) if top > 0 else float(np.abs(a[k]).max())
    return out


@pytest.mark.parametrize("T", [np.float64, np.float32])
@pytest.mark.parametrize("nb", SHAPES_2D[:4] + SHAPES_3D[:3] + [(300, 253), (20, 33, 62)])
def test_fused_step_close_to_strict_oracle(cuda, oracle, nb, T):
    phys = hb.Physics(T, nb)
    tol, floor = (1e-13, 1e-12) if T is np.float64 else (1e-5, 1e-6)
    for seed in range(2):
        st = seeded_state(nb, T, seed)
        oracle.ghost_x(st, nb)
        ref = (np.zeros_like(st[0]), np.zeros_like(st[1]))
        dtd = phys.dtd(cfl_dt(phys, seed))
        dref = oracle.step(st, ref, phys, dtd)
        cur = to_dev(cuda, st)
        nxt = tuple(cuda.zeros_like(a) for a in cur)
        dt = cuda.zeros(1, dtype=cur[0].dtype, device="cuda")
        _, info = hb.step(cur, nxt, dt, phys, dtd, kernel=hb.KERNEL_STRIP, arith="fused")
        assert info.kernel == hb.KERNEL_STRIP
        out = tuple(a.cpu().numpy() for a in nxt)
        err = max_rel(primitives(out, nb), primitives(ref, nb), floor)
        assert max(err.values()) <= tol, err
        assert abs(float(dt.item()) - float(dref)) <= tol * float(dref)


@pytest.mark.parametrize("nb,steps", [((60, 60), 200), ((60, 60, 60), 200), ((37, 23), 120)])
def test_fused_runs_within_1e12_of_strict_oracle(cuda, oracle, nb, steps):
    """The FP64 bar: whole runs in fused arithmetic within 1e-12 of the strict oracle."""
    ref = oracle.run(nb, np.float64, 2.0, steps)
    run = hb.BlastRun(nb, np.float64, arith="fused").run(2.0, steps)
    assert run.it == ref["it"]
    t, rt = np.array(run.t_log), ref["t"]
    assert np.all(np.abs(t - rt) <= 1e-12 * np.maximum(np.abs(rt), 1e-300))
    d, rd = np.array(run.dt_log, np.float64), ref["dt"]
    assert np.all(np.abs(d - rd) <= 1e-12 * rd)
    err = max_rel(primitives(run.host_state(), nb), primitives(ref["state"], nb), 1e-12)
    print(f"{nb} x {steps}: fused vs strict max rel err {err}")
    assert max(err.values()) <= 1e-12, err
    m1 = run.mass()
    assert abs(m1 - run.mass0) <= 1e-13 * abs(run.mass0)

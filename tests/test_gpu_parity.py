"""GPU parity: the CUDA kernels against the oracle and the reference's golden runs.

Bar: bit-for-bit for FP64 and FP32 (the kernels keep the reference's IEEE operation
order), states compared as bytes; FP32 vs the FP64 oracle stated as L1 / L-inf errors.
"""
from __future__ import annotations

import hashlib

import numpy as np
import pytest

from conftest import load_pkg
from test_oracle import SHAPES_2D, SHAPES_3D, cfl_dt, seeded_state

hb = load_pkg()
pytestmark = pytest.mark.gpu


def to_dev(cuda, st):
    return tuple(cuda.from_numpy(a.copy()).cuda() for a in st)


def digest(state):
    h = hashlib.sha256()
    for a in state:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def gpu_step(cuda, st_host, phys, dtd, kernel):
    cur = to_dev(cuda, st_host)
    nxt = tuple(cuda.zeros_like(a) for a in cur)
    tdt = cur[0].dtype
    dt = cuda.zeros(1, dtype=tdt, device="cuda")
    _, info = hb.step(cur, nxt, dt, phys, dtd, kernel=kernel, arith="strict")
    return tuple(a.cpu().numpy() for a in nxt), phys.dtype(dt.item()), info


@pytest.mark.parametrize("kernel", [hb.KERNEL_STRIP, hb.KERNEL_DIRECT])
@pytest.mark.parametrize("T", [np.float64, np.float32])
@pytest.mark.parametrize("nb", SHAPES_2D + [(128, 127), (300, 253), (1, 126), (1, 127), (257, 1)])
def test_step2d_bitwise(cuda, oracle, nb, T, kernel):
    phys = hb.Physics(T, nb)
    for seed in range(2):
        st = seeded_state(nb, T, seed)
        oracle.ghost_x(st, nb)  # the oracle reads ghost rows; the kernels wrap in-kernel
        ref = (np.zeros_like(st[0]), np.zeros_like(st[1]))
        dtd = phys.dtd(cfl_dt(phys, seed))
        dref = oracle.step(st, ref, phys, dtd)
        # FP32 with odd NB_Y: a row pitch TMA rejects, staged by per-lane copies instead
        out, d, info = gpu_step(cuda, st, phys, dtd, kernel)
        assert info.kernel == kernel
        assert d.tobytes() == dref.tobytes()
        assert out[0].tobytes() == ref[0].tobytes()
        assert out[1].tobytes() == ref[1].tobytes()
        m = oracle.mass(ref[0], nb)
        assert abs(info.mass - m) <= 1e-14 * abs(m)


@pytest.mark.parametrize("kernel", [hb.KERNEL_STRIP, hb.KERNEL_DIRECT])
@pytest.mark.parametrize("T", [np.float64, np.float32])
# (40, 150, 130): 22 x 5 tiles per plane (9-row FP64 tiles; 25 x 5 with 8 rows), most of
# them interior tiles that take the lean march; (3, 8, 34), (2, 1, 64), (5, 15, 30): 9-row
# tiles whose last tile holds one real row, a single row, a last tile one row short
@pytest.mark.parametrize("nb", SHAPES_3D + [(9, 14, 61), (4, 7, 30), (6, 13, 31), (5, 6, 62), (40, 150, 130),
                                            (3, 8, 34), (2, 1, 64), (5, 15, 30)])
def test_step3d_bitwise(cuda, oracle, nb, T, kernel):
    phys = hb.Physics(T, nb)
    for seed in range(2):
        st = seeded_state(nb, T, seed)
        oracle.ghost_x(st, nb)
        ref = (np.zeros_like(st[0]), np.zeros_like(st[1]))
        dtd = phys.dtd(cfl_dt(phys, seed))
        dref = oracle.step(st, ref, phys, dtd)
        out, d, info = gpu_step(cuda, st, phys, dtd, kernel)
        assert info.kernel == kernel
        if kernel == hb.KERNEL_STRIP:
            # FP64 planes by tensor maps where the rows are 16-byte pitched (even NB_Z)
            assert hb.last_launch_shape()["tma"] == (T is np.float64 and nb[2] % 2 == 0)
        assert d.tobytes() == dref.tobytes()
        assert out[0].tobytes() == ref[0].tobytes()
        assert out[1].tobytes() == ref[1].tobytes()


@pytest.mark.parametrize("kernel", [hb.KERNEL_AUTO, hb.KERNEL_DIRECT])
def test_golden_runs(cuda, orc, ref_runs, kernel):
    """Every committed run of the reference's own kernel, replayed through the GPU host
    loop (device IC, device step, host Dt chain): t, Dt and final state bit for bit."""
    meta, arrays = ref_runs
    for name, m in meta.items():
        T = np.dtype(m["dtype"]).type
        run = hb.BlastRun(tuple(m["nb"]), T, kernel=kernel, arith="strict").run(m["max_t"], m["max_it"])
        assert float(run.first_dt) == m["first_dt"], name
        assert run.it == m["it"], name
        assert np.array_equal(np.array(run.t_log), arrays[name + "__t"]), name
        assert np.array_equal(np.array(run.dt_log, T), arrays[name + "__dt"]), name
        assert orc.interior_digest(run.host_state(), run.nb) == m["sha256"], name


@pytest.mark.parametrize("nb", [(300, 253), (20, 33, 62)])
def test_speed_skip_redo_is_exact(cuda, oracle, nb):
    """A step whose skip threshold comes from a much faster previous state (same Dt_next
    and grid, so the history matches) must still return the exact Dt: the kernel skips
    every cell, finds its max below the threshold and the redo pass recomputes it."""
    T = np.float64
    phys = hb.Physics(T, nb)
    dt = cuda.zeros(1, dtype=cuda.float64, device="cuda")
    fast = seeded_state(nb, T, 5)
    fast[0][1::2] *= 50.0  # energy x50: signal speeds x~7
    calm = seeded_state(nb, T, 6)
    for st in (fast, calm):
        oracle.ghost_x(st, nb)
    dtd = phys.dtd(cfl_dt(phys, 0) / T(8))
    for kernel in (hb.KERNEL_STRIP, hb.KERNEL_AUTO):
        for sync in (True, False):
            for st in (fast, calm):
                cur = to_dev(cuda, st)
                nxt = tuple(cuda.zeros_like(a) for a in cur)
                hb.step(cur, nxt, dt, phys, dtd, kernel=kernel, sync=sync, arith="strict")
                cuda.cuda.synchronize()
                ref = (np.zeros_like(st[0]), np.zeros_like(st[1]))
                dref = oracle.step(st, ref, phys, dtd)
                assert T(dt.item()).tobytes() == dref.tobytes()
                assert nxt[0].cpu().numpy().tobytes() == ref[0].tobytes()


def test_strip_equals_direct_large(cuda):
    """Strip and direct kernels on a grid with many strips and chunks."""
    nb = (1500, 1000)
    for T in (np.float64, np.float32):
        a = hb.BlastRun(nb, T, kernel=hb.KERNEL_STRIP, arith="strict").run(1.0, 25)
        b = hb.BlastRun(nb, T, kernel=hb.KERNEL_DIRECT).run(1.0, 25)
        assert a.dt_log == b.dt_log
        sa, sb = a.host_state(), b.host_state()
        assert sa[0].tobytes() == sb[0].tobytes() and sa[1].tobytes() == sb[1].tobytes()
    nb3 = (70, 64, 62)
    a = hb.BlastRun(nb3, np.float64, kernel=hb.KERNEL_STRIP, arith="strict").run(1.0, 10)
    b = hb.BlastRun(nb3, np.float64, kernel=hb.KERNEL_DIRECT).run(1.0, 10)
    assert a.dt_log == b.dt_log
    assert digest(a.host_state()) == digest(b.host_state())


def primitives(st, nb):
    nv = 3 if len(nb) == 3 else 2
    r = st[0].reshape(-1, 2).astype(np.float64)
    m = st[1].reshape(-1, nv).astype(np.float64)
    shape = tuple(n + 2 for n in nb)
    inner = tuple(slice(1, n + 1) for n in nb)
    rho = r[:, 0].reshape(shape)[inner]
    E = r[:, 1].reshape(shape)[inner]
    vel = [m[:, c].reshape(shape)[inner] / rho for c in range(nv)]
    p = 0.4 * rho * (E / rho - 0.5 * sum(v * v for v in vel))
    return dict(rho=rho, p=p, **{"uvw"[c]: vel[c] for c in range(nv)})


@pytest.mark.parametrize("nb,steps", [((60, 60), 200), ((20, 16, 12), 60)])
def test_fp32_accuracy_vs_fp64_oracle(cuda, oracle, nb, steps):
    """The FP32 path against the FP64 oracle on the same blast: relative L1 on rho
    within 1e-5, L1 / L-inf of every primitive reported."""
    r64 = oracle.run(nb, np.float64, 2.0, steps)
    run = hb.BlastRun(nb, np.float32).run(2.0, steps)
    assert run.it == r64["it"]
    a, b = primitives(run.host_state(), nb), primitives(r64["state"], nb)
    for k in a:
        l1 = np.abs(a[k] - b[k]).sum() / max(np.abs(b[k]).sum(), 1e-300)
        linf = np.abs(a[k] - b[k]).max() / max(np.abs(b[k]).max(), 1e-300)
        print(f"{nb} FP32 vs FP64 {k}: rel L1 {l1:.3e}  rel Linf {linf:.3e}")
        if k == "rho":
            assert l1 <= 1e-5


def interior(a, nb, nv):
    return a.reshape(tuple(n + 2 for n in nb) + (nv,))[tuple(slice(1, n + 1) for n in nb)]


@pytest.mark.parametrize("T", [np.float64, np.float32])
@pytest.mark.parametrize("nb", [(1, 1), (6000, 1000), (3, 4000), (2500, 64), (1, 1, 1), (128, 128, 128),
                                (300, 5, 70), (7, 33, 65)])
def test_initial_condition_and_mass(cuda, oracle, nb, T):
    """Device blast IC and first Dt against the oracle, byte for byte, on grids where one
    thread covers many rows (planes) of its column and where it covers one; the device mass
    sum against the oracle's, on the same grids (many rows per block, 3D row stepping)."""
    phys = hb.Physics(T, nb)
    st = hb.alloc_state(nb, T)
    dt = hb.init_blast(st, phys)
    ref = tuple(np.zeros(a.numel(), dtype=T) for a in st)
    dref = oracle.init(ref, phys)
    assert T(dt).tobytes() == T(dref).tobytes()
    nv = 3 if len(nb) == 3 else 2
    for a, r, k in zip(st, ref, (2, nv)):
        assert interior(a.cpu().numpy(), nb, k).tobytes() == interior(r, nb, k).tobytes()
    m, mref = hb.mass(st[0], nb), oracle.mass(ref[0], nb)
    assert abs(m - mref) <= 1e-14 * abs(mref)
    # a seeded state (every cell different) through the mass sum
    rnd = seeded_state(nb, T, 3)
    m2 = hb.mass(cuda.from_numpy(rnd[0].copy()).cuda(), nb)
    assert abs(m2 - oracle.mass(rnd[0], nb)) <= 1e-14 * abs(oracle.mass(rnd[0], nb))


def test_mass_conservation(cuda):
    for nb in ((60, 60), (40, 30, 20)):
        run = hb.BlastRun(nb, np.float64).run(2.0, 200)
        m1 = run.mass()
        assert abs(m1 - run.mass0) <= 1e-13 * run.mass0
        assert abs(run.last_info.mass - m1) <= 1e-14 * m1


def test_launcher_abi(cuda):
    """The drop-in launcher signature (host DtDx refs, by-value queue) gives the same
    bits as the step entry point and returns elapsed microseconds."""
    nb = (64, 48)
    T = np.float64
    phys = hb.Physics(T, nb)
    st = seeded_state(nb, T, 7)
    cur = to_dev(cuda, st)
    n1 = tuple(cuda.zeros_like(a) for a in cur)
    n2 = tuple(cuda.zeros_like(a) for a in cur)
    d1 = cuda.zeros(1, dtype=cuda.float64, device="cuda")
    d2 = cuda.zeros(1, dtype=cuda.float64, device="cuda")
    dtd = phys.dtd(T(2e-4))
    us = hb.launcher2d(cur[0], cur[1], n1[0], n1[1], d1, phys.C_min, phys.g, phys.gm1, phys.divgamma, phys.k,
                       nb[0], nb[1], dtd[0], dtd[1])
    assert us > 0
    hb.step(cur, n2, d2, phys, dtd)
    assert cuda.equal(n1[0], n2[0]) and cuda.equal(n1[1], n2[1]) and cuda.equal(d1, d2)
    nb3 = (10, 12, 14)
    ph3 = hb.Physics(np.float32, nb3)
    st3 = seeded_state(nb3, np.float32, 3)
    c3 = to_dev(cuda, st3)
    m1 = tuple(cuda.zeros_like(a) for a in c3)
    m2 = tuple(cuda.zeros_like(a) for a in c3)
    e1 = cuda.zeros(1, dtype=cuda.float32, device="cuda")
    e2 = cuda.zeros(1, dtype=cuda.float32, device="cuda")
    dtd3 = ph3.dtd(np.float32(1e-3))
    us = hb.launcher3d(c3[0], c3[1], m1[0], m1[1], e1, ph3.C_min, ph3.g, ph3.gm1, ph3.divgamma, ph3.k, *nb3, *dtd3)
    assert us > 0
    hb.step(c3, m2, e2, ph3, dtd3)
    assert cuda.equal(m1[0], m2[0]) and cuda.equal(m1[1], m2[1]) and cuda.equal(e1, e2)


def test_errors_are_reported(cuda):
    """Argument errors return codes and latch a message; a non-physical state raises the
    flag (outputs still written) without faulting."""
    L = hb.lib()
    L.hydro_clear_error()
    nb = (16, 16)
    phys = hb.Physics(np.float64, nb)
    st = seeded_state(nb, np.float64, 1)
    cur = to_dev(cuda, st)
    nxt = tuple(cuda.zeros_like(a) for a in cur)
    dt = cuda.zeros(1, dtype=cuda.float64, device="cuda")
    rc = L.hydro2d_step_f64(None, hb._ptr(cur[1]), hb._ptr(nxt[0]), hb._ptr(nxt[1]), hb._ptr(dt), phys.C_min,
                            phys.g, phys.gm1, phys.divgamma, phys.k, 16, 16, 1e-3, 1e-3, None, 0, 1, None)
    assert rc == hb.HYDRO_ERR_ARG
    assert hb.last_error()[0] == hb.HYDRO_ERR_ARG
    bad = st[0].copy()
    bad[2 * (5 * 18 + 5)] = -1.0  # negative density in one interior cell
    cur = to_dev(cuda, (bad, st[1]))
    rc, info = hb.step(cur, nxt, dt, phys, phys.dtd(np.float64(1e-4)), check=False)
    assert rc == hb.HYDRO_ERR_NONPHYSICAL and (info.err & 1)
    # the next clean step succeeds (scratch words were re-armed)
    cur = to_dev(cuda, st)
    rc, info = hb.step(cur, nxt, dt, phys, phys.dtd(np.float64(1e-4)), check=False)
    assert rc == hb.HYDRO_OK and info.err == 0


def test_empty_grid(cuda):
    """No interior cell: the reference writes C_min / 0."""
    phys = hb.Physics(np.float64, (0, 5))
    cur = hb.alloc_state((0, 5), np.float64)
    nxt = hb.alloc_state((0, 5), np.float64)
    dt = cuda.zeros(1, dtype=cuda.float64, device="cuda")
    hb.step(cur, nxt, dt, phys, phys.dtd(np.float64(1e-3)))
    assert dt.item() == float("inf")


@pytest.mark.parametrize("kernel", [hb.KERNEL_STRIP, hb.KERNEL_DIRECT])
@pytest.mark.parametrize("T", [np.float64, np.float32])
@pytest.mark.parametrize("nb", [(7, 130), (33, 18), (3, 2, 33), (9, 14, 61)])
def test_step_x_ghosts_from_memory(cuda, oracle, nb, T, kernel):
    """With X_GHOSTS_FROM_MEMORY the kernels read the X ghost rows (planes) the caller
    filled, as the reference kernel does: arbitrary (non-periodic) ghost contents, bit for
    bit against the oracle, which reads them too."""
    phys = hb.Physics(T, nb)
    for seed in range(2):
        st = seeded_state(nb, T, seed)
        other = seeded_state(nb, T, seed + 10)  # ghost rows taken from an unrelated state
        row = int(np.prod([n + 2 for n in nb[1:]]))
        for a, b, nv in zip(st, other, (2, len(nb))):
            k = row * nv
            a[:k] = b[k:2 * k]
            a[-k:] = b[-2 * k:-k]
        ref = (np.zeros_like(st[0]), np.zeros_like(st[1]))
        dtd = phys.dtd(cfl_dt(phys, seed))
        dref = oracle.step(st, ref, phys, dtd)
        cur = to_dev(cuda, st)
        nxt = tuple(cuda.zeros_like(a) for a in cur)
        dt = cuda.zeros(1, dtype=cur[0].dtype, device="cuda")
        if kernel == hb.KERNEL_STRIP and len(nb) == 2 and T is np.float32 and (nb[1] + 2) % 2:
            continue
        _, info = hb.step(cur, nxt, dt, phys, dtd, kernel=kernel, x_ghosts=True, arith="strict")
        assert info.kernel == kernel
        assert phys.dtype(dt.item()).tobytes() == dref.tobytes()
        out = tuple(a.cpu().numpy() for a in nxt)
        assert out[0].tobytes() == ref[0].tobytes() and out[1].tobytes() == ref[1].tobytes()


@pytest.mark.parametrize("T", [np.float64, np.float32])
def test_launch_shapes_bitwise(cuda, oracle, T):
    """Every launch shape the autotuner may pick gives the oracle's bits: 3D tile heights
    (8, 9, 12, 16 rows in FP64; 8, 16 in FP32) with explicit chunks, 2D register budgets
    with 2D chunks."""
    warps = (8, 9, 12, 16) if T is np.float64 else (8, 16)
    alt = 5 if T is np.float64 else 8
    cases = [((40, 150, 130), w, c, 0) for w in warps for c in (0, 7, 64)] + \
            [((9, 14, 62), w, 3, 0) for w in warps] + \
            [((300, 253), 0, c, b) for c in (0, 5, 300) for b in (4, alt)]
    try:
        for nb, w, c, b in cases:
            phys = hb.Physics(T, nb)
            hb.set_launch_shape(len(nb), T, w, c, b)
            st = seeded_state(nb, T, 4)
            oracle.ghost_x(st, nb)
            ref = (np.zeros_like(st[0]), np.zeros_like(st[1]))
            dtd = phys.dtd(cfl_dt(phys, 4))
            dref = oracle.step(st, ref, phys, dtd)
            out, d, info = gpu_step(cuda, st, phys, dtd, hb.KERNEL_STRIP)
            shape = hb.last_launch_shape()
            if len(nb) == 3:
                assert shape["warps"] == w
            elif b:
                assert shape["blocks"] == b
            if c:
                assert shape["chunk"] <= c
            assert d.tobytes() == dref.tobytes(), (nb, w, c, b)
            assert out[0].tobytes() == ref[0].tobytes(), (nb, w, c, b)
            assert out[1].tobytes() == ref[1].tobytes(), (nb, w, c, b)
    finally:
        for dim in (2, 3):
            hb.set_launch_shape(dim, T, 0, 0, 0)

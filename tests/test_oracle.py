"""The oracle (C restatement of the reference path) pinned against the reference:
  - bit for bit against the reference's own kernel.cxx compiled unchanged, over
    seeded states and edge-case shapes (when oracle/_ref was built here);
  - bit for bit against committed golden runs of that kernel (always);
  - against the numbers printed by the reference's hardware runs (tests/golden/
    kat_logs.json): initial mass, initial Dt and the first iterations' t / Dt.
"""
from __future__ import annotations

import hashlib
import subprocess

import numpy as np
import pytest

from conftest import ROOT, load_pkg

hb = load_pkg()


def seeded_state(nb, T, seed):
    """A smooth random positive state in the reference layout, ghosts included."""
    rng = np.random.default_rng(seed)
    ncell = int(np.prod([n + 2 for n in nb]))
    nv = 3 if len(nb) == 3 else 2
    rho = rng.uniform(0.5, 2.0, ncell)
    vel = rng.uniform(-0.5, 0.5, (ncell, nv))
    p = rng.uniform(0.05, 10.0, ncell)
    E = p / 0.4 + 0.5 * rho * (vel ** 2).sum(1)
    rhoE = np.stack([rho, E], 1).reshape(-1).astype(T)
    uvx = (vel * rho[:, None]).reshape(-1).astype(T)
    return rhoE, uvx


def cfl_dt(phys, seed):
    """A stable time step for seeded_state (signal speeds below ~6): CFL 0.05-0.1."""
    return phys.dtype(0.05 * (1 + seed % 2)) * phys.min_spacing / phys.dtype(6)


SHAPES_2D = [(1, 1), (1, 9), (9, 1), (2, 3), (7, 5), (33, 17), (60, 60), (5, 130), (3, 257)]
SHAPES_3D = [(1, 1, 1), (1, 3, 4), (4, 1, 3), (3, 4, 1), (5, 6, 7), (12, 10, 9), (3, 2, 33)]


@pytest.mark.parametrize("T", [np.float64, np.float32])
@pytest.mark.parametrize("nb", SHAPES_2D + SHAPES_3D)
def test_oracle_step_matches_reference_kernel(oracle, orc, nb, T):
    if not orc.available_ref(len(nb), T):
        pytest.skip("oracle/_ref not built (reference sources absent)")
    ref = orc.RefKernel(len(nb), T)
    phys = hb.Physics(T, nb)
    for seed in range(3):
        st = seeded_state(nb, T, seed)
        a = (np.zeros_like(st[0]), np.zeros_like(st[1]))
        b = (np.zeros_like(st[0]), np.zeros_like(st[1]))
        dtd = phys.dtd(cfl_dt(phys, seed))
        d1 = oracle.step(st, a, phys, dtd)
        d2 = ref.step(st, b, phys, dtd)
        assert d1.tobytes() == d2.tobytes()
        assert a[0].tobytes() == b[0].tobytes() and a[1].tobytes() == b[1].tobytes()


@pytest.mark.parametrize("T", [np.float64, np.float32])
def test_oracle_loop_matches_reference_kernel_loop(oracle, orc, T):
    if not orc.available_ref(2, T):
        pytest.skip("oracle/_ref not built (reference sources absent)")
    nb = (24, 19)
    phys = hb.Physics(T, nb)
    st = hb_alloc(nb, T)
    first = oracle.init(st, phys)
    ref = orc.RefKernel(2, T)
    r1 = orc.host_loop(ref.step, st, phys, first, 2.0, 50)
    r2 = oracle.run(nb, T, 2.0, 50)
    assert np.array_equal(np.array(r1[2], T), r2["dt"])
    assert np.array_equal(np.array(r1[1]), r2["t"])
    assert r1[0][0].tobytes() == r2["state"][0].tobytes()


def hb_alloc(nb, T):
    ncell = int(np.prod([n + 2 for n in nb]))
    return (np.zeros(2 * ncell, T), np.zeros((3 if len(nb) == 3 else 2) * ncell, T))


def digest(state):
    h = hashlib.sha256()
    for a in state:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def test_oracle_matches_golden_runs(oracle, orc, ref_runs):
    meta, arrays = ref_runs
    for name, m in meta.items():
        if np.prod(m["nb"]) > 100_000:
            continue  # the 60^3 run is checked on the GPU box (slow on one core here)
        T = np.dtype(m["dtype"]).type
        r = oracle.run(tuple(m["nb"]), T, m["max_t"], m["max_it"])
        assert r["it"] == m["it"], name
        assert np.array_equal(r["t"], arrays[name + "__t"]), name
        assert np.array_equal(r["dt"], arrays[name + "__dt"]), name
        assert orc.interior_digest(r["state"], tuple(m["nb"])) == m["sha256"], name
        assert float(r["first_dt"]) == m["first_dt"], name


def test_oracle_kat_3d_170(oracle, kat):
    """hydro3d/reference_run/res_2000_170_170_170.res: initial mass, initial Dt and the
    first 3 iterations' t / Dt as printed (%.7e, %.2e, %.4e, %.3e)."""
    log = kat["res_2000_170_170_170"]
    r = oracle.run((170, 170, 170), np.float64, log["config"]["max_t"], 3)
    assert "%.7e" % r["mass0"] == log["initial_mass"]
    assert "%.2e" % r["first_dt"] == log["initial_dt"]
    for it in range(3):
        assert "%.4e" % r["t"][it] == log["t"][it]
        assert "%.3e" % r["dt"][it] == log["dt"][it]


def test_oracle_kat_initial_all_runs(oracle, kat):
    """Initial total mass (%.7e) and initial Dt (%.2e) printed by all six hardware runs,
    from the oracle's blast IC. The two-rank runs split X into two subdomains; the global
    state is the same, and the per-rank mass sums agree to the printed digits."""
    for name, log in kat.items():
        cfg = log["config"]
        nb = (cfg["nb_x"], cfg["nb_y"]) + ((cfg["nb_z"],) if "nb_z" in cfg else ())
        phys = hb.Physics(np.float64, nb)
        m, dt = oracle.blast_stats(nb, phys)
        assert "%.7e" % m == log["initial_mass"], name
        assert "%.2e" % dt == log["initial_dt"], name


def test_reference_ic_csv_matches_oracle(oracle, tmp_path):
    """The reference program's iteration-0 CSV (hydro2d/main.cxx:166-235, 6 digits)
    against the oracle's initial condition on an odd grid."""
    exe = ROOT / "oracle" / "_ref" / "hydro.cpu"
    if not exe.exists():
        pytest.skip("oracle/_ref not built")
    subprocess.run([str(exe), "-x", "37", "-y", "23", "-i", "0", "-w", "1"], cwd=tmp_path, check=True,
                   stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
    csv = (tmp_path / "output_0_0.0000.csv").read_text().splitlines()
    assert csv[0] == "x,y,rho,p,u,v"
    nb = (37, 23)
    phys = hb.Physics(np.float64, nb)
    st = hb_alloc(nb, np.float64)
    oracle.init(st, phys)
    r = st[0].reshape(39, 25, 2)
    u = st[1].reshape(39, 25, 2)
    rows = []
    for i in range(37):
        for j in range(23):
            rows.append("%d,%d,%s,%s,%s,%s" % (i, j, g6(r[i + 1, j + 1, 0]), g6(r[i + 1, j + 1, 1]),
                                               g6(u[i + 1, j + 1, 0]), g6(u[i + 1, j + 1, 1])))
    assert csv[1:] == rows


def g6(x):
    """C++ ostream default formatting (%g with 6 significant digits)."""
    return "%g" % x

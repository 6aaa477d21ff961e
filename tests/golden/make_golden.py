"""Generate the golden fixtures under tests/golden/ (run in a tree where the reference
sources and oracle/_ref exist; the fixtures are committed, this script is how they were
made).

kat_logs.json
    Every per-iteration "t=..., Dt=..." pair, the initial total mass, the initial Dt and
    the final "Total density / change in mass" line printed by the reference's six
    hardware runs (hydro2d/reference_run/*.res, hydro3d/reference_run/*.res), with the
    run configuration parsed from the same log header.

ref_runs.npz / ref_runs.json
    States, t and Dt sequences produced by the reference's own kernel.cxx (compiled
    unchanged, strict IEEE order: oracle/_ref/libref*.so) driven by the reference host
    loop restated in oracle/oracle.py:host_loop, from the oracle's blast initial
    condition. Small grids are stored whole; larger ones as SHA-256 digests of the
    final state bytes plus strided samples.
"""
from __future__ import annotations

import hashlib
import json
import os
import re
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT / "oracle"))
import importlib.util  # noqa: E402

spec = importlib.util.spec_from_file_location("hydro_b200", ROOT / "scalable-fpga-hydrodynamics_b200" / "__init__.py")
pkg = importlib.util.module_from_spec(spec)
sys.modules["hydro_b200"] = pkg
spec.loader.exec_module(pkg)
import oracle as orc  # noqa: E402

# the reference checkout: HYDRO_REFERENCE_DIR, else a checkout named `reference` beside
# this repository
REF = Path(os.environ.get("HYDRO_REFERENCE_DIR") or ROOT.parent / "reference")
OUT = Path(__file__).resolve().parent


def parse_res(path: Path):
    txt = path.read_text(errors="replace").splitlines()
    cfg = {}
    for line in txt[:20]:
        m = re.match(r"\s*Spatial Points ([XYZ]) axis .*:\s*(\d+)", line)
        if m:
            cfg["nb_" + m.group(1).lower()] = int(m.group(2))
        m = re.match(r"\s*Max Timestep .*:\s*([0-9.eE+-]+)", line)
        if m:
            cfg["max_t"] = float(m.group(1))
        m = re.match(r"\s*Max iterations .*:\s*(\d+)", line)
        if m:
            cfg["max_it"] = int(m.group(1))
    t, dt = [], []
    mass0 = dt0 = final = None
    for line in txt:
        m = re.match(r"\[it=\s*(\d+)\] hydro_fvm compute time t=(\S+) \(Dt=(\S+)\)", line)
        if m:
            assert int(m.group(1)) == len(t)
            t.append(m.group(2))
            dt.append(m.group(3))
            continue
        m = re.match(r"Initial total mass\s*:\s*(\S+)", line)
        if m:
            mass0 = m.group(1)
        m = re.match(r"Initial Dt : (\S+)", line)
        if m:
            dt0 = m.group(1)
        m = re.match(r"\[it=\s*(\d+)\] t=(\S+) Total density : (\S+), change in mass: (\S+)", line)
        if m:
            final = dict(it=int(m.group(1)), t=m.group(2), mass=m.group(3), change=m.group(4))
    return dict(config=cfg, initial_mass=mass0, initial_dt=dt0, t=t, dt=dt, final=final, source=str(path.relative_to(REF)))


def kat():
    logs = {}
    for p in sorted(REF.glob("hydro*/reference_run/res_*.res")):
        logs[p.stem] = parse_res(p)
    (OUT / "kat_logs.json").write_text(json.dumps(logs, indent=0))
    print("kat:", {k: len(v["t"]) for k, v in logs.items()})


def digest(state):
    h = hashlib.sha256()
    for a in state:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


RUNS = [
    # name, nb, dtype, max_t, max_it, store_whole
    ("s2d_f64_60x60", (60, 60), np.float64, 2.0, 200, True),
    ("s2d_f32_60x60", (60, 60), np.float32, 2.0, 200, True),
    ("odd2d_f64_37x23", (37, 23), np.float64, 2.0, 120, True),
    ("odd2d_f32_37x23", (37, 23), np.float32, 2.0, 120, True),
    ("thin2d_f64_1x17", (1, 17), np.float64, 2.0, 40, True),
    ("thin2d_f64_17x1", (17, 1), np.float64, 2.0, 40, True),
    ("s3d_f64_20x16x12", (20, 16, 12), np.float64, 2.0, 60, True),
    ("s3d_f32_20x16x12", (20, 16, 12), np.float32, 2.0, 60, True),
    ("l3d_f64_60x60x60", (60, 60, 60), np.float64, 2.0, 200, False),
]


def ref_runs():
    o = orc.Oracle()
    arrays, meta = {}, {}
    for name, nb, T, max_t, max_it, whole in RUNS:
        phys = pkg.Physics(T, nb)
        ncell = int(np.prod([n + 2 for n in nb]))
        st = (np.zeros(2 * ncell, T), np.zeros((3 if len(nb) == 3 else 2) * ncell, T))
        first = o.init(st, phys)
        ref = orc.RefKernel(len(nb), T)
        fin, t_log, dt_log = orc.host_loop(ref.step, st, phys, first, max_t, max_it)
        meta[name] = dict(nb=list(nb), dtype=np.dtype(T).name, max_t=max_t, max_it=max_it, it=len(t_log),
                          first_dt=float(first), sha256=orc.interior_digest(fin, nb), mass1=o.mass(fin[0], nb))
        arrays[name + "__t"] = np.array(t_log, np.float64)
        arrays[name + "__dt"] = np.array(dt_log, T)
        if whole:
            arrays[name + "__rhoE"] = fin[0]
            arrays[name + "__uvx"] = fin[1]
        else:
            arrays[name + "__rhoE_sample"] = fin[0][::97].copy()
            arrays[name + "__uvx_sample"] = fin[1][::97].copy()
        print(name, len(t_log), meta[name]["sha256"][:16])
    np.savez_compressed(OUT / "ref_runs.npz", **arrays)
    (OUT / "ref_runs.json").write_text(json.dumps(meta, indent=1))


if __name__ == "__main__":
    kat()
    ref_runs()

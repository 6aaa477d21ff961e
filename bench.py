#!/usr/bin/env python
"""Benchmark of the first-order finite-volume step (the reference's `launcher` path).

Workload at N=1: the 2D blast on a 40000 x 20000 grid in FP64 through the plain path,
one step = one launcher call over the whole grid followed by the host Dt read-back of
the reference loop (hydro2d/main.cxx:734-747). Inputs (51.2 GB double-buffered) are far
larger than L2, so no flush is needed between steps.

  value      whole-job cell-updates/s with the state resident in HBM (CUDA events)
  e2e        the same metric through the C-ABI drop-in `launcher` with the reference
             host loop's per-step traffic: ghost rows host->device from pinned memory,
             launcher, Dt and edge rows device->host (hydro2d/main.cxx:720-763)
  roofline   the strip kernel's algorithmic bytes (64 B per FP64 2D cell-update, the
             reference's own byte model, hydro2d/main.cxx:889) over its event-timed
             duration, against the measured HBM copy bandwidth
  cpu_baseline  the reference's own kernel.cxx (oracle/_ref) on the host cores, on a
             bounded sample of the same workload (rank 0, N=1)
  variants   FP32 2D and FP64/FP32 3D 512^3 plain-path numbers (a few steps each)

`--impl reference` times the reference's CPU kernel alone on the same metric.
`--tour` instead times every kernel of the library on a small case (state above L2
size), one JSON line per kernel with its GB/s against the measured copy bandwidth.
Under torchrun (N>1) each rank runs its own replica (no data-path collective; weak
scaling) and rank 0 prints the max-over-ranks timing.
"""
from __future__ import annotations

import argparse
import ctypes
import importlib.util
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
PKG = ROOT / "scalable-fpga-hydrodynamics_b200"
METRIC = "GCell-upd/s batched FP32 vs plain FP64 @<=1e-5 rel err; p50/p99 latency"
UNIT = "GCell-upd/s"
BYTES_PER_CELL = {(2, 8): 64, (2, 4): 32, (3, 8): 80, (3, 4): 40}


def load_pkg():
    name = "hydro_b200"
    if name in sys.modules:
        return sys.modules[name]
    spec = importlib.util.spec_from_file_location(name, PKG / "__init__.py", submodule_search_locations=[str(PKG)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# ----------------------------------------------------------------------- clocks ---
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: str):
        self.idx = gpu  # nvidia-smi -i accepts an index or a GPU UUID
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.idx), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "50"], stdout=self.f,
                                         stderr=subprocess.DEVNULL)
            # wait (at most 2 s) for its first sample, so that nvidia-smi's start-up does not
            # compete with the host loop of the timed region
            t0 = time.perf_counter()
            while time.perf_counter() - t0 < 2.0 and os.path.getsize(self.path) == 0 and self.proc.poll() is None:
                time.sleep(0.02)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.close()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in Path(self.path).read_text().splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        os.unlink(self.path)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def gpu_uuid(torch, index):
    """The NVML / nvidia-smi name of CUDA device `index` (robust to CUDA_VISIBLE_DEVICES)."""
    try:
        return "GPU-" + str(torch.cuda.get_device_properties(index).uuid)
    except Exception:
        return str(index)


class EnergyMeter:
    """GPU energy from NVML's total-energy counter (millijoules since driver load), read
    before and after a region. Read-only; None where NVML or the counter is missing."""

    def __init__(self, uuid: str):
        self.h = None
        try:
            import pynvml

            pynvml.nvmlInit()
            self.nv = pynvml
            self.h = (pynvml.nvmlDeviceGetHandleByUUID(uuid) if uuid.startswith("GPU-")
                      else pynvml.nvmlDeviceGetHandleByIndex(int(uuid)))
        except Exception:
            self.h = None

    def read(self):
        if self.h is None:
            return None
        try:
            return self.nv.nvmlDeviceGetTotalEnergyConsumption(self.h) / 1e3
        except Exception:
            return None


def energy_entry(joules, seconds, cell_updates):
    if joules is None or seconds <= 0:
        return None
    return dict(joules=joules, avg_w=joules / seconds, nj_per_cell_update=joules / cell_updates * 1e9,
                source="NVML total energy counter around the timed region")


# -------------------------------------------------------------- GPU measurements ---
def bench_resident(hb, torch, nb, T, steps, warmup, kernel=0, meter=None, arith=None):
    """Host loop with the state resident on the device; CUDA events on the launching
    stream: total time of `steps` steps and per-step kernel time (and the energy of the
    timed steps when a meter is given)."""
    run = hb.BlastRun(nb, T, kernel=kernel, arith=arith)
    for _ in range(warmup):
        run.step()
    shape = hb.last_launch_shape()
    torch.cuda.synchronize()
    j0 = meter.read() if meter else None
    stream = torch.cuda.current_stream()
    E = torch.cuda.Event
    e_start, e_end = E(enable_timing=True), E(enable_timing=True)
    per = [(E(enable_timing=True), E(enable_timing=True)) for _ in range(steps)]
    e_start.record(stream)
    for k in range(steps):
        per[k][0].record(stream)
        run.step_kernel_only()
        per[k][1].record(stream)
        run.step_finish()
    e_end.record(stream)
    torch.cuda.synchronize()
    j1 = meter.read() if meter else None
    total_ms = e_start.elapsed_time(e_end)
    kern_ms = [a.elapsed_time(b) for a, b in per]
    info = run.last_info
    # an asynchronous step launches the update kernel and the signal-speed check kernel
    # (which returns at once unless the fused maximum fell under its skip threshold)
    res = dict(total_ms=total_ms, kernel_ms=kern_ms, kernel=int(info.kernel), it=run.it, launches_per_step=2,
               shape=shape,
               energy_j=(j1 - j0) if (j0 is not None and j1 is not None) else None)
    del run
    torch.cuda.empty_cache()
    return res


def bench_e2e(hb, torch, nb, T, steps, warmup):
    """The reference host loop through the drop-in launcher (C ABI): per step, ghost
    rows host->device from pinned memory, launcher, Dt and edge rows device->host."""
    phys = hb.Physics(T, nb)
    tdt = torch.float64 if T is np.float64 else torch.float32
    cur = hb.alloc_state(nb, T)
    nxt = hb.alloc_state(nb, T)
    dt_dev = torch.zeros(1, dtype=tdt, device="cuda")
    dt = hb.init_blast(cur, phys)
    ys = nb[1] + 2
    row = 2 * ys  # elements per row per array
    # host copies of the rows the reference host keeps current: ghost 0, 1, nb_x, ghost nb_x+1
    h_rows = torch.zeros((2, 4, row), dtype=tdt, pin_memory=True)
    h_dt = torch.zeros(1, dtype=tdt, pin_memory=True)
    for a in range(2):
        h_rows[a, 1].copy_(cur[a][row * 1:row * 2])
        h_rows[a, 2].copy_(cur[a][row * nb[0]:row * (nb[0] + 1)])
    stream = torch.cuda.current_stream()
    big = T(1e20)

    def one_step(cur, nxt, dt):
        # host ghost exchange (hydro2d/main.cxx:349-378) then H2D of the ghost rows
        for a in range(2):
            h_rows[a, 0].copy_(h_rows[a, 2])
            h_rows[a, 3].copy_(h_rows[a, 1])
            cur[a][0:row].copy_(h_rows[a, 0], non_blocking=True)
            cur[a][row * (nb[0] + 1):row * (nb[0] + 2)].copy_(h_rows[a, 3], non_blocking=True)
        dtd = phys.dtd(dt)
        us = hb.launcher2d(cur[0], cur[1], nxt[0], nxt[1], dt_dev, phys.C_min, phys.g, phys.gm1, phys.divgamma,
                           phys.k, nb[0], nb[1], dtd[0], dtd[1])
        if us < 0:
            raise RuntimeError(hb.last_error())
        h_dt.copy_(dt_dev, non_blocking=True)
        for a in range(2):
            h_rows[a, 1].copy_(nxt[a][row * 1:row * 2], non_blocking=True)
            h_rows[a, 2].copy_(nxt[a][row * nb[0]:row * (nb[0] + 1)], non_blocking=True)
        stream.synchronize()
        dtn = T(h_dt.item())
        return nxt, cur, (dtn if dtn < big else big)

    for _ in range(warmup):
        cur, nxt, dt = one_step(cur, nxt, dt)
    torch.cuda.synchronize()
    E = torch.cuda.Event
    e0, e1 = E(enable_timing=True), E(enable_timing=True)
    t0 = time.perf_counter()
    e0.record(stream)
    for _ in range(steps):
        cur, nxt, dt = one_step(cur, nxt, dt)
    e1.record(stream)
    torch.cuda.synchronize()
    wall_ms = (time.perf_counter() - t0) * 1e3
    ev_ms = e0.elapsed_time(e1)
    isz = 8 if T is np.float64 else 4
    h2d = 2 * 2 * row * isz
    d2h = isz + 2 * 2 * row * isz
    del cur, nxt
    torch.cuda.empty_cache()
    return dict(ms=max(wall_ms, ev_ms), h2d=h2d, d2h=d2h)


# -------------------------------------------------------------- CPU (reference) ---
def cpu_threads():
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def cpu_flags():
    try:
        for line in Path("/proc/cpuinfo").read_text().splitlines():
            if line.startswith("flags"):
                return set(line.split(":", 1)[1].split())
    except Exception:
        pass
    return set()


def has_avx2_fma():
    f = cpu_flags()
    return {"avx2", "fma", "bmi2"} <= f


def has_avx512():
    """The x86-64-v4 level: AVX-512 F, BW, CD, DQ and VL."""
    return {"avx512f", "avx512bw", "avx512cd", "avx512dq", "avx512vl"} <= cpu_flags()


def cpu_reference_sample(nb_y: int, rows: int, seconds: float, threads: int):
    """The reference's own kernel.cxx (oracle/_ref, FMA-contracting build as in the
    reference Makefile, at the highest instruction-set level the host supports) on
    `threads` host threads, each stepping its own rows x nb_y
    slab of the blast (the reference's X-slab decomposition, one slab per core) for
    about `seconds`. Falls back to the oracle restatement when oracle/_ref is absent.
    Returns (cell-updates/s, kind, description, timed seconds)."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle as orc

    hb = load_pkg()
    T = np.float64
    nb = (rows, nb_y)
    phys = hb.Physics(T, (40000, nb_y))  # the full workload's constants
    phys.nb = nb
    o = orc.Oracle()
    kind = "reference"
    if orc.available_ref(2, T, fast=True, level="v4") and has_avx512():
        stepper = orc.RefKernel(2, T, fast=True, level="v4").step
        what = "oracle/_ref/libref2d_f64_fast_v4.so (reference kernel.cxx, -O2 -march=x86-64-v4)"
    elif orc.available_ref(2, T, fast=True) and has_avx2_fma():
        stepper = orc.RefKernel(2, T, fast=True).step
        what = "oracle/_ref/libref2d_f64_fast.so (reference kernel.cxx, -O2 -march=x86-64-v3)"
    elif orc.available_ref(2, T):
        stepper = orc.RefKernel(2, T).step
        what = "oracle/_ref/libref2d_f64.so (reference kernel.cxx, -O2 -ffp-contract=off)"
    else:
        stepper = o.step
        kind = "port"
        what = "oracle/liboracle.so (C restatement)"
    threading.stack_size(64 << 20)  # the reference kernel keeps a 2 MB line buffer on the stack
    dtd = phys.dtd(T(5e-6))
    counts = [0] * threads
    stop = threading.Event()

    def work(tid):
        ncell = (rows + 2) * (nb_y + 2)
        a = (np.zeros(2 * ncell, T), np.zeros(2 * ncell, T))
        b = (np.zeros(2 * ncell, T), np.zeros(2 * ncell, T))
        o.init(a, phys)
        stepper(a, b, phys, dtd)  # warm-up
        while not stop.is_set():
            orc.ghost_x_numpy(a, nb)
            stepper(a, b, phys, dtd)
            a, b = b, a
            counts[tid] += 1

    ths = [threading.Thread(target=work, args=(i,)) for i in range(threads)]
    for th in ths:
        th.start()
    time.sleep(0.5)
    c0 = sum(counts)
    t0 = time.perf_counter()
    time.sleep(seconds)
    c1 = sum(counts)
    t1 = time.perf_counter()
    stop.set()
    for th in ths:
        th.join()
    cells = (c1 - c0) * rows * nb_y
    return cells / (t1 - t0), kind, what, t1 - t0


# --------------------------------------------------------------- batched / serving ---
def bench_batched(hb, torch, n=256, steps=200, seed=0, plain_sample=None, chunk=0, log=print, meter=None):
    """The batched workload (256 seeded 2D blasts, sides log-uniform in [64, 2048], 200
    steps each) through the FP32 batch engine in fused and in strict arithmetic and the FP64
    engine in strict arithmetic (chunk from the autotuner), and the same instances one at a
    time through the plain FP64 path. Accuracy: each FP32 run against the FP64 batch
    (bit-identical to the plain FP64 path) on every instance. `chunk` > 0 fixes the rows per
    work item instead of asking the autotuner."""
    from hydro_b200.autotune import tune
    from hydro_b200.batch import Batch
    from hydro_b200.workloads import batch_blasts

    out = {}
    blasts = batch_blasts(n, seed=seed, steps=steps)
    cells = sum(int(np.prod(b.nb)) for b in blasts)
    states = {}
    for T, ar in ((np.float32, "fused"), (np.float32, "strict"), (np.float64, "strict")):
        ck = chunk if chunk > 0 else tune(2, T, log=log)
        s = torch.cuda.Stream()
        # warm-up: a throw-away batch of the same instances runs a few steps
        w = Batch(2, T, chunk=ck, capacity=n, stream=s, arith=ar)
        for bl in blasts[:32]:
            w.add(bl)
        w.run(3)
        w.close()
        b = Batch(2, T, chunk=ck, capacity=n, stream=s, arith=ar)
        slots = [b.add(bl) for bl in blasts]
        b.prepare(steps)  # graph captured and instantiated outside the timed region
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        j0 = meter.read() if meter else None
        t0 = time.perf_counter()
        e0.record(s)
        b.run(steps, sync=False)
        e1.record(s)
        b.sync()
        wall = time.perf_counter() - t0
        j1 = meter.read() if meter else None
        ms = e0.elapsed_time(e1)
        done = sum(b.status(k)["steps"] for k in slots)
        assert done == n * steps, (done, n * steps)
        key = ("fp32" if T is np.float32 else "fp64") + ("_fused" if ar == "fused" else "")
        out[f"batched_{key}"] = dict(arith=ar, value=cells * steps / (ms / 1e3) / 1e9, unit=UNIT, ms=ms, wall_s=wall,
                                     chunk=ck, instances=n, steps=steps, cells=cells,
                                     bytes_per_cell=32 if T is np.float32 else 64,
                                     energy=energy_entry(None if j0 is None or j1 is None else j1 - j0, wall,
                                                         cells * steps))
        states[key] = [b.state(k)[0] for k in slots]
        b.close()
    # accuracy of the FP32 batch against FP64 (rho, relative L1 and L-inf per instance)
    for key in ("fp32", "fp32_fused"):
        l1, linf = [], []
        for a, r, bl in zip(states[key], states["fp64"], blasts):
            sh = tuple(x + 2 for x in bl.nb) + (2,)
            inner = tuple(slice(1, x + 1) for x in bl.nb)
            ra = a.reshape(sh)[inner][..., 0].astype(np.float64)
            rr = r.reshape(sh)[inner][..., 0]
            l1.append(np.abs(ra - rr).sum() / np.abs(rr).sum())
            linf.append(np.abs(ra - rr).max() / np.abs(rr).max())
        out[f"batched_{key}"]["rho_rel_l1_vs_fp64_max"] = float(max(l1))
        out[f"batched_{key}"]["rho_rel_linf_vs_fp64_max"] = float(max(linf))
    # plain FP64 path, one instance at a time (the reference host loop per instance)
    sample = blasts if plain_sample is None else blasts[:plain_sample]
    pcells = sum(int(np.prod(b.nb)) for b in sample)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for bl in sample:
        hb.BlastRun(bl.nb, np.float64, blast=bl).run(float("inf"), steps)
    torch.cuda.synchronize()
    pw = time.perf_counter() - t0
    out["plain_fp64_one_at_a_time"] = dict(value=pcells * steps / pw / 1e9, unit=UNIT, wall_s=pw,
                                           instances=len(sample), steps=steps)
    out["batched_fp32_over_plain_fp64"] = out["batched_fp32"]["value"] / out["plain_fp64_one_at_a_time"]["value"]
    out["batched_fp32_fused_over_plain_fp64"] = (out["batched_fp32_fused"]["value"]
                                                 / out["plain_fp64_one_at_a_time"]["value"])
    return out


def bench_serving(hb, torch, rates=(10.0, 100.0, 1000.0), nreq=8, seed=0, max_wall=20.0, plain=True, log=print):
    """The serving workload: Poisson streams of mixed requests (70% 2D sides [128, 4096],
    30% 3D sides [32, 256], t_end in [0.05, 0.5] of the sound-crossing time, FP32/FP64 50/50),
    `nreq` requests per rate, through the continuous-batching server (150 GB budget) and
    through the plain path one request at a time, each request in its own precision. At the
    highest rate the same stream also runs all-FP32 through the server against all-FP64
    through the plain path. Each run is capped at `max_wall` seconds: latency percentiles
    cover the completed requests, throughput all the cell-updates done within the run."""
    from hydro_b200.autotune import best_chunk
    from hydro_b200.serving import Server, serve_plain, summarize
    from hydro_b200.workloads import request_stream

    def served(reqs, dtype=None):
        srv = Server(hbm_budget=150e9, steps_per_tick=8, chunk2d=best_chunk(2, np.float32),
                     chunk3d=best_chunk(3, np.float32), arith={np.float32: "fused"})
        recs, wall = srv.serve(reqs, max_wall=max_wall, dtype=dtype)
        srv.close()
        torch.cuda.empty_cache()
        return summarize(recs, wall)

    def plain_path(reqs, dtype=None):
        recs, wall = serve_plain(reqs, max_wall=max_wall, dtype=dtype)
        torch.cuda.empty_cache()
        return summarize(recs, wall)

    res = {}
    for rate in rates:
        reqs = request_stream(rate, seed=seed, count=nreq)
        entry = dict(batched=served(reqs))
        if plain:
            entry["plain_one_at_a_time"] = plain_path(reqs)
            entry["batched_over_plain"] = entry["batched"]["gcell_s"] / max(entry["plain_one_at_a_time"]["gcell_s"],
                                                                            1e-30)
        if plain and rate == max(rates):
            entry["batched_fp32"] = served(reqs, np.float32)
            entry["plain_fp64"] = plain_path(reqs, np.float64)
            entry["batched_fp32_over_plain_fp64"] = entry["batched_fp32"]["gcell_s"] / max(
                entry["plain_fp64"]["gcell_s"], 1e-30)
        res[f"rate_{rate:g}"] = entry
        log(f"serving rate {rate:g}/s: {json.dumps(entry)}")
    return res


# ------------------------------------------------------------ FP32 vs FP64 accuracy ---
def accuracy_vs_strict_fp64(hb, torch, nb, steps=100, variants=(("fp32_strict", np.float32, "strict"),
                                                                  ("fp32_fused", np.float32, "fused"),
                                                                  ("fp64_fused", np.float64, "fused"))):
    """The plain path from the same blast for `steps` iterations in strict FP64 (bit-identical
    to the reference's FP64 kernel: the GPU parity tests) and in each variant; per variant
    and field (rho, p and the velocities) the relative L1 (sum |a - b| / sum |b|), the
    relative L-infinity (max |a - b| / max |b|) and the max pointwise relative error with
    the denominator floored at 1e-12 max |b| (max |a - b| / max(|b|, 1e-12 max |b|))."""
    ref = hb.BlastRun(nb, np.float64, arith="strict").run(float("inf"), steps)
    out = dict(steps=steps, grid="x".join(map(str, nb)),
               reference="strict FP64 plain path (bit-identical to the oracle)")
    for name, T, arith in variants:
        r = hb.BlastRun(nb, T, arith=arith).run(float("inf"), steps)
        out[name] = _field_errors(torch, nb, r, ref)
        out[name]["same_iterations"] = r.it == ref.it
        del r
        torch.cuda.empty_cache()
    del ref
    torch.cuda.empty_cache()
    return out


def _field_errors(torch, nb, run, ref):
    """Errors of run's final state against ref's, field by field, on the device in chunks."""
    dim = len(nb)
    runs = {"a": run, "b": ref}
    gm1 = 0.4
    out = {}
    names = ["rho", "p", "u", "v", "w"][:dim + 2]
    # sum|d|, sum|b|, max|d|, max|b|, and per chunk the floored ratio needs max|b| first:
    # two passes (the first for max|b|)
    acc = {n: [0.0, 0.0, 0.0, 0.0, 0.0] for n in names}
    nplane = int(np.prod([n + 2 for n in nb[1:]]))
    inner = tuple(slice(1, n + 1) for n in nb[1:])
    nv = dim
    rows = max(1, int(1e8 // nplane))

    def chunks():
        for i0 in range(1, nb[0] + 1, rows):
            i1 = min(nb[0] + 1, i0 + rows)
            fields = {}
            for key, r in runs.items():
                rhoE = r.cur[0][2 * nplane * i0:2 * nplane * i1].double().view(i1 - i0, *[n + 2 for n in nb[1:]], 2)
                mom = r.cur[1][nv * nplane * i0:nv * nplane * i1].double().view(i1 - i0, *[n + 2 for n in nb[1:]],
                                                                               nv)
                rho = rhoE[(slice(None),) + inner + (0,)]
                E = rhoE[(slice(None),) + inner + (1,)]
                m = mom[(slice(None),) + inner]
                vel = m / rho.unsqueeze(-1)
                p = gm1 * (E - 0.5 * (m * vel).sum(-1))
                fields[key] = [rho, p] + [vel[..., c] for c in range(nv)]
            yield fields

    for fields in chunks():
        for n, a, b in zip(names, fields["a"], fields["b"]):
            d = (a - b).abs()
            acc[n][0] += float(d.sum())
            acc[n][1] += float(b.abs().sum())
            acc[n][2] = max(acc[n][2], float(d.max()))
            acc[n][3] = max(acc[n][3], float(b.abs().max()))
    for fields in chunks():
        for n, a, b in zip(names, fields["a"], fields["b"]):
            den = b.abs().clamp(min=1e-12 * acc[n][3]) if acc[n][3] > 0 else b.abs() + 1.0
            acc[n][4] = max(acc[n][4], float(((a - b).abs() / den).max()))
    for n, (sd, sb, md, mb, mr) in acc.items():
        out[n] = dict(rel_l1=sd / sb if sb > 0 else 0.0, rel_linf=md / mb if mb > 0 else 0.0, max_rel_floored=mr)
    return out


def config_for(nb, T):
    """The workload description both arms print (identical dicts)."""
    dim = len(nb)
    isz = np.dtype(T).itemsize
    bpc = BYTES_PER_CELL[(dim, isz)]
    cells = int(np.prod(nb))
    return dict(workload=(f"{dim}D blast {'x'.join(map(str, nb))} {'FP64' if isz == 8 else 'FP32'}, "
                          f"plain path (one launcher call per step)"),
                nb=list(nb), bytes_per_cell_update=bpc,
                l2=f"inputs larger than L2 ({cells * bpc / 2 / 1e9:.1f} GB state, 126 MB L2): no flush",
                parallelism="replicas: one per GPU, no data-path collective")


def bench_serving_sweep(hb, torch, rates=(10.0, 30.0, 100.0, 300.0, 1000.0), nreq=200, seed=0, plain=True,
                        bound_requests=2000, bound_wall=240.0, max_wall=None, trace_path=None, log=print):
    """The serving workload as configured: at each rate a seeded Poisson stream of `nreq`
    mixed requests (each in its own precision) through the continuous-batching server
    (150 GB budget) and, when `plain`, through the plain path one request at a time; then
    one stream of `bound_requests` at the highest rate, whose states together exceed the
    150 GB budget, through the server alone for at most `bound_wall` seconds (requests queue
    for memory; latency covers the requests completed by then). The trace of every
    stream (arrival, grid, blast parameters, t_end, precision) goes to `trace_path`."""
    from hydro_b200.autotune import best_chunk
    from hydro_b200.serving import Server, serve_plain, summarize
    from hydro_b200.workloads import request_stream

    def served(reqs, budget=150e9, wall_cap=max_wall):
        srv = Server(hbm_budget=budget, steps_per_tick=8, chunk2d=best_chunk(2, np.float32),
                     chunk3d=best_chunk(3, np.float32), arith={np.float32: "fused"})
        recs, wall = srv.serve(reqs, max_wall=wall_cap)
        stats = dict(srv.stats)
        srv.close()
        torch.cuda.empty_cache()
        out = summarize(recs, wall)
        out["budget"] = stats
        return out

    def trace(reqs):
        return [dict(rid=r.rid, arrival=r.arrival, nb=list(r.blast.nb), centre=list(r.blast.centre),
                     radius=r.blast.radius, p_in=r.blast.p_in, p_out=r.blast.p_out, t_end=r.blast.t_end,
                     dtype=np.dtype(r.dtype).name) for r in reqs]

    res, traces = {}, {}
    for rate in rates:
        reqs = request_stream(rate, seed=seed, count=nreq)
        traces[f"rate_{rate:g}"] = trace(reqs)
        entry = dict(batched=served(reqs))
        if plain:
            recs, wall = serve_plain(reqs, max_wall=max_wall)
            torch.cuda.empty_cache()
            entry["plain_one_at_a_time"] = summarize(recs, wall)
            entry["batched_over_plain"] = entry["batched"]["gcell_s"] / max(
                entry["plain_one_at_a_time"]["gcell_s"], 1e-30)
        res[f"rate_{rate:g}"] = entry
        log(f"serving sweep rate {rate:g}/s: {json.dumps(entry)}")
    if bound_requests:
        rate = max(rates)
        reqs = request_stream(rate, seed=seed + 1, count=bound_requests)
        traces[f"budget_bound_rate_{rate:g}"] = trace(reqs)
        # double-buffered states with ghosts (rows the engines pad to 16 bytes not counted)
        need = sum(2 * int(np.prod([n + 2 for n in r.blast.nb])) * (2 + len(r.blast.nb)) * np.dtype(r.dtype).itemsize
                   for r in reqs)
        entry = dict(batched=served(reqs, wall_cap=bound_wall), total_state_bytes=need)
        res[f"budget_bound_rate_{rate:g}"] = entry
        log(f"serving budget-bound run: {json.dumps(entry)}")
    if trace_path:
        Path(trace_path).write_text(json.dumps(dict(seed=seed, streams=traces)))
    return res


# ------------------------------------------------------------------- kernel tour ---
def bench_tour(hb, torch, hbm, reps=5, log=print, only=None):
    """Every kernel of the library on a case whose state is larger than L2 (126 MB), timed
    with CUDA events on the launching stream: one JSON line per entry with the algorithmic
    bytes of one call, its duration, GB/s and the fraction of the measured copy bandwidth.
    Pair it with an `ncu --metrics gpu__time_duration.sum,dram__bytes_read.sum,...` launch
    list of the same command for the DRAM bytes each kernel moves."""
    from hydro_b200.autotune import _blasts
    from hydro_b200.batch import Batch

    lines = []
    E = torch.cuda.Event

    def timed(name, fn, nbytes, note="", stream=None):
        if only and only not in name.replace(" ", "_"):
            return
        st = stream or torch.cuda.current_stream()
        for _ in range(2):
            fn()
        torch.cuda.synchronize()
        ms = []
        for _ in range(reps):
            a, b = E(enable_timing=True), E(enable_timing=True)
            a.record(st)
            fn()
            b.record(st)
            b.synchronize()
            ms.append(a.elapsed_time(b))
        m = statistics.median(ms)
        gbs = nbytes / (m / 1e3) / 1e9
        line = dict(tour=name, ms=m, bytes=int(nbytes), gb_s=gbs, frac=gbs / hbm, note=note)
        lines.append(line)
        log(json.dumps(line))

    nb2, nb3 = (4000, 2000), (256, 256, 256)
    for T, tn in ((np.float64, "double"), (np.float32, "float")):
        isz = np.dtype(T).itemsize
        # initial condition: writes every cell of both arrays (ghosts included)
        for nb in (nb2, nb3):
            d = len(nb)
            phys = hb.Physics(T, nb)
            st = hb.alloc_state(nb, T)
            allc = int(np.prod([n + 2 for n in nb]))
            timed(f"init{d}d_kernel<{tn}> {'x'.join(map(str, nb))}", lambda: hb.init_blast(st, phys),
                  allc * (2 + d) * isz, "writes all cells of both arrays; first Dt fused")
            cells = int(np.prod(nb))
            timed(f"mass_kernel<{tn}> {'x'.join(map(str, nb))}", lambda: hb.mass(st[0], nb), cells * 2 * isz,
                  "rho of the (rho, E) pairs: whole 32-byte sectors hold both")
            # the one-thread-per-cell kernel (every face from both sides, as the reference)
            nx = hb.alloc_state(nb, T)
            dtd = phys.dtd(T(1e-5))
            dt = torch.zeros(1, dtype=st[0].dtype, device="cuda")
            timed(f"direct{d}d<{tn}> {'x'.join(map(str, nb))}",
                  lambda: hb.step(st, nx, dt, phys, dtd, kernel=hb.KERNEL_DIRECT, sync=False),
                  cells * 2 * (2 + d) * isz, "plus the redo2d/redo3d launch, which returns at once")
            # the strip kernels in both arithmetics (built-in launch shape)
            for ar in ("strict", "fused"):
                timed(f"strip{d}d<{tn}> {ar} {'x'.join(map(str, nb))}",
                      lambda: hb.step(st, nx, dt, phys, dtd, kernel=hb.KERNEL_STRIP, sync=False, arith=ar),
                      cells * 2 * (2 + d) * isz, "plus the redo launch, which returns at once")
            del st, nx
            torch.cuda.empty_cache()
        # the exact signal-speed pass: a calm state stepped after a fast one on the same
        # Dt_next and grid skips every cell, so the redo pass recomputes the maximum
        phys = hb.Physics(T, nb2)
        fast, calm, nx = hb.alloc_state(nb2, T), hb.alloc_state(nb2, T), hb.alloc_state(nb2, T)
        hb.init_blast(fast, phys)
        hb.init_blast(calm, phys)
        fast[0][1::2] *= 50.0
        dtd = phys.dtd(T(1e-6))
        dt = torch.zeros(1, dtype=fast[0].dtype, device="cuda")

        def forced():
            hb.step(fast, nx, dt, phys, dtd, kernel=hb.KERNEL_STRIP, sync=False)
            hb.step(calm, nx, dt, phys, dtd, kernel=hb.KERNEL_STRIP, sync=False)

        cells = int(np.prod(nb2))
        timed(f"strip2d<{tn}> x2 + redo2d<{tn}> (forced) 4000x2000", forced, cells * (2 * 8 + 4) * isz,
              "two steps (2 x 64 or 32 B per cell) and one redo pass reading the new state")
        del fast, calm, nx
        torch.cuda.empty_cache()
        # batched engines: a run of 4 steps plus the conservation sums, as one graph
        for d, n in ((2, 64), (3, 48)):
            blasts = _blasts(d, n, 3)
            s = torch.cuda.Stream()
            b = Batch(d, T, capacity=n, stream=s)
            for bl in blasts:
                b.add(bl)
            cells = sum(int(np.prod(bl.nb)) for bl in blasts)
            timed(f"batch{d}d<{tn}> x4 + batch_sums ({n} instances, {cells / 1e6:.1f} M cells)",
                  lambda: b.run(4, sync=False), cells * (4 * 2 * (2 + d) + (2 + d)) * isz,
                  "4 steps and one conservation-sum pass", stream=s)
            b.close()
            torch.cuda.empty_cache()
    # CSV output on the GPU: state in, text out (the file write overlaps the next chunk)
    nbc = (2000, 1000)
    for T in (np.float64,):
        phys = hb.Physics(T, nbc)
        st = hb.alloc_state(nbc, T)
        hb.init_blast(st, phys)
        with tempfile.TemporaryDirectory() as td:
            out = Path(td) / "tour.csv"
            nbytes = hb.write_csv(st, nbc, out)
            timed("write_csv (format_lines + compact_lines + fwrite) 2000x1000 FP64",
                  lambda: hb.write_csv(st, nbc, out), int(np.prod(nbc)) * 4 * 8 + nbytes,
                  f"state read plus {nbytes / 1e6:.0f} MB of text written to a file")
        del st
        torch.cuda.empty_cache()
    return lines


# ------------------------------------------------------------------------ main ---
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--nb", type=int, nargs="+", default=[40000, 20000],
                    help="grid: NB_X NB_Y for 2D cases, NB_X NB_Y NB_Z for 3D cases")
    ap.add_argument("--case", default="2d_f64", choices=["2d_f64", "2d_f32", "3d_f64", "3d_f32"],
                    help="plain-path case timed as the headline (profiling runs pick one)")
    ap.add_argument("--no-variants", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-batched", action="store_true")
    ap.add_argument("--batched-instances", type=int, default=256)
    ap.add_argument("--batched-steps", type=int, default=200)
    ap.add_argument("--batched-chunk", type=int, default=0, help="rows per work item (0: autotuned)")
    ap.add_argument("--arith", default="strict", choices=["strict", "fused"],
                    help="arithmetic of the headline plain-path case (the variants time both)")
    ap.add_argument("--no-tune", action="store_true", help="built-in launch shapes (no plain-path autotuning)")
    ap.add_argument("--no-accuracy", action="store_true")
    ap.add_argument("--accuracy-steps", type=int, default=100,
                    help="iterations of the FP32-vs-FP64 accuracy runs on the large grids")
    ap.add_argument("--no-serving", action="store_true")
    ap.add_argument("--serving-rates", type=float, nargs="+", default=[1000.0],
                    help="request rates (the default run: one rate; --serving-sweep: pass 10 30 100 300 1000)")
    ap.add_argument("--serving-requests", type=int, default=16)
    ap.add_argument("--serving-wall", type=float, default=40.0, help="cap per serving run, seconds")
    ap.add_argument("--no-serving-plain", action="store_true")
    ap.add_argument("--serving-sweep", action="store_true",
                    help="the serving workload as configured (rates 10..1000/s, 200 requests each, plus a "
                         "budget-bound stream) instead of the plain-path benchmark; one JSON line")
    ap.add_argument("--serving-trace", default=None, help="file for the sweep's request traces")
    ap.add_argument("--serving-bound-requests", type=int, default=2000,
                    help="requests of the sweep's budget-bound stream (0: none)")
    ap.add_argument("--tour-only", default=None,
                    help="with --tour: only the entries whose name (spaces as underscores) contains this")
    ap.add_argument("--tour", action="store_true",
                    help="time every kernel of the library on a small case (one JSON line each) and exit")
    args = ap.parse_args()

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dim = int(args.case[0])
    Tcase = np.float64 if args.case.endswith("f64") else np.float32
    nb = tuple(args.nb) if len(args.nb) == dim else ((512, 512, 512) if dim == 3 else (40000, 20000))

    if args.impl == "reference":
        if rank != 0:
            return
        if dim != 2 or Tcase is not np.float64:
            print(json.dumps(dict(impl="reference", unavailable="the CPU reference arm times the 2D FP64 case")))
            return
        thr = cpu_threads()
        rows = 32
        per_step, secs = [], []
        for k in range(args.warmup + args.steps):
            rate, kind, what, el = cpu_reference_sample(nb[1], rows, 2.0 if k >= args.warmup else 0.5, thr)
            if k >= args.warmup:
                per_step.append(rate)
                secs.append(el)
        rate = statistics.median(per_step)
        v = rate / 1e9
        timed = sum(secs)
        sample = (f"{thr} threads x {rows}x{nb[1]} slabs of the blast, ~2 s per step ({what}); "
                  f"value = the sample's cell-updates/s")
        line = dict(metric=METRIC, value=v, unit=UNIT, n_gpus=args.gpus, steps=args.steps, warmup=args.warmup,
                    ms_per_step=timed / args.steps * 1e3, higher_is_better=True, scaling="weak", vs_baseline=None,
                    dtype="f64", data="synthetic (reference blast IC)", impl="reference",
                    config=config_for(nb, Tcase),
                    extrapolated=dict(value=True, timed_region_s=timed,
                                      sample_cells_per_step=thr * rows * nb[1],
                                      full_grid_ms_per_step_at_this_rate=int(np.prod(nb)) / rate * 1e3,
                                      note="each timed step is a ~2 s sample of the workload on every host "
                                           "core; a full-grid step is not run"),
                    cpu_baseline=dict(value=v, unit=UNIT, cores=thr, kind=kind, sample=sample),
                    e2e=dict(value=v, unit=UNIT, h2d_bytes_per_step=0, d2h_bytes_per_step=0))
        print(json.dumps(line), flush=True)
        return

    # the timed GPU runs of the full-size workload take at least 3 warm-up steps
    assert args.warmup >= 3 or args.nb != [40000, 20000] or args.tour, "at least 3 warm-up steps"
    import torch

    hb = load_pkg()
    hb.build()
    torch.cuda.set_device(local)
    from hydro_b200.replicas import Replicas

    reps = Replicas("nccl", timeout_s=300)
    max_over_ranks, barrier = reps.max_over_ranks, reps.barrier

    hbm, peak_kind = peaks()
    if args.serving_sweep:
        if rank == 0:
            sw = bench_serving_sweep(hb, torch, rates=tuple(args.serving_rates), nreq=args.serving_requests,
                                     plain=not args.no_serving_plain, trace_path=args.serving_trace,
                                     bound_requests=args.serving_bound_requests,
                                     log=lambda m: print(m, file=sys.stderr, flush=True))
            print(json.dumps(dict(serving_sweep=sw)), flush=True)
        reps.barrier()
        reps.close()
        return
    if args.tour:
        if rank == 0:
            bench_tour(hb, torch, hbm, log=lambda m: print(m, flush=True), only=args.tour_only)
        reps.barrier()
        reps.close()
        return
    cells = int(np.prod(nb))
    isz = np.dtype(Tcase).itemsize
    bpc = BYTES_PER_CELL[(dim, isz)]
    kname = f"strip{dim}d<{'double' if isz == 8 else 'float'}>"

    tuned = {}
    log = lambda msg: print(msg, file=sys.stderr, flush=True)

    def tune(vnb, T, ar):
        # the launch shape of the plain path for (dim, precision, arithmetic), timed on this
        # grid once (untimed here) and cached on the machine
        if args.no_tune:
            return None
        from hydro_b200.autotune import tune_plain

        key = f"{len(vnb)}d_{np.dtype(T).name}_{ar}"
        if key not in tuned:
            tuned[key] = tune_plain(vnb, T, ar, log=log)
        hb.set_launch_shape(len(vnb), T, tuned[key]["warps"], tuned[key]["chunk"], tuned[key].get("blocks", 0))
        return tuned[key]

    tune(nb, Tcase, args.arith)
    barrier()
    uuid = gpu_uuid(torch, local)
    meter = EnergyMeter(uuid)
    sampler = ClockSampler(uuid)
    sampler.start()
    r = bench_resident(hb, torch, nb, Tcase, args.steps, args.warmup, meter=meter, arith=args.arith)
    clocks = sampler.stop()
    barrier()
    total_ms = max_over_ranks(r["total_ms"])
    ms_step = total_ms / args.steps
    value = world * cells * args.steps / (total_ms / 1e3) / 1e9
    kern_ms = statistics.mean(r["kernel_ms"])
    achieved = cells * bpc / (kern_ms / 1e3) / 1e9
    roofline = dict(bound="hbm", achieved=achieved, peak=hbm, unit="GB/s", frac=achieved / hbm,
                    peak_kind=peak_kind, traffic=None, kernel=kname, bytes_per_cell=bpc, kernel_ms=kern_ms,
                    kernel_ms_median=statistics.median(r["kernel_ms"]), kernel_ms_min=min(r["kernel_ms"]),
                    kernel_ms_max=max(r["kernel_ms"]), frac_of_nominal_8tbs=achieved / 8000.0,
                    arith=args.arith, launch_shape=r["shape"])
    tp = ROOT / "profiles" / "traffic.json"
    if tp.exists():
        tr = json.loads(tp.read_text()).get(f"{kname}_dram_bytes_per_cell")
        if tr:
            roofline["traffic"] = tr * cells

    e2e = None
    if not args.no_e2e and dim == 2:
        barrier()
        e = bench_e2e(hb, torch, nb, Tcase, max(3, args.steps // 3), 2)
        barrier()
        e_ms = max_over_ranks(e["ms"])
        nst = max(3, args.steps // 3)
        e2e = dict(value=world * cells * nst / (e_ms / 1e3) / 1e9, unit=UNIT, h2d_bytes_per_step=e["h2d"],
                   d2h_bytes_per_step=e["d2h"], path="drop-in launcher (C ABI) + reference host-loop copies")

    variants = {}
    if not args.no_variants and args.case == "2d_f64":
        n3 = (512, 512, 512)
        other = "fused" if args.arith == "strict" else "strict"
        for name, vnb, T, ar in ((f"2d_f64_40000x20000_{other}", nb, np.float64, other),
                                 ("2d_f32_40000x20000_strict", nb, np.float32, "strict"),
                                 ("2d_f32_40000x20000_fused", nb, np.float32, "fused"),
                                 ("3d_f64_512^3_strict", n3, np.float64, "strict"),
                                 ("3d_f64_512^3_fused", n3, np.float64, "fused"),
                                 ("3d_f32_512^3_strict", n3, np.float32, "strict"),
                                 ("3d_f32_512^3_fused", n3, np.float32, "fused")):
            tune(vnb, T, ar)
            barrier()
            vsampler = ClockSampler(uuid)
            vsampler.start()
            vr = bench_resident(hb, torch, vnb, T, max(10, args.steps // 2), 3, arith=ar)
            vclocks = vsampler.stop()
            barrier()
            vms = max_over_ranks(vr["total_ms"])
            nst = max(10, args.steps // 2)
            vc = int(np.prod(vnb))
            km = statistics.mean(vr["kernel_ms"])
            vbpc = BYTES_PER_CELL[(len(vnb), np.dtype(T).itemsize)]
            variants[name] = dict(value=world * vc * nst / (vms / 1e3) / 1e9, unit=UNIT,
                                  kernel_gbs=vc * vbpc / (km / 1e3) / 1e9, frac=vc * vbpc / (km / 1e3) / 1e9 / hbm,
                                  kernel=int(vr["kernel"]), ms_per_step=vms / nst, clocks=vclocks,
                                  kernel_ms_median=statistics.median(vr["kernel_ms"]),
                                  kernel_ms_spread=max(vr["kernel_ms"]) - min(vr["kernel_ms"]),
                                  launch_shape=vr["shape"])

    accuracy = {}
    if rank == 0 and world == 1 and not args.no_accuracy and args.case == "2d_f64":
        # FP32 and fused FP64 against strict FP64 on the large grids, 100 iterations each
        for name, vnb in (("2d_40000x20000", nb), ("3d_512^3", (512, 512, 512))):
            accuracy[name] = accuracy_vs_strict_fp64(hb, torch, vnb, steps=args.accuracy_steps)

    batched = serving = None
    if rank == 0 and world == 1 and not args.no_batched and args.case == "2d_f64":
        barrier()
        batched = bench_batched(hb, torch, n=args.batched_instances, steps=args.batched_steps,
                                chunk=args.batched_chunk, log=log, meter=meter)
        torch.cuda.empty_cache()
    if rank == 0 and world == 1 and not args.no_serving and args.case == "2d_f64":
        serving = bench_serving(hb, torch, rates=tuple(args.serving_rates), nreq=args.serving_requests,
                                max_wall=args.serving_wall, plain=not args.no_serving_plain, log=log)
        torch.cuda.empty_cache()

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline and dim == 2:
        thr = cpu_threads()
        rate, kind, what, _el = cpu_reference_sample(nb[1], 32, 3.0, thr)
        cpu = dict(value=rate / 1e9, unit=UNIT, cores=thr, kind=kind,
                   sample=f"{thr} threads x 32x{nb[1]} slabs of the blast for 3 s ({what})")

    if rank == 0:
        line = dict(metric=METRIC, value=value, unit=UNIT, n_gpus=world, steps=args.steps, warmup=args.warmup,
                    ms_per_step=ms_step, higher_is_better=True, scaling="weak", vs_baseline=None,
                    dtype="f64" if isz == 8 else "f32", data="synthetic (reference blast IC, built on the device)",
                    config=config_for(nb, Tcase), gpu_launches=args.steps * r["launches_per_step"],
                    e2e=e2e, roofline=roofline, cpu_baseline=cpu, clocks=clocks)
        # the metric's own quantities, compact, ahead of the detailed records
        if batched:
            line["batched_fp32_gcell_s"] = batched["batched_fp32"]["value"]
            line["batched_fp32_fused_gcell_s"] = batched["batched_fp32_fused"]["value"]
            line["batched_fp64_gcell_s"] = batched["batched_fp64"]["value"]
            line["batched_fp32_over_plain_fp64_same_instances"] = batched["batched_fp32_over_plain_fp64"]
            line["batched_fp32_over_plain_fp64_large_grid"] = batched["batched_fp32"]["value"] / value
            line["batched_fp32_rho_rel_l1_vs_fp64"] = batched["batched_fp32"]["rho_rel_l1_vs_fp64_max"]
            line["batched_fp32_fused_rho_rel_l1_vs_fp64"] = batched["batched_fp32_fused"]["rho_rel_l1_vs_fp64_max"]
        if serving:
            top = serving[max(serving, key=lambda k: float(k.split("_")[1]))]
            line["serving"] = {k: dict(p50_s=v["batched"]["p50_s"], p99_s=v["batched"]["p99_s"],
                                       completed=v["batched"]["completed"], gcell_s=v["batched"]["gcell_s"],
                                       over_plain=v.get("batched_over_plain")) for k, v in serving.items()}
            if "batched_fp32_over_plain_fp64" in top:
                line["serving_fp32_over_plain_fp64_top_rate"] = top["batched_fp32_over_plain_fp64"]
        if variants:
            line["variants_gcell_s"] = {k: v["value"] for k, v in variants.items()}
            line["variants_frac"] = {k: v["frac"] for k, v in variants.items()}
        if accuracy:
            line["accuracy_vs_strict_fp64"] = accuracy
        if tuned:
            line["autotuned_shapes"] = {k: dict(warps=v["warps"], blocks=v.get("blocks", 0), chunk=v["chunk"])
                                        for k, v in tuned.items()}
        line["energy"] = energy_entry(r["energy_j"], total_ms / 1e3, cells * args.steps)
        line["variants"] = variants
        line["batched"] = batched
        line["serving_detail"] = serving
        print(json.dumps(line), flush=True)
    reps.barrier()
    reps.close()


if __name__ == "__main__":
    main()

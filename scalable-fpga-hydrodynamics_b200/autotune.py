"""Tile-shape autotuner, keyed on dimensionality and precision.

Plain path (`tune_plain`): the strip kernels take two shape parameters each. Both take the
most X rows (2D) or planes (3D) one block marches (`chunk`, 0 for the built-in 256; grids
too small to fill the GPU with such blocks take fewer, so a value tuned on one grid suits
others): longer chunks re-read fewer halo rows but give fewer blocks. The 3D kernel also
takes its tile height in rows with the one-row halo: 8, 9, 12 or 16 in FP64, 8 or 16 in
FP32. Tiles of 8, 12 and 16 rows run one warp per row (taller tiles recompute fewer halo
rows but hold one block per SM); the 9-row tile runs on 8 warps, warp 0 holding both halo
rows (FP64 with tensor-map staging). The 2D kernel also takes its register budget in resident
blocks per SM (4, or 5 in FP64 / 8 in FP32): more resident warps against fewer registers
per thread. `tune_plain` times a few steps of the blast on the grid it is given for every
candidate, keeps the fastest and installs it in the library (hydro_set_launch_shape); the
results do not depend on the shape.

Batched path (`tune`): the batched kernels take a fixed block shape (2D: 128 lanes over
126 interior columns; 3D: 8 x 32 lanes over 6 x 30 interior columns) and one free tile
parameter, the rows (planes) a work item marches, `chunk`. Longer chunks re-read fewer halo rows and take fewer work items; shorter ones
balance uneven instances better, so the best value depends on how much work a step holds:
`tune` times a batch drawn like the batched workload in 2D (256 seeded blasts, sides
log-uniform in [64, 2048]; a smaller batch favours shorter chunks) and 48 seeded 3D blasts
with sides in [32, 256] in 3D, for each candidate, and keeps the fastest.

Results are cached per (GPU name, dimensionality, precision[, arithmetic]) in a JSON file
next to this module (written on the machine that runs it, not shipped).
"""
from __future__ import annotations

import json
import os
import time
from pathlib import Path

import numpy as np

from . import BlastRun, _torch, last_launch_shape, set_launch_shape
from .batch import Batch
from .workloads import batch_blasts

CACHE = Path(os.environ.get("HYDRO_B200_TUNE_CACHE", Path(__file__).resolve().parent / "autotune_cache.json"))
CANDIDATES = {2: (32, 48, 64, 96, 128, 256), 3: (16, 32, 64, 128)}
TUNE_INSTANCES = {2: 256, 3: 48}


def _key(dim, dtype):
    torch = _torch()
    return f"{torch.cuda.get_device_name()}|{dim}d|{np.dtype(dtype).name}"


def _load():
    try:
        return json.loads(CACHE.read_text())
    except Exception:
        return {}


def _blasts(dim, n, seed):
    if dim == 2:
        return batch_blasts(n, seed=seed, steps=10 ** 9)
    from .workloads import _blast, _sides

    rng = np.random.default_rng(seed)
    return [_blast(rng, _sides(rng, 32, 256, 3)) for _ in range(n)]


def measure(dim, dtype, chunk, n=48, steps=6, seed=11):
    """Cell-updates per second of the batched step on `n` seeded blasts."""
    torch = _torch()
    blasts = _blasts(dim, n, seed)
    s = torch.cuda.Stream()
    b = Batch(dim, dtype, chunk=chunk, capacity=n, stream=s)
    cells = 0
    for bl in blasts:
        b.add(bl)
        cells += int(np.prod(bl.nb))
    b.run(2)  # warm-up (builds the graph)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    b.run(steps, sync=False)  # a different step count: the timed graph below is built here
    b.sync()
    e0.record(s)
    b.run(steps, sync=False)
    e1.record(s)
    b.sync()
    ms = e0.elapsed_time(e1)
    b.close()
    return cells * steps / (ms / 1e3)


def tune(dim, dtype, force=False, log=None, candidates=None, n=None, steps=10):
    """The fastest chunk for (this GPU, dim, dtype), measured once and then cached."""
    cache = _load()
    key = _key(dim, dtype)
    if key in cache and not force:
        return int(cache[key]["chunk"])
    n = n or TUNE_INSTANCES[dim]
    results = {}
    for c in candidates or CANDIDATES[dim]:
        t0 = time.perf_counter()
        results[c] = measure(dim, dtype, c, n=n, steps=steps)
        if log:
            log(f"autotune {key} chunk {c}: {results[c] / 1e9:.1f} GCell/s ({time.perf_counter() - t0:.1f} s)")
    best = max(results, key=results.get)
    cache[key] = dict(chunk=best, gcell_s={str(k): v / 1e9 for k, v in results.items()})
    try:
        CACHE.write_text(json.dumps(cache, indent=1))
    except OSError:
        pass
    return best


def best_chunk(dim, dtype):
    """The tuned chunk if known on this machine, else the engine default (0)."""
    entry = _load().get(_key(dim, dtype))
    return int(entry["chunk"]) if entry else 0


# plain-path candidates per (dim, precision bytes): (3D tile rows with halo or 2D blocks
# per SM, the other 0) and chunks
PLAIN_SHAPES = {(2, 4): [(0, 4), (0, 8)], (2, 8): [(0, 4), (0, 5)], (3, 4): [(8, 0), (16, 0)],
                (3, 8): [(9, 0), (8, 0), (12, 0), (16, 0)]}
PLAIN_CHUNKS = {2: (0, 32, 64, 128, 256), 3: (0, 16, 32, 64, 128)}


def measure_plain(run, warps, chunk, blocks=0, steps=3, warmup=1):
    """Cell-updates per second of the plain path with one launch shape: CUDA events around
    `steps` steps of `run` (a BlastRun) after `warmup`, and the shape that ran."""
    torch = _torch()
    set_launch_shape(len(run.nb), run.T, warps, chunk, blocks)
    for _ in range(warmup):
        run.step()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    for _ in range(steps):
        run.step()
    e1.record()
    torch.cuda.synchronize()
    return int(np.prod(run.nb)) * steps / (e0.elapsed_time(e1) / 1e3), last_launch_shape()


def tune_plain(nb, dtype, arith="strict", force=False, log=None):
    """The fastest launch shape of the plain path for (this GPU, dim, dtype, arith), timed
    on the blast of grid `nb` once and then cached; installs it and returns it as a dict.
    One run steps through every candidate twice, in opposite orders (the state evolves
    between candidates), and each candidate keeps its faster pass."""
    dim = len(nb)
    T = np.dtype(dtype)
    cache = _load()
    key = f"plain|{_key(dim, dtype)}|{arith}"
    if key in cache and not force:
        best = cache[key]
        set_launch_shape(dim, dtype, best["warps"], best["chunk"], best.get("blocks", 0))
        return best
    torch = _torch()
    cands = [(w, b, c) for w, b in PLAIN_SHAPES[(dim, T.itemsize)] for c in PLAIN_CHUNKS[dim]]
    run = BlastRun(nb, np.dtype(dtype).type, arith=arith)
    rates, shapes = {}, {}
    for order in (cands, cands[::-1]):
        for w, b, c in order:
            rate, shape = measure_plain(run, w, c, b)
            rates[(w, b, c)] = max(rates.get((w, b, c), 0.0), rate)
            shapes[(w, b, c)] = shape
    del run
    torch.cuda.empty_cache()
    if log:
        for (w, b, c), r in rates.items():
            log(f"autotune {key} warps {w} blocks {b} chunk {c}: {r / 1e9:.1f} GCell/s (ran {shapes[(w, b, c)]})")
    (w, b, c), rate = max(rates.items(), key=lambda kv: kv[1])
    best = dict(warps=w, blocks=b, chunk=c, gcell_s=rate / 1e9, grid=list(nb), ran=shapes[(w, b, c)],
                tried={f"w{k[0]}_b{k[1]}_c{k[2]}": v / 1e9 for k, v in rates.items()})
    cache[key] = best
    try:
        CACHE.write_text(json.dumps(cache, indent=1))
    except OSError:
        pass
    set_launch_shape(dim, dtype, w, c, b)
    return best

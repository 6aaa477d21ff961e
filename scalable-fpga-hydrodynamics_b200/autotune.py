"""Tile-shape autotuner for the batched step, keyed on dimensionality and precision.

The batched kernels take a fixed block shape (2D: 128 lanes over 126 interior columns;
3D: 8 x 32 lanes over 6 x 30 interior columns in FP64, 16 x 32 over 14 x 30 in FP32) and
one free tile parameter: the number
of X rows (planes) a work item marches, `chunk`. Longer chunks re-read fewer halo rows
and take fewer work items; shorter ones balance uneven instances better. `tune` times a
seeded mini-batch of the batched workload for each candidate and keeps the fastest;
results are cached per (GPU name, dimensionality, precision) in a JSON file next to this
module (written on the machine that runs it, not shipped).
"""
from __future__ import annotations

import json
import os
import time
from pathlib import Path

import numpy as np

from . import _torch
from .batch import Batch
from .workloads import batch_blasts

CACHE = Path(os.environ.get("HYDRO_B200_TUNE_CACHE", Path(__file__).resolve().parent / "autotune_cache.json"))
CANDIDATES = {2: (32, 64, 128, 256, 512), 3: (16, 32, 64, 128)}


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
    """Cell-updates per second of the batched step on a seeded mini-batch."""
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


def tune(dim, dtype, force=False, log=None, candidates=None, n=48, steps=6):
    """The fastest chunk for (this GPU, dim, dtype), measured once and then cached."""
    cache = _load()
    key = _key(dim, dtype)
    if key in cache and not force:
        return int(cache[key]["chunk"])
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

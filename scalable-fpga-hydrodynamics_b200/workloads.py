"""Seeded synthetic blast workloads for the batched and serving paths.

No dataset is involved: every instance is a blast problem drawn from a fixed seed.

* batch_blasts(n, seed): the batched workload -- 2D instances with the long side
  log-uniform in [64, 2048] and aspect ratio uniform in [1, 2]; density 1 everywhere at
  rest; pressure p_in inside a circle, p_out = 0.1 outside, p_in/p_out log-uniform in
  [10, 1000]; radius uniform in [0.05, 0.2] x the short side; centre uniform in the middle
  half of each axis; gamma 1.4 (K = 1.1, C = 0.5 as the reference); 200 steps each.
* request_stream(rate, duration, seed): the serving workload -- Poisson arrivals at `rate`
  per second; 70% 2D blasts with sides log-uniform in [128, 4096], 30% 3D blasts with
  sides log-uniform in [32, 256]; initial conditions as above; t_end uniform in
  [0.05, 0.5] of the sound-crossing time L / c_out (L = 1, c_out = sqrt(gamma p_out / rho));
  FP32 or FP64 per request (50/50 unless stated).
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

from .batch import Blast


def _blast(rng, nb, t_end=float("inf"), max_steps=2 ** 62, C=None):
    nb = tuple(int(n) for n in nb)
    short = min(nb)
    centre = tuple(1.0 + (n - 1) * rng.uniform(0.25, 0.75) for n in nb)
    radius = rng.uniform(0.05, 0.2) * short
    p_out = 0.1
    p_in = p_out * math.exp(rng.uniform(math.log(10.0), math.log(1000.0)))
    return Blast(nb=nb, centre=centre, radius=radius, rho_in=1.0, rho_out=1.0, p_in=p_in, p_out=p_out, gamma=1.4,
                 K=1.1, C=C, t_end=t_end, max_steps=max_steps)


def _sides(rng, lo, hi, dim):
    long_side = math.exp(rng.uniform(math.log(lo), math.log(hi)))
    if dim == 2:
        other = long_side / rng.uniform(1.0, 2.0)
        sides = [long_side, other]
        rng.shuffle(sides)
        return tuple(max(2, int(round(s))) for s in sides)
    return tuple(max(2, int(round(math.exp(rng.uniform(math.log(lo), math.log(hi)))))) for _ in range(3))


def batch_blasts(n: int = 256, seed: int = 0, steps: int = 200):
    rng = np.random.default_rng(seed)
    return [_blast(rng, _sides(rng, 64, 2048, 2), max_steps=steps) for _ in range(n)]


@dataclass
class Request:
    rid: int
    arrival: float          # seconds from the start of the stream
    blast: Blast
    dtype: type             # np.float32 or np.float64


def sound_crossing_time(p_out=0.1, rho=1.0, gamma=1.4, length=1.0):
    return length / math.sqrt(gamma * p_out / rho)


def request_stream(rate: float, duration: float = math.inf, seed: int = 0, frac_3d: float = 0.3,
                   frac_fp64: float = 0.5, sides_2d=(128, 4096), sides_3d=(32, 256), t_end_frac=(0.05, 0.5),
                   count: int = None):
    """Requests arriving within `duration` seconds, at most `count` of them (one of the two
    must be finite)."""
    if count is None and not math.isfinite(duration):
        raise ValueError("request_stream needs a finite duration or a count")
    rng = np.random.default_rng(seed)
    out, t, rid = [], 0.0, 0
    tc = sound_crossing_time()
    while count is None or len(out) < count:
        t += rng.exponential(1.0 / rate)
        if t > duration:
            break
        dim = 3 if rng.uniform() < frac_3d else 2
        nb = _sides(rng, *(sides_3d if dim == 3 else sides_2d), dim)
        t_end = rng.uniform(*t_end_frac) * tc
        b = _blast(rng, nb, t_end=t_end)
        dt = np.float64 if rng.uniform() < frac_fp64 else np.float32
        out.append(Request(rid, t, b, dt))
        rid += 1
    return out

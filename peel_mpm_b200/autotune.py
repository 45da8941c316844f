"""Autotuner for the P2G tile: sorted particles per P2G block.

The P2G scatter kernel gives each block a fixed range of particles in sorted
(cell) order.  Small ranges let the hardware scheduler balance blocks whose
cell structure differs; large ranges amortise the shared-tile set-up and flush
over more particles.  The best range depends on how many particles share a
sort block (particles per cell, scene size) and on the grid, so it is
measured: ``tune(obj)`` times a few substeps of ``obj`` (an ``AnisoMPM`` or a
``BatchedAnisoMPM``) with each candidate range, restores the state, sets
``obj.p2g_range`` to the fastest and caches the choice per size bucket
(log2 of particles per scene, grid size, number of scenes), so scenes of the
same bucket reuse it.  ``save``/``load`` persist the cache as JSON.

The range changes only the float summation order inside P2G, never which
contributions are summed.
"""
from __future__ import annotations

import json
import math
from typing import Iterable, Optional

import torch

CANDIDATES = (128, 256, 512, 1024, 2048)
_CACHE: dict = {}


def bucket(obj) -> tuple:
    """Size bucket of a solver or batch."""
    sims = getattr(obj, "sims", None)
    if sims is None:
        return ("plain", int(round(math.log2(max(obj.n, 1)))), int(obj.n_grid), 1)
    mean_n = sum(s.n for s in sims) / len(sims)
    return ("batch", int(round(math.log2(max(mean_n, 1)))), int(max(s.n_grid for s in sims)), len(sims))


def _mutable_state(obj):
    sims = getattr(obj, "sims", None)
    if sims is None:
        return obj._S[:27].clone(), [obj._step]
    return obj._S[:27].clone(), [s._step for s in sims]


def _restore(obj, saved):
    S, steps = saved
    obj._S[:27].copy_(S)
    sims = getattr(obj, "sims", None)
    if sims is None:
        obj._step = steps[0]
    else:
        for s, k in zip(sims, steps):
            s._step = k


def _time_frame(obj, substeps: int, reps: int) -> float:
    dev = obj.device
    s = torch.cuda.current_stream(dev)
    obj.run_frame(substeps, 0.0)          # capture / warm-up
    torch.cuda.synchronize(dev)
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    best = float("inf")
    for _ in range(reps):
        a.record(s)
        obj.run_frame(substeps, 0.0)
        b.record(s)
        torch.cuda.synchronize(dev)
        best = min(best, a.elapsed_time(b))
    return best


def tune(obj, candidates: Iterable[int] = CANDIDATES, substeps: int = 4, reps: int = 2,
         force: bool = False) -> int:
    """Pick ``obj.p2g_range`` by timing; returns the chosen range."""
    key = bucket(obj)
    if not force and key in _CACHE:
        obj.p2g_range = _CACHE[key]["range"]
        return obj.p2g_range
    saved = _mutable_state(obj)
    times = {}
    try:
        for r in candidates:
            obj.p2g_range = int(r)
            times[int(r)] = _time_frame(obj, substeps, reps)
            _restore(obj, saved)
    finally:
        _restore(obj, saved)
    best = min(times, key=times.get)
    obj.p2g_range = best
    _CACHE[key] = {"range": best, "ms": times}
    return best


def cache() -> dict:
    return {"|".join(map(str, k)): v for k, v in _CACHE.items()}


def save(path: str):
    with open(path, "w") as f:
        json.dump(cache(), f, indent=1)


def load(path: str):
    with open(path) as f:
        data = json.load(f)
    for k, v in data.items():
        parts = k.split("|")
        _CACHE[(parts[0], int(parts[1]), int(parts[2]), int(parts[3]))] = v

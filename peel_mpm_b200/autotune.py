"""Autotuner for the substep's launch knobs, per size bucket.

Four knobs shape the launches and never the results (the P2G grid sums are
exact integers, every other kernel computes each particle or node the same
way whatever its launch shape):

* ``p2g_ctas_per_sm``: resident CTAs per SM of the persistent P2G kernel,
  which takes 4^3-cell sub-blocks from a work list (0: the 80-register build
  at 3 per SM; 4: the 64-register build at 4 per SM).  More CTAs hide more
  latency; fewer registers spill a little.
* ``stress_ctas_per_sm``: resident CTAs per SM of the constitutive update
  (3: the 80-register build; 4: the 64-register build, which spills a few
  values to L1 but runs more warps per SM).
* ``g2p_ctas_per_sm``: the same choice for G2P (0: the library default, 4 for
  one scene and 3 for a batch).
* ``grid_ctas_per_sm``: CTAs per SM of the grid update over the active 4^3
  node blocks (a grid-stride cap; 0 gives every 4-node row its own thread).

``tune(obj)`` times a few substeps of ``obj`` (an ``AnisoMPM`` or a
``BatchedAnisoMPM``) per candidate, one knob at a time in the order above,
each at the values already chosen for the ones before it, restores the state, sets the knobs to
the fastest and caches the choice per size bucket (log2 of particles per
scene, grid size, number of scenes), so scenes of the same bucket reuse it.
``save``/``load`` persist the cache as JSON.
"""
from __future__ import annotations

import json
import math
from typing import Optional

import torch

P2G_CANDIDATES = (0, 2, 4)             # 0: as many as fit of the 80-register build (3 per SM)
STRESS_CANDIDATES = (3, 4)
G2P_CANDIDATES = (3, 4)
GRID_CANDIDATES = (0, 4, 8, 16, 32)    # 0: one thread per node row
KNOBS = ("p2g_ctas_per_sm", "stress_ctas_per_sm", "g2p_ctas_per_sm", "grid_ctas_per_sm")
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


def _apply(obj, knobs: dict):
    for name in KNOBS:
        setattr(obj, name, int(knobs.get(name, 0)))


def tune(obj, substeps: int = 4, reps: int = 2, force: bool = False, p2g_candidates=P2G_CANDIDATES,
         grid_candidates=GRID_CANDIDATES, stress_candidates=STRESS_CANDIDATES, g2p_candidates=G2P_CANDIDATES) -> dict:
    """Pick the launch knobs of ``obj`` by timing; returns them as a dict."""
    key = bucket(obj)
    if not force and key in _CACHE:
        _apply(obj, _CACHE[key]["knobs"])
        return dict(_CACHE[key]["knobs"])
    saved = _mutable_state(obj)
    cands_of = {"p2g_ctas_per_sm": p2g_candidates, "stress_ctas_per_sm": stress_candidates,
                "g2p_ctas_per_sm": g2p_candidates, "grid_ctas_per_sm": grid_candidates}
    times = {name: {} for name in KNOBS}
    knobs = {name: 0 for name in KNOBS}
    try:
        for name in KNOBS:
            cands = cands_of[name]
            for c in cands:
                _apply(obj, dict(knobs, **{name: int(c)}))
                times[name][int(c)] = _time_frame(obj, substeps, reps)
                _restore(obj, saved)
            knobs[name] = min(times[name], key=times[name].get)
    finally:
        _restore(obj, saved)
    _apply(obj, knobs)
    _CACHE[key] = {"knobs": dict(knobs), "ms": times, "substeps": substeps}
    return dict(knobs)


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
        v["ms"] = {name: {int(c): t for c, t in d.items()} for name, d in v["ms"].items()}
        _CACHE[(parts[0], int(parts[1]), int(parts[2]), int(parts[3]))] = v

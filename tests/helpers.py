"""Shared test helpers: goldens, error metrics, scene -> solver builders."""
from __future__ import annotations

import json
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden")
FIELDS = ("x", "v", "F", "C", "d", "lap", "D_hist")

_GOLD = None


def goldens():
    """(arrays, meta) written by tests/golden/make_golden.py from the reference solver."""
    global _GOLD
    if _GOLD is None:
        z = np.load(os.path.join(GOLDEN, "reference_goldens.npz"))
        with open(os.path.join(GOLDEN, "reference_goldens.json")) as f:
            meta = json.load(f)
        _GOLD = ({k: z[k] for k in z.files}, meta)
    return _GOLD


def rel_l2(a, b):
    a = np.asarray(a, np.float64).ravel()
    b = np.asarray(b, np.float64).ravel()
    den = max(np.linalg.norm(a), 1e-30)
    return float(np.linalg.norm(a - b) / den)


def golden_state(name, tag, step):
    arr, meta = goldens()
    return {f: arr[f"{name}/{tag}/{step}/{f}"] for f in FIELDS if f"{name}/{tag}/{step}/{f}" in arr}


def make_gpu_sim(scene, device="cuda:0"):
    """This package's solver populated with a scene through the reference API."""
    import torch
    import peel_mpm_b200 as pm
    from peel_mpm_b200 import scenes

    sim = pm.AnisoMPM(n_grid=scene.n_grid, grid_lim=scene.grid_lim, dt=scene.dt, gravity=tuple(scene.gravity),
                      grid_damp=scene.grid_damp, f_clamp=scene.f_clamp, damage_every=scene.damage_every,
                      device=device)

    def mk_col(c):
        if c.kind == "halfspace":
            return pm.halfspace_collider(c.origin_fn(), list(c.normal), mode=c.mode, friction=c.friction)
        return pm.sphere_collider(c.origin_fn(), c.radius, mode=c.mode, friction=c.friction)

    scenes.apply_scene(sim, scene, pm.grip_bc, mk_col, torch)
    return sim


def gpu_state(sim, stride=1):
    out = {}
    for f in FIELDS:
        out[f] = getattr(sim, f).detach().cpu().numpy()[::stride]
    return out

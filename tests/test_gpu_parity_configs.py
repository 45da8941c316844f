"""Parity at the configurations the throughput is quoted on, against the
oracle (the C restatement of anisompm.py:593-803, pinned to the reference's
goldens), at their stated sizes and step counts.

Every comparison is relative L2 over all particles, per field, printed beside
the reference algorithm's own reordering envelope for the same configuration:
the oracle run a second time on a permuted particle order, which changes only
the summation order inside the grid scatters (the same experiment that gives
the reference's own envelope in tests/golden/reference_goldens.json).  Bounds:
x, v, F, C within 1e-4 (the parity target); the chaotic damage fields d, lap,
D_hist within ten times the larger of that envelope and 1e-4, since damage
threshold branches flip under any change of rounding, float64 included.

With PEELMPM_PARITY_LOG set, each test appends its numbers to that file as one
JSON line.
"""
import json
import os

import numpy as np
import pytest
import torch

from helpers import FIELDS, gpu_state, make_gpu_sim, rel_l2
import oracle as orc
from peel_mpm_b200 import scenes
import peel_mpm_b200 as pm

pytestmark = pytest.mark.gpu

KIN = ("x", "v", "F", "C")
DMG = ("d", "lap", "D_hist")
CORES = os.cpu_count() or 1


def _log(record):
    print(json.dumps(record))
    path = os.environ.get("PEELMPM_PARITY_LOG")
    if path:
        with open(path, "a") as f:
            f.write(json.dumps(record) + "\n")


def _permute_scene(sc, perm):
    import copy
    s2 = copy.copy(sc)
    s2.x = sc.x[perm]
    s2.vol = sc.vol[perm]
    s2.E = sc.E[perm]
    s2.sigma_c = sc.sigma_c[perm]
    s2.fibers = None if sc.fibers is None else sc.fibers[perm]
    s2.d0 = None if sc.d0 is None else sc.d0[perm]
    s2.allow = None if sc.allow is None else sc.allow[perm]
    s2.grips = [scenes.Grip(g.mask[perm], g.velocity, g.ramp) for g in sc.grips]
    if sc.interface is not None:
        s2.interface = (sc.interface[0][perm], sc.interface[1][perm])
    return s2


def _oracle_pair(sc, seed=1234):
    """The oracle in the scene's order and in a permuted order (for the
    envelope), both on every host core with the deterministic slab scatter."""
    perm = np.random.default_rng(seed).permutation(sc.n)
    a = orc.OracleSim(sc, np.float32, nthreads=CORES, scatter_mode=1)
    b = orc.OracleSim(_permute_scene(sc, perm), np.float32, nthreads=CORES, scatter_mode=1)
    return a, b, np.argsort(perm)


def _errors(ora, other):
    return {f: rel_l2(getattr(ora, f), other[f]) for f in FIELDS}


def _envelope(a, b, inv):
    return {f: rel_l2(getattr(a, f), getattr(b, f)[inv]) for f in FIELDS}


def _check(errs, env, kin_bound=1e-4):
    for f in KIN:
        assert errs[f] < kin_bound, (f, errs[f], env[f])
    for f in DMG:
        assert errs[f] < 10 * max(env[f], 1e-4), (f, errs[f], env[f])


def _fmt(d):
    return {k: float(f"{v:.3e}") for k, v in d.items()}


def test_plain_1m_full_500_substeps_vs_oracle():
    """The headline scene at its stated size and step count: 1,048,576
    particles on 128^3, dt 5e-5, all 500 substeps, the GPU advancing by
    graph-replayed frames of 100 substeps as the benchmark does.  Snapshots
    at 100, 250 and 500 substeps show where any divergence grows."""
    sc = scenes.plain_1m()
    assert sc.n == 1048576 and sc.n_steps == 500
    sim = make_gpu_sim(sc)
    ora, orp, inv = _oracle_pair(sc)
    snaps = (100, 250, 500)
    rec = {"test": "plain_1m", "particles": sc.n, "substeps": 500, "snapshots": {}}
    done = 0
    for stop in snaps:
        sim.run_frame(stop - done, done * sc.dt)
        for s in range(done, stop):
            ora.substep(s * sc.dt)
            orp.substep(s * sc.dt)
        done = stop
        torch.cuda.synchronize()
        errs = _errors(ora, gpu_state(sim))
        env = _envelope(ora, orp, inv)
        rec["snapshots"][stop] = {"gpu_vs_oracle": _fmt(errs), "oracle_reorder_envelope": _fmt(env),
                                  "d_max": float(ora.d.max())}
    _log(rec)
    st = sim.status()
    assert st["nonfinite"] == 0
    for stop in snaps:
        r = rec["snapshots"][stop]
        _check(r["gpu_vs_oracle"], r["oracle_reorder_envelope"])


def test_peel_eighth_200_substeps_vs_oracle():
    """The two-layer peel scene (256^3 grid, 27 particles per cell, gravity,
    bonding band of critical stress 40 under layers of 400) with its in-plane
    extent divided by 8 (138,240 particles), 200 substeps."""
    sc = scenes.peel_8m(scale=8)
    sim = make_gpu_sim(sc)
    ora, orp, inv = _oracle_pair(sc)
    sim.run_frame(100, 0.0)
    sim.run_frame(100, 100 * sc.dt)
    for s in range(200):
        ora.substep(s * sc.dt)
        orp.substep(s * sc.dt)
    torch.cuda.synchronize()
    errs = _errors(ora, gpu_state(sim))
    env = _envelope(ora, orp, inv)
    _log({"test": "peel_eighth", "particles": sc.n, "substeps": 200, "gpu_vs_oracle": _fmt(errs),
          "oracle_reorder_envelope": _fmt(env), "d_max": float(ora.d.max())})
    assert sim.status()["nonfinite"] == 0
    _check(errs, env)


def test_batch_of_64_scenes_vs_oracle():
    """The 64-scene batch (log-uniform 4k-256k particles, grids 32^3-112^3,
    per-scene E, nu, fibers, critical stress and pull), one BatchedAnisoMPM
    frame of 20 substeps; every scene against its own oracle run."""
    scs = scenes.batch_scenes(seed=0)
    assert len(scs) == 64

    def build(sc):
        sim = pm.AnisoMPM(n_grid=sc.n_grid, grid_lim=sc.grid_lim, dt=sc.dt, gravity=tuple(sc.gravity),
                          grid_damp=sc.grid_damp, f_clamp=sc.f_clamp, damage_every=sc.damage_every,
                          device="cuda:0")
        scenes.apply_scene(sim, sc, pm.grip_bc, None, torch)
        return sim

    batch = pm.BatchedAnisoMPM([build(sc) for sc in scs])
    n_sub = 20
    batch.run_frame(n_sub, [0.0] * len(scs))
    torch.cuda.synchronize()
    worst = {f: 0.0 for f in FIELDS}
    worst_env = {f: 0.0 for f in FIELDS}
    per_scene = []
    for k, (sc, sim) in enumerate(zip(scs, batch.sims)):
        ora, orp, inv = _oracle_pair(sc, seed=100 + k)
        for s in range(n_sub):
            ora.substep(s * sc.dt)
            orp.substep(s * sc.dt)
        errs = _errors(ora, gpu_state(sim))
        env = _envelope(ora, orp, inv)
        per_scene.append((k, sc.n, sc.n_grid, errs, env))
        for f in FIELDS:
            worst[f] = max(worst[f], errs[f])
            worst_env[f] = max(worst_env[f], env[f])
    _log({"test": "batch64", "scenes": len(scs), "particles": sum(sc.n for sc in scs), "substeps": n_sub,
          "worst_gpu_vs_oracle": _fmt(worst), "worst_oracle_reorder_envelope": _fmt(worst_env)})
    assert all(st["nonfinite"] == 0 for st in batch.status())
    for k, n, ng, errs, env in per_scene:
        _check(errs, env)

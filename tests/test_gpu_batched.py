"""BatchedAnisoMPM against the same scenes stepped one by one.

The batch runs every kernel once over all scenes (one sort over all scenes'
keys, per-scene grids, parameters, grips, colliders and clocks read from the
workspace).  Each scene must evolve as the plain solver evolves it alone;
atomic summation order differs between runs, so the comparison uses the
float32-rounding bounds of the graph tests, not bit equality.
"""
import ctypes as C

import numpy as np
import pytest
import torch

from helpers import gpu_state, make_gpu_sim, rel_l2
from peel_mpm_b200 import BatchedAnisoMPM, _lib, scenes

pytestmark = pytest.mark.gpu


def mixed_scenes():
    # uneven sizes and grids, plus the scenes that exercise colliders,
    # f_clamp, damage_every=2, grid damping, ramps and interface normals
    return scenes.batch_scenes(seed=1, n_scenes=5, n_lo=500, n_hi=20000) + [
        scenes.knobs_drop(), scenes.tiny_bar(), scenes.interface_peel()]


# d, lap and D_hist fracture chaotically: any change of float summation order
# moves them by up to ~3e-4 (the reference against itself with its particles
# permuted), so they are held to 10x that; x, v, F, C to float32 rounding.
def compare(sa, sb, tight=1e-5, loose=3e-3):
    for f in ("x", "v", "F", "C"):
        assert rel_l2(sb[f], sa[f]) < tight, f
    for f in ("d", "lap", "D_hist"):
        assert rel_l2(sb[f], sa[f]) < loose, f


@pytest.mark.parametrize("graphs", [True, False])
def test_batch_matches_individual_scenes(graphs):
    scs = mixed_scenes()
    solo = [make_gpu_sim(sc) for sc in scs]
    packed = [make_gpu_sim(sc) for sc in scs]
    batch = BatchedAnisoMPM(packed, use_graphs=graphs)
    n_sub, frames = 6, 3
    for f in range(frames):
        t0 = [f * n_sub * sc.dt for sc in scs]
        batch.run_frame(n_sub, t0)
        for sim, t in zip(solo, t0):
            sim.run_frame(n_sub, t)
    torch.cuda.synchronize()
    for sim_a, sim_b in zip(solo, packed):
        assert sim_b._step == sim_a._step == n_sub * frames
        compare(gpu_state(sim_a), gpu_state(sim_b))
    st = batch.check()
    assert len(st) == len(scs) and all(s["nonfinite"] == 0 for s in st)
    if graphs:
        assert len(batch._graphs) == 1


def test_batch_views_alias_the_batch_and_unpack_copies():
    scs = scenes.batch_scenes(seed=2, n_scenes=3, n_lo=300, n_hi=3000)
    sims = [make_gpu_sim(sc) for sc in scs]
    x0 = [s.x.clone() for s in sims]
    batch = BatchedAnisoMPM(sims)
    for s, x in zip(sims, x0):
        assert torch.equal(s.x, x)                      # packing kept the state
    batch.run_frame(4, 0.0)
    torch.cuda.synchronize()
    moved = [s.x.clone() for s in sims]
    assert any(not torch.equal(m, x) for m, x in zip(moved, x0))
    with pytest.raises(RuntimeError):
        sims[0].add_object(torch.zeros(1, 3) + 0.5, torch.ones(1) * 1e-6)
    batch.unpack()
    for s, m in zip(sims, moved):
        assert torch.equal(s.x, m)
        assert s._batch is None
    sims[0].run_frame(2, 0.0)                         # standalone again
    torch.cuda.synchronize()
    assert np.isfinite(sims[0].x.cpu().numpy()).all()


def test_batch_parameter_change_reaches_the_graph():
    scs = scenes.batch_scenes(seed=3, n_scenes=2, n_lo=400, n_hi=2000)
    a = [make_gpu_sim(sc) for sc in scs]
    b = [make_gpu_sim(sc) for sc in scs]
    batch = BatchedAnisoMPM(a)
    batch.run_frame(3, 0.0)
    for s in b:
        s.run_frame(3, 0.0)
    a[1].gravity = (0.0, -20.0, 0.0)
    b[1].gravity = (0.0, -20.0, 0.0)
    t0 = [3 * sc.dt for sc in scs]
    batch.run_frame(3, t0)
    for s, t in zip(b, t0):
        s.run_frame(3, t)
    torch.cuda.synchronize()
    assert len(batch._graphs) == 1                   # parameters live in the workspace
    for sa, sb in zip(b, a):
        compare(gpu_state(sa), gpu_state(sb))


def test_batch_rejects_a_workspace_of_another_batch():
    lib = _lib.load()
    scs = scenes.batch_scenes(seed=4, n_scenes=2, n_lo=300, n_hi=1000)
    batch = BatchedAnisoMPM([make_gpu_sim(sc) for sc in scs])
    batch.run_frame(1, 0.0)
    torch.cuda.synchronize()
    P = batch._sync_descriptors()
    wrong_n = (C.c_int64 * 2)(batch.ns[1], batch.ns[0])
    rc = lib.pm_batch_substep(2, wrong_n, batch._g_arr, C.byref(P), batch._ws.data_ptr(), batch._ws_bytes,
                              batch._ws.data_ptr(), torch.cuda.current_stream().cuda_stream)
    assert rc in (_lib.PM_ERR_ARG, _lib.PM_ERR_WORKSPACE)
    other = torch.empty(batch._ws_bytes, dtype=torch.uint8, device="cuda")
    rc = lib.pm_batch_substep(2, batch._n_arr, batch._g_arr, C.byref(P), other.data_ptr(), batch._ws_bytes,
                              other.data_ptr(), torch.cuda.current_stream().cuda_stream)
    assert rc == _lib.PM_ERR_WORKSPACE


def test_autotuned_knobs_keep_results_bit_for_bit():
    """The tuned launch knobs change how the work is spread over the SMs,
    never the result: the grid sums are exact, so the state is the same
    bits."""
    from peel_mpm_b200 import autotune
    scs = scenes.batch_scenes(seed=5, n_scenes=4, n_lo=500, n_hi=8000)
    a = BatchedAnisoMPM([make_gpu_sim(sc) for sc in scs])
    b = BatchedAnisoMPM([make_gpu_sim(sc) for sc in scs])
    k = autotune.tune(a, substeps=2, reps=1, force=True)
    assert k["p2g_ctas_per_sm"] in autotune.P2G_CANDIDATES and k["grid_ctas_per_sm"] in autotune.GRID_CANDIDATES
    assert k["stress_ctas_per_sm"] in autotune.STRESS_CANDIDATES and k["g2p_ctas_per_sm"] in autotune.G2P_CANDIDATES
    for name in autotune.KNOBS:
        assert getattr(a, name) == k[name], name
        assert set(autotune._CACHE[autotune.bucket(a)]["ms"][name]) == set(autotune.__dict__[
            {"p2g_ctas_per_sm": "P2G_CANDIDATES", "grid_ctas_per_sm": "GRID_CANDIDATES",
             "stress_ctas_per_sm": "STRESS_CANDIDATES", "g2p_ctas_per_sm": "G2P_CANDIDATES"}[name]])
    assert autotune.bucket(a) in autotune._CACHE
    a.run_frame(5, 0.0)
    b.run_frame(5, 0.0)
    torch.cuda.synchronize()
    for sa, sb in zip(a.sims, b.sims):
        for f, v in gpu_state(sb).items():
            assert np.array_equal(v, gpu_state(sa)[f]), f


@pytest.mark.parametrize("p2g,grid,stress,g2p", [(1, 0, 4, 3), (2, 4, 3, 4), (0, 32, 4, 4)])
def test_plain_launch_knobs_keep_results_bit_for_bit(p2g, grid, stress, g2p):
    sc = scenes.knobs_drop()
    a, b = make_gpu_sim(sc), make_gpu_sim(sc)
    a.p2g_ctas_per_sm, a.grid_ctas_per_sm = p2g, grid
    a.stress_ctas_per_sm, a.g2p_ctas_per_sm = stress, g2p
    a.run_frame(6, 0.0)
    b.run_frame(6, 0.0)
    torch.cuda.synchronize()
    for f, v in gpu_state(b).items():
        assert np.array_equal(v, gpu_state(a)[f]), f


def test_substeps_are_bit_reproducible():
    """Two runs of the same scene give the same bits (exact grid sums): the
    property the adjoint's checkpoint re-runs rely on."""
    sc = scenes.plain_1m(cells=(16, 16, 16), lo=(56, 56, 56))
    a, b = make_gpu_sim(sc), make_gpu_sim(sc)
    a.run_frame(40, 0.0)
    for s in range(40):
        b.substep(s * sc.dt)
    torch.cuda.synchronize()
    for f, v in gpu_state(b).items():
        assert np.array_equal(v, gpu_state(a)[f]), f

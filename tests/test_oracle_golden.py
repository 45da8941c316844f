"""Pins the CPU oracle to the reference solver's own outputs (CPU only).

The goldens come from running the unmodified reference AnisoMPM on the same
seeded scenes (tests/golden/make_golden.py).  The oracle restates the
reference op by op, so x, v, F and C agree to float32 rounding; d, lap and
D_hist agree to the same level until fracture starts, after which the
phase-field damage amplifies rounding differences chaotically.  The bound on
d at late steps is set by the reference's own scatter-order noise (the same
reference run with particles permuted), stored beside the goldens.
"""
import numpy as np
import pytest

from helpers import FIELDS, golden_state, goldens, rel_l2
import oracle as orc
from peel_mpm_b200 import scenes

# x, v, F, C: float32 rounding level.  d/lap/D_hist before fracture: same.
TOL_KIN = 1e-5
TOL_EARLY_DMG = 1e-4


def _run_and_compare(name, steps, stride, dtype=np.float32, tag="f32"):
    sc = scenes.SCENES[name]()
    sim = orc.OracleSim(sc, dtype)
    errs = {}
    for s in range(max(steps)):
        sim.substep(s * sim.dt)
        if s + 1 in steps:
            g = golden_state(name, tag, s + 1)
            st = sim.state()
            errs[s + 1] = {f: rel_l2(g[f], st[f][::stride]) for f in FIELDS}
    return errs


@pytest.mark.parametrize("name", ["tiny_bar", "plain_small", "knobs_drop", "interface_peel"])
def test_scene_inputs_match_golden_hash(name):
    """The seeded generators still produce the inputs the goldens were made from."""
    import hashlib
    _, meta = goldens()
    sc = scenes.SCENES[name]()
    h = hashlib.sha256()
    for a in (sc.x, sc.vol, sc.E, sc.sigma_c):
        h.update(np.ascontiguousarray(a).tobytes())
    assert h.hexdigest()[:16] == meta["scenes"][name]["hash"]


def test_tiny_bar_fp32_matches_reference():
    _, meta = goldens()
    env = meta["noise_envelope"]["tiny_bar_200"]
    errs = _run_and_compare("tiny_bar", [1, 10, 50, 200], 1)
    for f in FIELDS:
        assert errs[1][f] < 1e-6, (f, errs[1])
        assert errs[10][f] < TOL_EARLY_DMG, (f, errs[10])
    for s in (50, 200):
        for f in ("x", "v", "F", "C"):
            assert errs[s][f] < TOL_KIN, (s, f, errs[s])
    # late damage: within 10x the reference's own reordering noise
    for f in ("d", "lap"):
        assert errs[200][f] < 10 * max(env[f], 1e-4), (f, errs[200], env)


def test_tiny_bar_fp64_matches_reference_fp64():
    # float64 rounding (1e-16) amplified by 200 fracturing substeps
    errs = _run_and_compare("tiny_bar", [200], 1, np.float64, "f64")
    for f in ("x", "v", "F", "C"):
        assert errs[200][f] < 1e-6, (f, errs[200])
    # the damage update has threshold branches (relu, history max, monotone
    # max, clamp at 1), so even float64 rounding flips some particles late
    _, meta = goldens()
    env = meta["noise_envelope"]["tiny_bar_200"]
    for f in ("d", "lap"):
        assert errs[200][f] < 10 * max(env[f], 1e-4), (f, errs[200])


def test_plain_small_fp32_matches_reference():
    _, meta = goldens()
    env = meta["noise_envelope"]["plain_small_200"]
    errs = _run_and_compare("plain_small", [1, 50, 200], 8)
    for f in FIELDS:
        assert errs[1][f] < 1e-6, (f, errs[1])
    for s in (50, 200):
        for f in ("x", "v", "F", "C"):
            assert errs[s][f] < TOL_KIN, (s, f, errs[s])
    for f in ("d", "lap"):
        assert errs[200][f] < 10 * max(env[f], 1e-4), (f, errs[200], env)


@pytest.mark.parametrize("name", ["knobs_drop", "interface_peel"])
def test_knob_scenes_match_reference(name):
    errs = _run_and_compare(name, [10, 60], 1)
    for f in FIELDS:
        assert errs[10][f] < TOL_EARLY_DMG, (f, errs[10])
    for f in ("x", "v", "F", "C"):
        assert errs[60][f] < 1e-4, (f, errs[60])


def test_sym_eig_matches_reference():
    arr, _ = goldens()
    A = arr["sym_eig/A"]
    ev, V = orc.sym_eig(A)
    assert np.max(np.abs(ev - arr["sym_eig/evals"])) <= 1e-5 * max(1.0, np.abs(arr["sym_eig/evals"]).max())
    # eigenvectors: identical up to float rounding (same rotation sequence)
    assert np.max(np.abs(V - arr["sym_eig/evecs"])) < 1e-4
    recon = V @ (ev[:, :, None] * np.swapaxes(V, 1, 2))
    assert np.max(np.abs(recon - A)) < 1e-4 * max(1.0, np.abs(A).max())


@pytest.mark.parametrize("name", ["plain_small", "tiny_bar"])
@pytest.mark.parametrize("s", [0, 1])
def test_bin_keys_bit_exact(name, s):
    arr, _ = goldens()
    x = arr[f"bin/{name}/{s}/x"]
    sc = scenes.SCENES[name]()
    keys, perm = orc.bin_particles(x, sc.n_grid, 1.0 / sc.dx)
    assert np.array_equal(keys, arr[f"bin/{name}/{s}/keys"])
    assert np.array_equal(perm, arr[f"bin/{name}/{s}/perm"])


def test_oracle_parallel_scatter_is_deterministic_and_close():
    sc = scenes.tiny_bar()
    a = orc.OracleSim(sc, np.float32, nthreads=1, scatter_mode=1)
    b = orc.OracleSim(sc, np.float32, nthreads=4, scatter_mode=1)
    c = orc.OracleSim(sc, np.float32, nthreads=1, scatter_mode=0)
    a.run(15); b.run(15); c.run(15)
    for f in FIELDS:
        assert np.array_equal(getattr(a, f), getattr(b, f)), f
        assert rel_l2(getattr(c, f), getattr(a, f)) < 1e-4, f

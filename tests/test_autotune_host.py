"""Host logic of the launch-knob autotuner, without a GPU: the timing of a
frame is replaced by a cost model of the knobs, so the test checks the search
(one knob at a time, in order, each at the values chosen before it), the
state restore, the per-bucket cache and its JSON round trip."""
import json

import torch

from peel_mpm_b200 import autotune


class FakeSim:
    """Stands in for an AnisoMPM: n, n_grid, a mutable state and the knobs."""

    def __init__(self, n=1 << 20, n_grid=128):
        self.n, self.n_grid, self.device = n, n_grid, "cpu"
        self._S = torch.arange(27 * 8, dtype=torch.float32).reshape(27, 8)
        self._step = 7
        for k in autotune.KNOBS:
            setattr(self, k, 0)


def cost(obj, substeps, reps):
    # best at p2g 4, stress 3, g2p 4, grid 16; the state is scribbled on as a
    # frame would, and must be restored after every candidate
    obj._S += 1.0
    obj._step += substeps
    return (abs(obj.p2g_ctas_per_sm - 4) + abs(obj.stress_ctas_per_sm - 3) + abs(obj.g2p_ctas_per_sm - 4)
            + abs(obj.grid_ctas_per_sm - 16) / 16.0)


def test_tune_searches_each_knob_and_restores_the_state(monkeypatch, tmp_path):
    monkeypatch.setattr(autotune, "_time_frame", cost)
    autotune._CACHE.clear()
    sim = FakeSim()
    S0, step0 = sim._S.clone(), sim._step
    knobs = autotune.tune(sim)
    assert knobs == {"p2g_ctas_per_sm": 4, "stress_ctas_per_sm": 3, "g2p_ctas_per_sm": 4, "grid_ctas_per_sm": 16}
    assert all(getattr(sim, k) == v for k, v in knobs.items())
    assert torch.equal(sim._S, S0) and sim._step == step0
    entry = autotune._CACHE[autotune.bucket(sim)]
    for name, cands in (("p2g_ctas_per_sm", autotune.P2G_CANDIDATES), ("stress_ctas_per_sm",
                        autotune.STRESS_CANDIDATES), ("g2p_ctas_per_sm", autotune.G2P_CANDIDATES),
                        ("grid_ctas_per_sm", autotune.GRID_CANDIDATES)):
        assert set(entry["ms"][name]) == set(cands)
    # a second solver of the same bucket takes the cached knobs without timing
    monkeypatch.setattr(autotune, "_time_frame", lambda *a: (_ for _ in ()).throw(AssertionError("timed")))
    other = FakeSim()
    assert autotune.tune(other) == knobs
    # JSON round trip
    path = tmp_path / "knobs.json"
    autotune.save(str(path))
    saved = json.loads(path.read_text())
    autotune._CACHE.clear()
    autotune.load(str(path))
    assert autotune._CACHE[autotune.bucket(sim)]["knobs"] == knobs
    assert json.loads(path.read_text()) == saved
    autotune._CACHE.clear()

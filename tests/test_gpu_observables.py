"""Device observables against the harness's own torch reductions
(peel_test.py:263-307 restated on the solver's tensors)."""
import numpy as np
import pytest
import torch

from helpers import make_gpu_sim
from peel_mpm_b200 import scenes
from peel_mpm_b200.observables import FrameObservables

pytestmark = pytest.mark.gpu


def test_frame_observables_match_torch_reductions():
    sc = scenes.interface_peel()
    sim = make_gpu_sim(sc)
    n = sim.n
    band = torch.tensor(sc.interface[0], device="cuda")
    top = sim.x[:, 1] > float(sim.x[:, 1].median())
    groups = {"interface": band, "top": top & ~band, "rest": ~top & ~band}
    frames, n_sub = 12, 5
    obs = FrameObservables(sim, groups, frames, d_threshold=0.1, onset_group="interface", onset_fraction=0.02)
    ref_rows, phi_pp = [], torch.zeros(n, device="cuda")
    onset_ref, snap_ref = -1, None
    for f in range(frames):
        sim.run_frame(n_sub, f * n_sub * sc.dt)
        obs.update(f)
        row = {}
        for name, m in groups.items():
            d = sim.d[m]
            row[name] = {"phi_max": float(sim.phi[m].max()), "phi_shear_max": float(sim.phi_shear[m].max()),
                         "d_mean": float(d.mean()), "d_max": float(d.max()),
                         "broken": float((d > 0.1).float().mean()), "y_mean": float(sim.x[m, 1].mean())}
        ref_rows.append(row)
        phi_pp = torch.maximum(phi_pp, sim.phi)
        if onset_ref < 0 and row["interface"]["broken"] > 0.02:
            onset_ref, snap_ref = f, sim.d.clone()
    r = obs.read()
    for f in range(frames):
        for name in groups:
            a, b = r["table"][f][name], ref_rows[f][name]
            for k in ("phi_max", "phi_shear_max", "d_max"):
                assert a[k] == pytest.approx(b[k], rel=1e-6, abs=1e-12), (f, name, k)
            for k in ("d_mean", "broken", "y_mean"):
                assert a[k] == pytest.approx(b[k], rel=1e-5, abs=1e-9), (f, name, k)
    assert torch.equal(r["phi_peak"], phi_pp)
    assert r["onset_frame"] == onset_ref
    if onset_ref >= 0:
        assert torch.equal(r["snap_d"], snap_ref)
    assert r["nonfinite"] == 0

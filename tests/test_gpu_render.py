"""The CUDA splat renderer against images made by the reference's own
renderer (tests/golden/make_render_golden.py: render.py on the CPU in
float32).  Float atomics change the summation order of the soft z-buffer
blend, and CUDA's expf/logf differ from the CPU's in the last bits, so the
bound is 1e-4 absolute on every pixel channel (an 8-bit image resolves 4e-3).
"""
import os
import sys

import numpy as np
import pytest
import torch

from helpers import GOLDEN
from peel_mpm_b200.render import Camera, render_gaussians

sys.path.insert(0, GOLDEN)
from make_render_golden import CASES  # noqa: E402

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", list(CASES))
def test_render_matches_reference_images(name):
    z = np.load(os.path.join(GOLDEN, "reference_render.npz"))
    g = {k.split("/")[1]: z[k] for k in z.files if k.startswith(name + "/")}
    W, H, fx, fy = g["cam"]
    kw = CASES[name][6]
    cam = Camera(R=g["R"], T=g["T"], fx=float(fx), fy=float(fy), width=int(W), height=int(H), device="cuda:0")
    t = lambda a: torch.tensor(a, device="cuda:0")
    img = render_gaussians(cam, t(g["xyz"]), t(g["cov"]), t(g["color"]), t(g["opacity"]), **kw)
    out = img.cpu().numpy()
    assert out.shape == g["img"].shape
    err = np.abs(out - g["img"])
    print(name, "max abs err", err.max(), "mean", err.mean())
    assert err.max() < 1e-4


def test_render_edge_cases():
    cam = Camera(R=np.eye(3), T=np.zeros(3), fx=50.0, fy=50.0, width=16, height=8, device="cuda:0")
    e = torch.empty((0, 3), device="cuda:0")
    img = render_gaussians(cam, e, torch.empty((0, 3, 3), device="cuda:0"), e, torch.empty(0, device="cuda:0"),
                           bg=(0.2, 0.4, 0.6))
    assert torch.allclose(img, torch.tensor([0.2, 0.4, 0.6], device="cuda:0").expand(8, 16, 3))
    # every splat behind the camera: background
    xyz = torch.tensor([[0.0, 0.0, -1.0], [0.1, 0.0, 0.01]], device="cuda:0")
    cov = torch.eye(3, device="cuda:0").expand(2, 3, 3) * 1e-3
    img = render_gaussians(cam, xyz, cov, torch.ones(2, 3, device="cuda:0"), torch.ones(2, device="cuda:0"),
                           bg=(0.0, 0.0, 0.0))
    assert float(img.abs().max()) == 0.0


def test_carried_gaussians_match_torch_restatement():
    """run_orange.deform_and_render's carrying formulas in torch vs the kernel."""
    from helpers import make_gpu_sim
    from peel_mpm_b200 import scenes
    from peel_mpm_b200.render import carry_gaussians
    sc = scenes.tiny_bar()
    sim = make_gpu_sim(sc)
    sim.run_frame(20, 0.0)
    torch.cuda.synchronize()
    rng = np.random.default_rng(3)
    g = 3000
    bind = torch.tensor(rng.integers(0, sim.n, g), device="cuda:0")
    off0 = torch.tensor(rng.normal(size=(g, 3)) * 0.01, dtype=torch.float32, device="cuda:0")
    B = rng.normal(size=(g, 3, 3)) * 0.01
    cov0 = torch.tensor(B @ np.transpose(B, (0, 2, 1)), dtype=torch.float32, device="cuda:0")
    col0 = torch.tensor(rng.uniform(size=(g, 3)), dtype=torch.float32, device="cuda:0")
    A = np.diag([2.0, 2.0, 2.0]); t = np.array([-1.0, -1.0, -0.5])
    pos, cov, col = carry_gaussians(sim, bind, off0, cov0, col0, (A, t), crack_tint=0.7)
    F = sim.F[bind]
    xw = sim.x @ torch.tensor(A.T, dtype=torch.float32, device="cuda:0") + torch.tensor(t, dtype=torch.float32,
                                                                                         device="cuda:0")
    pos_ref = xw[bind] + torch.bmm(F, off0.unsqueeze(-1)).squeeze(-1)
    cov_ref = F @ cov0 @ F.transpose(1, 2)
    col_ref = col0 * (1.0 - 0.7 * sim.d[bind].unsqueeze(1))
    assert torch.allclose(pos, pos_ref, rtol=1e-6, atol=1e-7)
    assert torch.allclose(cov, cov_ref, rtol=1e-5, atol=1e-12)
    assert torch.allclose(col, col_ref, rtol=1e-6, atol=1e-7)
    # the same map prepared once on the device, bindings not re-checked: identical
    from peel_mpm_b200.render import world_map
    p2, c2, k2 = carry_gaussians(sim, bind.to(torch.int32), off0, cov0, col0, world_map(A, t, "cuda:0"),
                                 crack_tint=0.7, check_bind=False)
    assert torch.equal(p2, pos) and torch.equal(c2, cov) and torch.equal(k2, col)
    # unchecked ids must already be int32: a wider type could wrap into range when narrowed
    with pytest.raises(TypeError):
        carry_gaussians(sim, bind, off0, cov0, col0, world_map(A, t, "cuda:0"), check_bind=False)


def test_carry_rejects_unbound_gaussians():
    from helpers import make_gpu_sim
    from peel_mpm_b200 import scenes
    from peel_mpm_b200.render import carry_gaussians
    sim = make_gpu_sim(scenes.tiny_bar())
    z3 = torch.zeros((2, 3), device="cuda:0")
    cov = torch.zeros((2, 3, 3), device="cuda:0")
    for bad in ([0, sim.n], [-1, 0]):
        with pytest.raises(IndexError):
            carry_gaussians(sim, torch.tensor(bad, device="cuda:0"), z3, cov, z3)
    pos, c, col = carry_gaussians(sim, torch.empty(0, dtype=torch.long, device="cuda:0"), z3[:0], cov[:0], z3[:0])
    assert pos.shape == (0, 3) and c.shape == (0, 3, 3) and col.shape == (0, 3)

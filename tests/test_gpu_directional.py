"""The directional (delamination) stress at interface particles, against the
reference's own validation gates for it (anisompm_py/src/1_fd_check.py:79-120,
which call reconstruction_check and release_check, anisompm.py:230-300).

The CUDA substep applies the split at registered interface particles
(anisompm.py:697-703): tau = Q tau_c Q + gI P tau_c P + gII (P tau_c Q +
Q tau_c P) with P = m m^T, m = F n0 / |F n0|, g(d) = (1 - d)^2 (1 - k_r) + k_r
and the tension gate gI = g only where m^T tau_c m > 0.  These tests step the
solver once from hand-set F with record_stress on and read the stress it used
(tau_last):

* Gate 2 (reconstruction): at d = 0 the split reproduces the plain corotated
  Kirchhoff stress tau_c = 2 mu (F - R) F^T + lam (J - 1) J I, computed here in
  float64 from an SVD of the same F;
* Gate 3 (release): at d = 1 the normal traction (where it is tensile) and the
  interfacial shear keep only the residual k_r of tau_c's, the in-plane stress
  is kept whole, and a compressive normal traction is kept whole (the tension
  gate, which the reference's release_check leaves out by design).
"""
import numpy as np
import pytest
import torch

import peel_mpm_b200 as pm

pytestmark = pytest.mark.gpu


def _random_F(rng, n):
    """The gates' recipe: F = I + 0.15 N(0,1), det F > 0.2 (1_fd_check.py:84-86)."""
    F = np.eye(3)[None] + 0.15 * rng.normal(size=(4 * n, 3, 3))
    F = F[np.linalg.det(F) > 0.2][:n]
    assert F.shape[0] == n
    return F


def _corotated(F, mu, lam):
    U, S, Vt = np.linalg.svd(F)
    R = U @ Vt
    J = np.prod(S, axis=1)
    tau = 2.0 * mu[:, None, None] * (F - R) @ np.transpose(F, (0, 2, 1))
    tau += (lam * (J - 1.0) * J)[:, None, None] * np.eye(3)[None]
    return tau


def _step_interface_block(F, normals, d, seed=0):
    """A 4,096-particle block, every particle an interface particle with the
    given normal, no damage evolution (allow False), F set by hand; one
    substep with record_stress.  Returns (tau_last, mu, lam, residual) in
    float64."""
    n = F.shape[0]
    rng = np.random.default_rng(seed)
    ng = 32
    dx = 1.0 / ng
    side = round(n ** (1.0 / 3.0))
    assert side ** 3 == n
    g = (np.arange(side) + 0.5) * dx * 0.5
    x = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3) + 0.3
    x += rng.uniform(-0.1 * dx, 0.1 * dx, size=x.shape)
    sim = pm.AnisoMPM(n_grid=ng, dt=1e-6, gravity=(0.0, 0.0, 0.0), device="cuda:0")
    sim.add_object(torch.tensor(x), torch.full((n,), (dx / 2) ** 3, dtype=torch.float64), rho=1000.0, E=1e4, nu=0.3,
                   residual=1e-3, allow_damage=False)
    mask = torch.ones(n, dtype=torch.bool, device="cuda:0")
    sim.set_interface_normals(mask, torch.tensor(normals))
    sim.F[:] = torch.tensor(F, dtype=torch.float32, device="cuda:0")
    sim.d[:] = float(d)
    sim.record_stress = True
    sim.substep(0.0)
    torch.cuda.synchronize()
    assert sim.status()["nonfinite"] == 0
    F32 = F.astype(np.float32).astype(np.float64)   # the F the substep used
    n0 = sim.n_interface.cpu().numpy().astype(np.float64)
    return (sim.tau_last.cpu().numpy().astype(np.float64), F32, n0, sim.mu.cpu().numpy().astype(np.float64),
            sim.lam.cpu().numpy().astype(np.float64), sim.residual.cpu().numpy().astype(np.float64))


def _normals(rng, n):
    v = rng.normal(size=(n, 3))
    return v / np.linalg.norm(v, axis=1, keepdims=True)


def test_gate2_reconstruction_at_zero_damage():
    """d = 0: the split rebuilds the corotated stress exactly (to float32)."""
    rng = np.random.default_rng(1)
    n = 4096
    tau, F, n0, mu, lam, _ = _step_interface_block(_random_F(rng, n), _normals(rng, n), d=0.0)
    tau_c = _corotated(F, mu, lam)
    scale = np.abs(tau_c).reshape(n, -1).max(1)
    err = np.abs(tau - tau_c).reshape(n, -1).max(1) / scale
    print(f"gate 2: max rel err {err.max():.2e}, median {np.median(err):.2e}")
    assert err.max() < 2e-5


def test_gate3_release_at_full_damage():
    """d = 1: tensile normal traction and interfacial shear released to k_r,
    in-plane stress kept; compressive normal traction kept (tension gate)."""
    rng = np.random.default_rng(2)
    n = 4096
    tau, F, n0, mu, lam, res = _step_interface_block(_random_F(rng, n), _normals(rng, n), d=1.0)
    tau_c = _corotated(F, mu, lam)
    m = np.einsum("pij,pj->pi", F, n0)
    m /= np.linalg.norm(m, axis=1, keepdims=True) + 1e-9
    Pm = m[:, :, None] * m[:, None, :]
    Qm = np.eye(3)[None] - Pm
    fro = lambda t: np.linalg.norm(t.reshape(n, -1), axis=1)
    tnc = np.einsum("pi,pij,pj->p", m, tau_c, m)
    tn1 = np.einsum("pi,pij,pj->p", m, tau, m)
    shc = fro(Pm @ tau_c @ Qm + Qm @ tau_c @ Pm)
    sh1 = fro(Pm @ tau @ Qm + Qm @ tau @ Pm)
    ipc = fro(Qm @ tau_c @ Qm)
    ip1 = fro(Qm @ tau @ Qm)
    scale = np.abs(tau_c).reshape(n, -1).max(1)
    # ratios only where the compared component stands well above the float32
    # rounding of tau (~1e-7 of its largest entry; the released part is 1e-3)
    ok_n = np.abs(tnc) > 5e-2 * scale
    ok_s = shc > 5e-2 * scale
    ok_i = ipc > 5e-2 * scale
    tensile = tnc > 0
    normal_kept_t = np.abs(tn1 / tnc)[ok_n & tensile]
    normal_kept_c = np.abs(tn1 / tnc)[ok_n & ~tensile]
    shear_kept = (sh1 / shc)[ok_s]
    inplane_kept = (ip1 / ipc)[ok_i]
    r = float(res[0])
    print(f"gate 3: normal kept (tensile) {normal_kept_t.max():.4e}, (compressive) {normal_kept_c.min():.4f}, "
          f"shear kept {shear_kept.max():.4e}, in-plane kept {inplane_kept.min():.6f}..{inplane_kept.max():.6f}")
    assert min(normal_kept_t.size, normal_kept_c.size, shear_kept.size, inplane_kept.size) > n // 10
    assert np.all(np.abs(normal_kept_t - r) < 2e-2 * r)      # released to the residual
    assert np.all(np.abs(shear_kept - r) < 2e-2 * r)
    assert np.all(np.abs(normal_kept_c - 1.0) < 1e-4)        # the tension gate keeps compression
    assert np.all(np.abs(inplane_kept - 1.0) < 1e-4)         # the sheet stays coherent in-plane

"""Golden gradients from the reference solver's own PyTorch autograd.

Run where a checkout of the reference is available (it is read, never
written); its ``anisompm_py/src`` directory is given by ``--ref`` or by the
environment variable PEELMPM_REFERENCE_SRC:

    python tests/golden/make_grad_golden.py --ref <checkout>/anisompm_py/src

For each case the reference ``AnisoMPM`` (anisompm.py:303-807) runs on the
CPU in float64 with per-particle Young's modulus E, fiber directions,
critical stress sigma_c and initial velocity v0 as autograd leaves: mu, lam
and A0 are formed from them with add_object's formulas (anisompm.py:371-372,
395-404) and assigned to the solver before the first substep.  The target is
the final position of the same scene run with E * 1.2, fibers rotated 15
degrees about z and sigma_c * 0.8; the loss is the mean over particles of the
squared distance to it.  The script saves the loss, the final positions, the
target and dL/dE, dL/dfibers, dL/dsigma_c, dL/dv0.

The reference ``sym_eig`` (anisompm.py:48-95) divides by the off-diagonal
entry before masking skipped rotations with torch.where, so its backward is
NaN wherever an entry is exactly zero (every particle at F = I).  It is
replaced for this run by the same iteration with the division guarded
(forward values are bit-identical: the guarded value only feeds the masked
branch).

The GPU box has no reference checkout; tests read only the saved file.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import sys

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, HERE)

from peel_mpm_b200 import scenes  # noqa: E402
from make_golden import ref_grip, make_ref_collider  # noqa: E402

# name -> (scene factory, substeps)
CASES = {
    "tiny_bar": (scenes.tiny_bar, 40),
    "plain_small": (scenes.plain_small, 20),
}


def guarded_sym_eig(A: torch.Tensor, sweeps: int = 5):
    """The reference iteration with zeta's division guarded for autograd."""
    A = torch.nan_to_num(0.5 * (A + A.transpose(1, 2)))
    N = A.shape[0]
    Am = A.clone()
    V = torch.eye(3, device=A.device, dtype=A.dtype).expand(N, 3, 3).contiguous()
    for _ in range(sweeps):
        for (p, q) in ((0, 1), (0, 2), (1, 2)):
            r = 3 - p - q
            app = Am[:, p, p].clone(); aqq = Am[:, q, q].clone(); apq = Am[:, p, q].clone()
            apr = Am[:, p, r].clone(); aqr = Am[:, q, r].clone()
            live = apq.abs() > 1e-30
            apq_s = torch.where(live, apq, torch.ones_like(apq))
            zeta = (aqq - app) / (2.0 * apq_s)
            sgn = torch.where(zeta >= 0, torch.ones_like(zeta), -torch.ones_like(zeta))
            t = sgn / (zeta.abs() + torch.sqrt(1.0 + zeta * zeta))
            t = torch.where(live, t, torch.zeros_like(t))
            c = 1.0 / torch.sqrt(1.0 + t * t); s = c * t
            Am[:, p, p] = c * c * app - 2.0 * s * c * apq + s * s * aqq
            Am[:, q, q] = s * s * app + 2.0 * s * c * apq + c * c * aqq
            Am[:, p, q] = 0.0; Am[:, q, p] = 0.0
            npr = c * apr - s * aqr; nqr = s * apr + c * aqr
            Am[:, p, r] = npr; Am[:, r, p] = npr
            Am[:, q, r] = nqr; Am[:, r, q] = nqr
            vp = V[:, :, p].clone(); vq = V[:, :, q].clone()
            V[:, :, p] = c.unsqueeze(1) * vp - s.unsqueeze(1) * vq
            V[:, :, q] = s.unsqueeze(1) * vp + c.unsqueeze(1) * vq
    evals = torch.diagonal(Am, dim1=1, dim2=2)
    evals, idx = torch.sort(evals, dim=1)
    V = torch.gather(V, 2, idx.unsqueeze(1).expand(-1, 3, -1))
    return evals, V


def rot_z(deg):
    a = math.radians(deg)
    return np.array([[math.cos(a), -math.sin(a), 0.0], [math.sin(a), math.cos(a), 0.0], [0.0, 0.0, 1.0]])


def run(mod, sc, n_steps, E, fib, sig, v0):
    """Final positions of the reference solver with the given parameters."""
    dt = torch.float64
    sim = mod.AnisoMPM(n_grid=sc.n_grid, grid_lim=sc.grid_lim, dt=sc.dt, gravity=tuple(sc.gravity),
                       grid_damp=sc.grid_damp, f_clamp=sc.f_clamp, damage_every=sc.damage_every,
                       device="cpu", dtype=dt)
    scenes.apply_scene(sim, sc, ref_grip, make_ref_collider(mod), torch)
    nu = sc.nu
    sim.mu = E / (2.0 * (1.0 + nu))
    sim.lam = E * nu / ((1.0 + nu) * (1.0 - 2.0 * nu))
    a = fib / (fib.norm(dim=1, keepdim=True) + 1e-12)
    eye = torch.eye(3, dtype=dt).expand(sc.n, 3, 3)
    sim.A0 = eye + sc.alpha * a.unsqueeze(2) * a.unsqueeze(1)
    sim.sigma_c = sig * 1.0
    sim.v = v0 * 1.0
    for s in range(n_steps):
        sim.substep(s * sc.dt)
    return sim.x


# one-substep cases: (scene, forward substeps before the differentiated one)
ONESTEP = {"tiny_bar": (5, 25, 38), "colliders_drop": (20,), "limit_drop": (57,), "clamp_drop": (14,),
           "interface_peel": (15,)}
COMPACT = ("colliders_drop", "limit_drop", "clamp_drop", "interface_peel")
ONESTEP_SCENES = {"tiny_bar": scenes.tiny_bar, "colliders_drop": scenes.colliders_drop,
                  "limit_drop": scenes.limit_drop, "clamp_drop": scenes.clamp_drop,
                  "interface_peel": scenes.interface_peel}
STATE = ("x", "v", "F", "C", "d", "lap", "D_hist")
PARAMS = ("mu", "lam", "sigma_c", "A0")


def onestep(mod, name, factory, pre_steps, out, meta, tag, compact=False):
    """Adjoint of one substep from a state with damage under way: random
    adjoints of the post-substep state, gradients of their inner product with
    the post state with respect to the pre state and the per-particle
    parameters.  compact: the pre state is rounded to float32 before the
    substep (the GPU path starts from float32 values) and the arrays are
    saved in float32, without the adjoints, which the test draws again from
    the same seed (numpy's default_rng(7), normal, in STATE order)."""
    sc = factory()
    dt = torch.float64
    sim = mod.AnisoMPM(n_grid=sc.n_grid, grid_lim=sc.grid_lim, dt=sc.dt, gravity=tuple(sc.gravity),
                       grid_damp=sc.grid_damp, f_clamp=sc.f_clamp, damage_every=sc.damage_every,
                       device="cpu", dtype=dt)
    scenes.apply_scene(sim, sc, ref_grip, make_ref_collider(mod), torch)
    with torch.no_grad():
        for s in range(pre_steps):
            sim.substep(s * sc.dt)
    leaves = {}
    for k in STATE + PARAMS:
        t = getattr(sim, k).detach().clone()
        if compact:
            t = t.to(torch.float32).to(dt)
        out[f"{tag}/pre_{k}"] = t.numpy().astype(np.float32) if compact else t.numpy()
        leaves[k] = t.requires_grad_(True)
        setattr(sim, k, leaves[k] * 1.0)
    step = sim._step
    sim.substep(pre_steps * sc.dt)
    rng = np.random.default_rng(7)
    total = 0.0
    for k in STATE:
        post = getattr(sim, k)
        w = torch.tensor(rng.normal(size=tuple(post.shape)), dtype=dt)
        if not compact:
            out[f"{tag}/bar_{k}"] = w.numpy()
        out[f"{tag}/post_{k}"] = post.detach().numpy().astype(np.float32 if compact else np.float64)
        total = total + (w * post).sum()
    total.backward()
    for k in STATE + PARAMS:
        g = leaves[k].grad
        g = (torch.zeros_like(leaves[k]) if g is None else g).numpy()
        out[f"{tag}/grad_{k}"] = g.astype(np.float32) if compact else g
    meta[tag] = {"pre_steps": pre_steps, "step": step, "time": pre_steps * sc.dt, "n": sc.n,
                 "bars": "seed 7" if compact else "saved"}
    print(tag, {k: float(np.linalg.norm(out[f"{tag}/grad_{k}"])) for k in STATE + PARAMS}, flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("PEELMPM_REFERENCE_SRC"),
                    help="the reference's anisompm_py/src directory (default: $PEELMPM_REFERENCE_SRC)")
    ap.add_argument("--out", default=os.path.join(HERE, "reference_grads.npz"))
    ap.add_argument("--only", nargs="*", default=None,
                    help="compute only these one-substep cases and merge them into --out")
    args = ap.parse_args()
    if not args.ref:
        ap.error("give --ref or set PEELMPM_REFERENCE_SRC")
    sys.path.insert(0, args.ref)
    import anisompm as mod  # the unmodified reference module
    mod.sym_eig = guarded_sym_eig
    torch.set_num_threads(os.cpu_count() or 1)
    out, meta = {}, {}
    for name, (factory, n_steps) in CASES.items():
        if args.only:
            break
        sc = factory()
        n = sc.n
        E0 = torch.tensor(sc.E, dtype=torch.float64)
        fib0 = torch.tensor(sc.fibers, dtype=torch.float64)
        sig0 = torch.tensor(sc.sigma_c, dtype=torch.float64)
        v00 = torch.zeros(n, 3, dtype=torch.float64)
        with torch.no_grad():
            target = run(mod, sc, n_steps, E0 * 1.2, fib0 @ torch.tensor(rot_z(15.0)).t(), sig0 * 0.8, v00)
        E = E0.clone().requires_grad_(True)
        fib = fib0.clone().requires_grad_(True)
        sig = sig0.clone().requires_grad_(True)
        v0 = v00.clone().requires_grad_(True)
        xT = run(mod, sc, n_steps, E, fib, sig, v0)
        loss = ((xT - target) ** 2).sum(1).mean()
        loss.backward()
        for k, v in (("xT", xT.detach()), ("target", target), ("E", E.grad), ("fibers", fib.grad),
                     ("sigma_c", sig.grad), ("v0", v0.grad)):
            out[f"{name}/{k}"] = v.numpy()
        meta[name] = {"n_steps": n_steps, "loss": float(loss), "n": n,
                      "grad_norms": {k: float(g.norm()) for k, g in (("E", E.grad), ("fibers", fib.grad),
                                                                   ("sigma_c", sig.grad), ("v0", v0.grad))}}
        print(name, meta[name], flush=True)
    for name, pres in ONESTEP.items():
        if args.only and name not in args.only:
            continue
        for pre in pres:
            onestep(mod, name, ONESTEP_SCENES[name], pre, out, meta, f"one_{name}_{pre}", compact=name in COMPACT)
    if args.only and os.path.exists(args.out):   # merge into the existing file (cases computed now replace theirs)
        old = np.load(args.out)
        keep = [k for k in old.files if k.split("/")[0] not in {f"one_{n}_{p}" for n in args.only
                                                                 for p in ONESTEP.get(n, ())}]
        out = {**{k: old[k] for k in keep}, **out}
        with open(args.out.replace(".npz", ".json")) as f:
            meta = {**json.load(f), **meta}
    np.savez_compressed(args.out, **out)
    with open(args.out.replace(".npz", ".json"), "w") as f:
        json.dump(meta, f, indent=1)


if __name__ == "__main__":
    main()

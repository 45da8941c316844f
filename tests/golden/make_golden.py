"""Generate golden fixtures by running the reference solver itself.

Run where a checkout of the reference is available (it is read, never
written); its ``anisompm_py/src`` directory is given by ``--ref`` or by the
environment variable PEELMPM_REFERENCE_SRC:

    python tests/golden/make_golden.py --ref <checkout>/anisompm_py/src [--part all|sweeps]

``--part sweeps`` writes only ``reference_sym_eig_sweeps.npz``: the reference
``sym_eig`` at sweep counts other than the default 5.

For each seeded scene of ``peel_mpm_b200.scenes`` the reference ``AnisoMPM``
(anisompm.py:303-807) runs on the CPU in float32 (and float64 where listed),
with grips as particle_bc closures and colliders from its own
``halfspace_collider``/``sphere_collider`` factories.  Snapshots of the
particle state are saved (every ``stride``-th particle) as compressed npz.
Also saved: the reference ``sym_eig`` on a batch of random and degenerate
symmetric matrices (the ``_la_selftest`` recipe, anisompm.py:871-886), the
reference binning keys (``_weights`` base + ``_node_index``), and the
reference's own scatter-order noise envelope (particle order permuted).

The GPU box has no reference checkout; tests read only these files.
"""
from __future__ import annotations

import argparse
import hashlib
import json
import os
import sys
import time

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from peel_mpm_b200 import scenes  # noqa: E402

FIELDS = ("x", "v", "F", "C", "d", "lap", "D_hist")
DIAG = ("phi", "phi_shear", "tau_last", "J_last")

# scene name -> (fp32 snapshot steps, fp64 snapshot steps, particle stride, diagnostics)
PLAN = {
    "tiny_bar": ([1, 10, 50, 200], [200], 1, True),
    "plain_small": ([1, 50, 200], [200], 8, False),
    "knobs_drop": ([10, 60], [60], 1, True),
    "interface_peel": ([10, 60], [60], 1, True),
}


def scene_hash(sc):
    h = hashlib.sha256()
    for a in (sc.x, sc.vol, sc.E, sc.sigma_c):
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()[:16]


def ref_grip(mask, vel, ramp):
    def bc(s, t):
        f = scenes.grip_factor(t, ramp)
        s.v[mask] = torch.tensor([vel[0] * f, vel[1] * f, vel[2] * f], dtype=s.dtype)
    return bc


def make_ref_collider(mod):
    def mk(spec):
        if spec.kind == "halfspace":
            return mod.halfspace_collider(spec.origin_fn(), list(spec.normal), mode=spec.mode,
                                          friction=spec.friction)
        return mod.sphere_collider(spec.origin_fn(), spec.radius, mode=spec.mode, friction=spec.friction)
    return mk


def build_ref(mod, sc, dtype, perm=None):
    if perm is not None:
        sc = permute_scene(sc, perm)
    sim = mod.AnisoMPM(n_grid=sc.n_grid, grid_lim=sc.grid_lim, dt=sc.dt, gravity=tuple(sc.gravity),
                       grid_damp=sc.grid_damp, f_clamp=sc.f_clamp, damage_every=sc.damage_every,
                       device="cpu", dtype=dtype)
    scenes.apply_scene(sim, sc, ref_grip, make_ref_collider(mod), torch)
    return sim


def permute_scene(sc, perm):
    import copy
    s2 = copy.copy(sc)
    s2.x = sc.x[perm]; s2.vol = sc.vol[perm]; s2.E = sc.E[perm]; s2.sigma_c = sc.sigma_c[perm]
    s2.fibers = None if sc.fibers is None else sc.fibers[perm]
    s2.d0 = None if sc.d0 is None else sc.d0[perm]
    s2.allow = None if sc.allow is None else sc.allow[perm]
    s2.grips = [scenes.Grip(g.mask[perm], g.velocity, g.ramp) for g in sc.grips]
    if sc.interface is not None:
        s2.interface = (sc.interface[0][perm], sc.interface[1][perm])
    return s2


def snap(sim, stride, diag):
    out = {}
    for f in FIELDS:
        out[f] = getattr(sim, f).detach().cpu().numpy()[::stride].copy()
    if diag:
        for f in DIAG:
            if hasattr(sim, f):
                out[f] = getattr(sim, f).detach().cpu().numpy()[::stride].copy()
    return out


def run_scene(mod, name, steps32, steps64, stride, diag, out):
    sc = scenes.SCENES[name]()
    meta = {"scene": name, "n": sc.n, "stride": stride, "hash": scene_hash(sc)}
    for dtype, steps, tag in ((torch.float32, steps32, "f32"), (torch.float64, steps64, "f64")):
        if not steps:
            continue
        sim = build_ref(mod, sc, dtype)
        t0 = time.time()
        for s in range(max(steps)):
            sim.substep(s * sim.dt)
            if s + 1 in steps:
                for k, v in snap(sim, stride, diag and dtype == torch.float32).items():
                    out[f"{name}/{tag}/{s + 1}/{k}"] = v
        meta[f"secs_{tag}"] = round(time.time() - t0, 2)
        print(f"  {name} {tag}: {max(steps)} steps in {meta[f'secs_{tag}']} s", flush=True)
    return meta


def noise_envelope(mod, name, steps):
    """Relative L2 between the reference run on permuted vs original order."""
    sc = scenes.SCENES[name]()
    rng = np.random.default_rng(1234)
    perm = rng.permutation(sc.n)
    a = build_ref(mod, sc, torch.float32)
    b = build_ref(mod, sc, torch.float32, perm=perm)
    for s in range(steps):
        a.substep(s * a.dt); b.substep(s * b.dt)
    inv = np.argsort(perm)
    env = {}
    for f in FIELDS:
        xa = getattr(a, f).numpy().astype(np.float64)
        xb = getattr(b, f).numpy().astype(np.float64)[inv]
        env[f] = float(np.linalg.norm(xa - xb) / max(np.linalg.norm(xa), 1e-30))
    return env


def sym_eig_golden(mod, out, n=4096, seed=0):
    g = torch.Generator().manual_seed(seed)
    B = torch.randn(n, 3, 3, generator=g, dtype=torch.float64)
    A = 0.5 * (B + B.transpose(1, 2))
    A[0] = torch.tensor([[0.0, 2, 0], [2, 0, 0], [0, 0, 0]], dtype=torch.float64)
    A[1] = 3.0 * torch.eye(3, dtype=torch.float64)
    A[2] = torch.eye(3, dtype=torch.float64)
    A[3] = torch.diag(torch.tensor([2.0, 2.0, 5.0], dtype=torch.float64))
    # right Cauchy-Green tensors of stretched rotations, the substep's actual input
    Q = torch.linalg.qr(torch.randn(n // 4, 3, 3, generator=g, dtype=torch.float64)).Q
    S = 0.5 + torch.rand(n // 4, 3, generator=g, dtype=torch.float64)
    Fm = Q @ torch.diag_embed(S)
    A[-(n // 4):] = Fm.transpose(1, 2) @ Fm
    A32 = A.to(torch.float32)
    ev, V = mod.sym_eig(A32)
    out["sym_eig/A"] = A32.numpy()
    out["sym_eig/evals"] = ev.numpy()
    out["sym_eig/evecs"] = V.numpy()


SWEEP_COUNTS = (0, 1, 3, 7, 12)


def sym_eig_sweeps_golden(mod, out, n=2048, seed=3):
    """The reference sym_eig with `sweeps` other than 5 (anisompm.py:48, 68)."""
    g = torch.Generator().manual_seed(seed)
    B = torch.randn(n, 3, 3, generator=g, dtype=torch.float64)
    A = 0.5 * (B + B.transpose(1, 2))
    A[0] = torch.diag(torch.tensor([2.0, 2.0, 5.0], dtype=torch.float64))
    A[1] = torch.tensor([[0.0, 2, 0], [2, 0, 0], [0, 0, 0]], dtype=torch.float64)
    A32 = A.to(torch.float32)
    out["sym_eig_sweeps/A"] = A32.numpy()
    for k in SWEEP_COUNTS:
        ev, V = mod.sym_eig(A32, sweeps=k)
        out[f"sym_eig_sweeps/{k}/evals"] = ev.numpy()
        out[f"sym_eig_sweeps/{k}/evecs"] = V.numpy()


def bin_golden(mod, out):
    for name in ("plain_small", "tiny_bar"):
        sc = scenes.SCENES[name]()
        sim = build_ref(mod, sc, torch.float32)
        for s in range(2):
            base, fx, w, w2 = sim._weights(sim.x)
            keys = sim._node_index(base).numpy()
            out[f"bin/{name}/{s}/x"] = sim.x.numpy().copy()
            out[f"bin/{name}/{s}/keys"] = keys.astype(np.int64)
            out[f"bin/{name}/{s}/perm"] = torch.argsort(torch.from_numpy(keys), stable=True).numpy().astype(np.int64)
            for _ in range(25):
                sim.substep(sim._step * sim.dt)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("PEELMPM_REFERENCE_SRC"),
                    help="the reference's anisompm_py/src directory (default: $PEELMPM_REFERENCE_SRC)")
    ap.add_argument("--skip-noise", action="store_true")
    ap.add_argument("--part", default="all", choices=["all", "sweeps"])
    args = ap.parse_args()
    if not args.ref:
        ap.error("give --ref or set PEELMPM_REFERENCE_SRC")
    sys.path.insert(0, args.ref)
    import anisompm as mod  # the reference solver, unmodified

    torch.set_num_threads(os.cpu_count() or 1)
    if args.part == "sweeps":
        out = {}
        sym_eig_sweeps_golden(mod, out)
        np.savez_compressed(os.path.join(HERE, "reference_sym_eig_sweeps.npz"), **out)
        print("wrote", len(out), "arrays")
        return
    out = {}
    meta = {"torch": torch.__version__, "numpy": np.__version__, "scenes": {}}
    for name, (s32, s64, stride, diag) in PLAN.items():
        meta["scenes"][name] = run_scene(mod, name, s32, s64, stride, diag, out)
    sym_eig_golden(mod, out)
    bin_golden(mod, out)
    if not args.skip_noise:
        meta["noise_envelope"] = {"plain_small_200": noise_envelope(mod, "plain_small", 200),
                                  "tiny_bar_200": noise_envelope(mod, "tiny_bar", 200)}
        print("  noise:", json.dumps(meta["noise_envelope"]), flush=True)
    np.savez_compressed(os.path.join(HERE, "reference_goldens.npz"), **out)
    with open(os.path.join(HERE, "reference_goldens.json"), "w") as f:
        json.dump(meta, f, indent=1, sort_keys=True)
    print("wrote", len(out), "arrays")


if __name__ == "__main__":
    main()

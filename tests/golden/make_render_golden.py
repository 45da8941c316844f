"""Golden images from the reference's own Gaussian-splat renderer.

Run where a checkout of the reference is available (it is read, never
written); its ``anisompm_py/src`` directory is given by ``--ref`` or by the
environment variable PEELMPM_REFERENCE_SRC:

    python tests/golden/make_render_golden.py --ref <checkout>/anisompm_py/src

The reference ``render_gaussians`` (render.py:71-162: EWA projection, soft
z-buffer in two passes, coverage compositing) renders seeded synthetic
gaussians on the CPU in float32: an anisotropic cloud in front of the camera
with some splats behind it, partly outside the frame and one oversized
splat (dropped by max_raw_radius); the cases vary tau, r_max, the scale
modifier, the background, the random downsampling and the overdraw.  Inputs,
camera and images are saved;
the GPU box has no reference checkout, the tests read only this file.
"""
from __future__ import annotations

import argparse
import os
import sys

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))


def scene(seed, n):
    rng = np.random.default_rng(seed)
    xyz = rng.normal(size=(n, 3)) * np.array([0.35, 0.25, 0.3]) + np.array([0.0, 0.0, 2.5])
    xyz[: n // 20, 2] = rng.uniform(-1.0, 0.02, n // 20)          # behind / at the camera plane
    xyz[n // 20: n // 10, 0] += rng.choice([-3.0, 3.0], n // 20)  # far outside the frame
    A = rng.normal(size=(n, 3, 3)) * 0.02
    cov = A @ np.transpose(A, (0, 2, 1)) + 1e-5 * np.eye(3)
    cov[-1] = np.eye(3) * 4.0                                      # a blown-up splat
    color = rng.uniform(0, 1, size=(n, 3))
    opacity = rng.uniform(0.2, 1.0, size=n)
    th = 0.3
    R = np.array([[np.cos(th), 0, np.sin(th)], [0, 1, 0], [-np.sin(th), 0, np.cos(th)]])
    T = np.array([0.1, -0.05, 0.2])
    return xyz, cov, color, opacity, R, T


CASES = {
    # name: (seed, n, W, H, fx, fy, kwargs)
    "cloud_default": (0, 3000, 128, 96, 150.0, 140.0, {}),
    "cloud_tau_rmax": (1, 5000, 160, 120, 220.0, 220.0, {"tau": 0.05, "r_max": 16, "scale_modifier": 1.3,
                                                         "bg": (0.1, 0.2, 0.3)}),
    # the reference's random subset (torch.randperm on a seeded CPU generator)
    "cloud_downsample": (2, 6000, 96, 96, 120.0, 120.0, {"downsample": 2500, "seed": 7}),
    # heavy overdraw (hundreds of splats per pixel at r_max 24) on a frame that
    # is not a multiple of the 8-pixel screen tile
    "cloud_dense": (3, 10000, 101, 75, 160.0, 160.0, {"r_max": 24, "scale_modifier": 2.6}),
}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("PEELMPM_REFERENCE_SRC"),
                    help="the reference's anisompm_py/src directory (default: $PEELMPM_REFERENCE_SRC)")
    ap.add_argument("--out", default=os.path.join(HERE, "reference_render.npz"))
    args = ap.parse_args()
    if not args.ref:
        ap.error("give --ref or set PEELMPM_REFERENCE_SRC")
    sys.path.insert(0, args.ref)
    import render as ref   # the unmodified reference module
    out = {}
    for name, (seed, n, W, H, fx, fy, kw) in CASES.items():
        xyz, cov, color, opacity, R, T = scene(seed, n)
        cam = ref.Camera(R=R, T=T, fx=fx, fy=fy, width=W, height=H, device="cpu")
        f = lambda a: torch.tensor(a, dtype=torch.float32)
        img = ref.render_gaussians(cam, f(xyz), f(cov), f(color), f(opacity), **kw)
        for k, v in (("xyz", xyz), ("cov", cov), ("color", color), ("opacity", opacity), ("R", R), ("T", T),
                     ("img", img.numpy())):
            out[f"{name}/{k}"] = np.asarray(v, np.float32)
        out[f"{name}/cam"] = np.array([W, H, fx, fy], np.float64)
        print(name, img.shape, float(img.mean()))
    np.savez_compressed(args.out, **out)


if __name__ == "__main__":
    main()

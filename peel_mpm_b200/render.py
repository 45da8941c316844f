"""Gaussian-splat renderer on the GPU with the reference's API (render.py).

``Camera`` and ``render_gaussians`` keep the signatures of the reference's
pure-PyTorch renderer (render.py:21-162), used by its orange demo to draw the
simulated particles as gaussians; the work runs in ``pm_render_gaussians``
(EWA projection, two-pass soft z-buffer, coverage compositing) and the image
is a (H, W, 3) CUDA tensor.
"""
from __future__ import annotations

import ctypes as C
import json

import numpy as np
import torch

from . import _lib


class Camera:
    def __init__(self, json_path=None, R=None, T=None, fx=None, fy=None, width=None, height=None,
                 device="cuda:0"):
        if json_path is not None:
            with open(json_path) as f:
                c = json.load(f)
            R, T = np.array(c["R"], np.float32), np.array(c["T"], np.float32)
            fx, fy = float(c["fx"]), float(c["fy"])
            width, height = int(c["width"]), int(c["height"])
        self.device = torch.device(device)
        self.R = torch.tensor(np.asarray(R, np.float32), device=device)
        self.T = torch.tensor(np.asarray(T, np.float32), device=device)
        self.fx, self.fy = fx, fy
        self.W, self.H = width, height
        self.cx, self.cy = width / 2.0, height / 2.0

    def world_to_cam(self, X):
        return X @ self.R + self.T

    def _struct(self):
        # R and T live on the device; their host copy is read back only when a
        # tensor is replaced (the cache holds the tensor objects themselves and
        # compares identity), modified in place (version counter) or given new
        # storage through .data (data pointer), so rendering a sequence of
        # frames does not synchronise
        cached = getattr(self, "_rt_cache", None)
        R, T = self.R, self.T
        fresh = cached is not None and cached[0] is R and cached[1] is T and \
            cached[2] == (R._version, T._version, R.data_ptr(), T.data_ptr())
        if not fresh:
            self._rt_host = (R.detach().cpu().numpy().reshape(-1).tolist(),
                             T.detach().cpu().numpy().reshape(-1).tolist())
            self._rt_cache = (R, T, (R._version, T._version, R.data_ptr(), T.data_ptr()))
        c = _lib.pm_camera()
        for k, v in enumerate(self._rt_host[0]):
            c.R[k] = v
        for k, v in enumerate(self._rt_host[1]):
            c.T[k] = v
        c.fx, c.fy = float(self.fx), float(self.fy)
        c.width, c.height = int(self.W), int(self.H)
        return c


@torch.no_grad()
def render_gaussians(cam: Camera, xyz, cov3d, color, opacity, bg=(1.0, 1.0, 1.0), scale_modifier=1.0, r_max=10,
                     tau=None, near=0.05, downsample=None, seed=0, chunk=500_000, max_raw_radius=70):
    """(H, W, 3) image in [0, 1] of the gaussians (xyz (N,3), cov3d (N,3,3),
    color (N,3)).  ``opacity`` is accepted and, as in the reference, does not
    enter the compositing; ``chunk`` (the reference's memory bound) has no
    effect here: (splat, pixel) pairs are never materialised, only per-tile
    splat lists."""
    dev = cam.device
    if downsample is not None and downsample < xyz.shape[0]:
        g = torch.Generator(device="cpu").manual_seed(seed)
        sel = torch.randperm(xyz.shape[0], generator=g)[:downsample].to(dev)
        xyz, cov3d, color = xyz[sel], cov3d[sel], color[sel]
    f32 = lambda t: torch.as_tensor(t, device=dev).to(torch.float32).contiguous()
    xyz, cov3d, color = f32(xyz), f32(cov3d).reshape(-1, 9), f32(color)
    n = xyz.shape[0]
    lib = _lib.load()
    rp = _lib.pm_render_params()
    for k in range(3):
        rp.bg[k] = float(bg[k])
    rp.scale_modifier = float(scale_modifier)
    rp.r_max = int(r_max)
    rp.tau = -1.0 if tau is None else float(tau)
    rp.near = float(near)
    rp.max_raw_radius = float(max_raw_radius)
    need = C.c_size_t(0)
    _lib.check(lib.pm_render_workspace_size(n, int(cam.W), int(cam.H), int(r_max), C.byref(need)),
               "pm_render_workspace_size")
    ws = torch.empty(need.value, dtype=torch.uint8, device=dev)
    img = torch.empty((cam.H, cam.W, 3), dtype=torch.float32, device=dev)
    camst = cam._struct()
    with torch.cuda.device(dev):
        _lib.check(lib.pm_render_gaussians(C.byref(camst), C.byref(rp), xyz.data_ptr(), cov3d.data_ptr(),
                                           color.data_ptr(), n, img.data_ptr(), ws.data_ptr(), need.value,
                                           torch.cuda.current_stream().cuda_stream), "pm_render_gaussians")
    return img


def to_uint8(img):
    return (img.clamp(0, 1) * 255).to(torch.uint8).cpu().numpy()


def world_map(A=None, t=None, device="cuda:0"):
    """The affine sim-to-world map x -> A x + t as the (3, 4) float32 device
    tensor [A | t] that ``carry_gaussians`` takes (identity by default)."""
    A = np.eye(3) if A is None else np.asarray(A, np.float64).reshape(3, 3)
    t = np.zeros(3) if t is None else np.asarray(t, np.float64).reshape(3)
    return torch.tensor(np.concatenate([A, t[:, None]], 1), dtype=torch.float32, device=device)


def carry_gaussians(sim, bind, off0, cov0, color0, sim_to_world=None, crack_tint=0.0, check_bind=True):
    """Gaussians carried by the solver's particles (run_orange.py:116-133):
    positions ``A x + t + F off0``, covariances ``F cov0 F^T`` and colours
    darkened by damage, for gaussian i bound to particle ``bind[i]``.
    ``sim_to_world`` is ``(A (3,3), t (3,))``, a (3, 4) device tensor from
    ``world_map`` (no host-to-device copy per call), or None (identity).
    ``check_bind`` range-checks the bindings, which synchronises the host once;
    a caller that checked them already passes False together with ``bind`` as
    an int32 tensor on the solver's device (an out-of-range id then gives NaN
    outputs; a wider integer type is rejected on that path, since narrowing
    it unchecked could wrap an id into range).  Arrays given as numpy are
    copied to the device on every call: keep ``off0``, ``cov0`` and ``color0``
    as device tensors for per-frame use."""
    dev = sim.device
    f32 = lambda a: torch.as_tensor(a, device=dev).to(torch.float32).contiguous()
    bind = torch.as_tensor(bind, device=dev)
    g = bind.shape[0]
    if check_bind:
        if g and (int(bind.min()) < 0 or int(bind.max()) >= sim.n):   # torch indexing would raise too
            raise IndexError(f"gaussian bindings must lie in [0, {sim.n})")
    elif bind.dtype != torch.int32:
        raise TypeError("with check_bind=False, bind must be an int32 tensor (ids checked by the caller)")
    bind = bind.to(torch.int32).contiguous()
    off0, cov0, color0 = f32(off0), f32(cov0).reshape(-1, 9), f32(color0)
    if off0.shape != (g, 3) or cov0.shape != (g, 9) or color0.shape != (g, 3):
        raise ValueError("off0 (n,3), cov0 (n,3,3) and color0 (n,3) must match bind (n,)")
    if isinstance(sim_to_world, torch.Tensor):
        aff = sim_to_world
        if aff.shape != (3, 4) or aff.dtype != torch.float32 or aff.device != torch.device(dev) or \
                not aff.is_contiguous():
            raise ValueError("sim_to_world tensor must be a contiguous (3, 4) float32 tensor on the solver's device")
    else:
        A, t = (None, None) if sim_to_world is None else sim_to_world
        aff = world_map(A, t, dev)
    pos = torch.empty((g, 3), dtype=torch.float32, device=dev)
    cov = torch.empty((g, 3, 3), dtype=torch.float32, device=dev)
    col = torch.empty((g, 3), dtype=torch.float32, device=dev)
    P = sim._particles()
    lib = _lib.load()
    with torch.cuda.device(dev):
        _lib.check(lib.pm_carry_gaussians(C.byref(P), bind.data_ptr(), off0.data_ptr(), cov0.data_ptr(),
                                          color0.data_ptr(), g, aff.data_ptr(), float(crack_tint), pos.data_ptr(),
                                          cov.data_ptr(), col.data_ptr(), torch.cuda.current_stream().cuda_stream),
                   "pm_carry_gaussians")
    return pos, cov, col

"""AnisoMPM solver: the reference's state/step API over the sm_100a kernels.

``AnisoMPM`` keeps the constructor, ``add_object``, the ``set_*`` setters,
``substep``, ``run_frame`` and the attribute names of the reference class
(anisompm_py/src/anisompm.py:303-807), so ``from peel_mpm_b200 import
AnisoMPM`` replaces ``from anisompm import AnisoMPM`` for the plain substep.

Storage.  Particle state lives in one float32 device tensor of planes
(structure-of-arrays, each plane padded to a multiple of 64 floats); the
attributes ``x``, ``v``, ``F``, ``C``, ``d``, ... are reference-shaped views
((N,3), (N,3,3), (N,)) into it, so in-place writes such as
``sim.mu[mask] = ...`` or ``sim.allow[left] = False`` reach the next substep
exactly as in the reference.  Assigning an attribute copies into the planes.
Unlike the reference, which rebinds ``self.x`` etc. every substep, a view
obtained before a substep shows the new values after it: ``clone()`` what
must be kept.

Differences that are errors rather than fallbacks:
  * ``dtype`` must be float32 and ``device`` a CUDA device (sm_100);
  * ``colliders`` accept only the objects returned by this module's
    ``halfspace_collider`` / ``sphere_collider`` (same signatures as the
    reference factories, anisompm.py:828-867);
  * ``particle_bc`` accepts ``grip_bc`` descriptors (run inside the P2G
    kernel) and, in eager substeps only, plain callables ``bc(sim, time)``
    as in the reference (their torch ops run on the GPU before the kernels).
``tau_last`` / ``J_last`` (anisompm.py:705-706) are recorded only when
``record_stress`` is True, since they cost 40 bytes per particle per
substep of writes.
"""
from __future__ import annotations

import ctypes as C
import math
from typing import Callable, Optional, Sequence

import torch

from . import _lib

# plane offsets in the float32 store (structure-of-arrays)
_PLANES = {}
_o = 0
for _name, _k in (("x", 3), ("v", 3), ("F", 9), ("C", 9), ("d", 1), ("lap", 1), ("D_hist", 1),
                  ("vol0", 1), ("mass", 1), ("mu", 1), ("lam", 1), ("sigma_c", 1), ("eta", 1), ("zeta", 1),
                  ("l0", 1), ("residual", 1), ("A0", 9), ("n_interface", 3), ("a0", 3), ("alpha", 1),
                  ("phi", 1), ("phi_shear", 1), ("J_last", 1), ("tau_last", 9)):
    _PLANES[_name] = (_o, _k)
    _o += _k
N_PLANES = _o
_PAD = 64


def _stride_for(n: int) -> int:
    return max(_PAD, (n + _PAD - 1) // _PAD * _PAD)


# --------------------------------------------------------------------------- descriptors
class ParticleGrip:
    """Prescribed-velocity particles: ``v = velocity * min(t / ramp, 1)``
    (ramp <= 0: no ramp) overwrites v before P2G, inside the P2G kernel.
    Device form of a particle_bc closure that pins ``s.v[mask]``
    (test_block.py:109-113, peel_test.py:233-236).  The solver turns the mask
    into a per-particle tag once per descriptor: make a new descriptor rather
    than editing the mask of one already in ``particle_bc``."""

    def __init__(self, mask, velocity: Sequence[float], ramp: float = 0.0):
        self.mask = mask
        self.velocity = tuple(float(c) for c in velocity)
        if len(self.velocity) != 3:
            raise ValueError("velocity must have 3 components")
        self.ramp = float(ramp)

    def velocity_at(self, t: float):
        f = min(t / self.ramp, 1.0) if self.ramp > 0.0 else 1.0
        return tuple(c * f for c in self.velocity)


def grip_bc(mask, velocity, ramp: float = 0.0) -> ParticleGrip:
    return ParticleGrip(mask, velocity, ramp)


class Collider:
    """A grid collider descriptor (anisompm.py:811-867).  ``origin_fn(t)``
    gives the half-space origin or sphere centre; it is evaluated on the host
    at t and t + 1e-4 each substep (the velocity is their forward difference,
    as in the reference)."""

    def __init__(self, kind: str, origin_fn: Callable, normal=None, radius: float = 0.0, mode: str = "slip",
                 friction: float = 0.0):
        if mode not in ("slip", "sticky"):
            raise ValueError("mode must be 'slip' or 'sticky'")
        self.kind = kind
        self.origin_fn = origin_fn
        self.radius = float(radius)
        self.mode = mode
        self.friction = float(friction)
        if normal is not None:
            nrm = torch.tensor(normal, dtype=torch.float64)
            self.normal = (nrm / nrm.norm()).tolist()
        else:
            self.normal = [0.0, 0.0, 0.0]


def sphere_collider(center_fn, radius, mode="sticky", friction=0.0) -> Collider:
    """Same signature as the reference factory (anisompm.py:828)."""
    return Collider("sphere", center_fn, radius=radius, mode=mode, friction=friction)


def halfspace_collider(origin_fn, normal, mode="slip", friction=0.0) -> Collider:
    """Same signature as the reference factory (anisompm.py:847)."""
    return Collider("halfspace", origin_fn, normal=normal, mode=mode, friction=friction)


# --------------------------------------------------------------------------- sym_eig
def sym_eig(A: torch.Tensor, sweeps: int = 5):
    """Batched 3x3 symmetric eigendecomposition by cyclic Jacobi on the GPU
    (anisompm.py:48-95): ascending eigenvalues (N,3) and eigenvector columns
    (N,3,3).  CUDA tensors only (computed in float32); runs as
    ``torch.ops.peelmpm.sym_eig``."""
    if not A.is_cuda:
        raise ValueError("sym_eig runs on CUDA tensors only")
    if A.dim() != 3 or A.shape[1:] != (3, 3):
        raise ValueError("A must be (N,3,3)")
    from . import ops  # noqa: F401  (registers torch.ops.peelmpm)
    return torch.ops.peelmpm.sym_eig(A, int(sweeps))


def bin_particles(x: torch.Tensor, n_grid: int, inv_dx: float):
    """Cell key (``_node_index`` of the quadratic base cell, anisompm.py:544-548,
    586-590) of every particle, sorted, and the stable sorting permutation,
    on the GPU.  ``x`` is an (N,3) CUDA float32 tensor (any strides whose
    component planes are equally spaced, e.g. ``AnisoMPM.x``); runs as
    ``torch.ops.peelmpm.bin_sort``."""
    if not x.is_cuda or x.dtype != torch.float32 or x.dim() != 2 or x.shape[1] != 3:
        raise ValueError("x must be an (N,3) CUDA float32 tensor")
    from . import ops  # noqa: F401
    return torch.ops.peelmpm.bin_sort(x, int(n_grid), float(inv_dx))


# --------------------------------------------------------------------------- solver
class AnisoMPM:
    def __init__(
        self,
        n_grid: int = 96,
        grid_lim: float = 1.0,
        dt: float = 1e-4,
        gravity=(0.0, -9.8, 0.0),
        grid_damp: float = 1.0,
        f_clamp=None,
        damage_every: int = 1,
        device: str = "cuda:0",
        dtype=torch.float32,
    ):
        if dtype != torch.float32:
            raise NotImplementedError("the sm_100a substep computes in float32 only")
        self.device = torch.device(device)
        if self.device.type != "cuda":
            raise ValueError("AnisoMPM runs on a CUDA (sm_100) device; there is no CPU path")
        if self.device.index is None:
            self.device = torch.device("cuda", torch.cuda.current_device())
        self._lib = _lib.load()
        self.dtype = dtype
        self.n_grid = int(n_grid)
        self.grid_lim = float(grid_lim)
        self.dx = grid_lim / n_grid
        self.inv_dx = 1.0 / self.dx
        self.dt = float(dt)
        self._gravity_host = tuple(float(g) for g in gravity)
        self._gravity = torch.tensor(self._gravity_host, device=self.device, dtype=dtype)
        self.grid_damp = float(grid_damp)
        self.f_clamp = f_clamp
        self.damage_every = max(1, int(damage_every))
        self._step = 0
        off = torch.arange(3, device=self.device)
        gx, gy, gz = torch.meshgrid(off, off, off, indexing="ij")
        self.offsets = torch.stack([gx.reshape(-1), gy.reshape(-1), gz.reshape(-1)], 1)
        off4 = torch.arange(4, device=self.device)
        g4x, g4y, g4z = torch.meshgrid(off4, off4, off4, indexing="ij")
        self.offsets4 = torch.stack([g4x.reshape(-1), g4y.reshape(-1), g4z.reshape(-1)], 1)
        self.colliders = []
        self.particle_bc = []
        self.n = 0
        self.record_stress = False
        self.use_graphs = True
        self.p2g_ctas_per_sm = 0  # launch knobs (0 = library defaults; autotune.tune sets them); results
        self.grid_ctas_per_sm = 0  # do not depend on them
        self.stress_ctas_per_sm = 0
        self.g2p_ctas_per_sm = 0
        self._S = None            # float32 planes (N_PLANES, stride)
        self._allow = None        # bool (N)
        self._imask = None        # bool (N)
        self._tag = None          # int8 (N)
        self._iface_used = False
        self._ws = None
        self._ws_bytes = 0
        self._P = None
        self._params = None
        self._params_key = None
        self._tag_key = None
        self._graphs = {}
        self._batch = None

    # ------------------------------------------------------------------ views
    def _view(self, name):
        o, k = _PLANES[name]
        n = self.n
        if k == 1:
            return self._S[o, :n]
        if k == 3:
            return self._S[o:o + 3, :n].t()
        return self._S[o:o + 9, :n].t().view(n, 3, 3)

    def _set(self, name, value):
        self._view(name).copy_(torch.as_tensor(value, device=self.device, dtype=self.dtype))

    @property
    def gravity(self):
        return self._gravity

    @gravity.setter
    def gravity(self, g):
        g = torch.as_tensor(g, dtype=torch.float64).flatten().tolist()
        self._gravity_host = tuple(float(c) for c in g)
        self._gravity = torch.tensor(self._gravity_host, device=self.device, dtype=self.dtype)

    @property
    def allow(self):
        return self._allow

    @allow.setter
    def allow(self, v):
        self._allow.copy_(torch.as_tensor(v, device=self.device).bool())

    @property
    def interface_mask(self):
        self._iface_used = True
        self._P = None
        return self._imask

    @interface_mask.setter
    def interface_mask(self, v):
        self._iface_used = True
        self._P = None
        self._imask.copy_(torch.as_tensor(v, device=self.device).bool())

    @property
    def n_interface(self):
        self._iface_used = True
        self._P = None
        return self._view("n_interface")

    @n_interface.setter
    def n_interface(self, v):
        self._iface_used = True
        self._P = None
        self._set("n_interface", v)

    @property
    def tau_last(self):
        if not self.record_stress:
            raise AttributeError("tau_last is recorded only when record_stress = True")
        return self._view("tau_last")

    @property
    def J_last(self):
        if not self.record_stress:
            raise AttributeError("J_last is recorded only when record_stress = True")
        return self._view("J_last")

    # ------------------------------------------------------------------ setup
    def add_object(self, x, vol, rho: float = 500.0, E: float = 1.0e4, nu: float = 0.4, fibers=None,
                   alpha: float = -1.0, percentage: float = 0.15, l0_scale: float = 0.5, eta: float = 0.01,
                   zeta: float = 1.0, residual: float = 0.001, allow_damage: bool = True):
        """Append particles (anisompm.py:350-427, _append 429-463)."""
        if getattr(self, "_batch", None) is not None:
            raise RuntimeError("this scene is packed into a BatchedAnisoMPM; call its unpack() before add_object")
        dev, dt = self.device, self.dtype
        x = torch.as_tensor(x).to(dev, dt)
        vol = torch.as_tensor(vol).to(dev, dt)
        N = x.shape[0]
        mu = E / (2.0 * (1.0 + nu))
        lam = E * nu / ((1.0 + nu) * (1.0 - 2.0 * nu))
        new = {
            "x": x, "v": torch.zeros_like(x), "F": torch.eye(3, device=dev, dtype=dt).expand(N, 3, 3),
            "C": torch.zeros(N, 3, 3, device=dev, dtype=dt), "vol0": vol.clone(), "mass": vol * rho,
            "mu": torch.full((N,), mu, device=dev, dtype=dt), "lam": torch.full((N,), lam, device=dev, dtype=dt),
            "d": torch.zeros(N, device=dev, dtype=dt), "lap": torch.zeros(N, device=dev, dtype=dt),
            "D_hist": torch.zeros(N, device=dev, dtype=dt), "n_interface": torch.zeros(N, 3, device=dev, dtype=dt),
        }
        if fibers is None or alpha == 0.0:
            a0 = torch.zeros(N, 3, device=dev, dtype=dt)
            al = torch.zeros(N, device=dev, dtype=dt)
        else:
            f = torch.as_tensor(fibers).to(dev, dt)
            a0 = f / (f.norm(dim=1, keepdim=True) + 1e-12)
            al = torch.full((N,), float(alpha), device=dev, dtype=dt)
        new["a0"], new["alpha"] = a0, al
        aa0 = a0.unsqueeze(2) * a0.unsqueeze(1)
        new["A0"] = torch.eye(3, device=dev, dtype=dt).expand(N, 3, 3) + al.view(-1, 1, 1) * aa0
        sigma_c = max(percentage, 1e-8) * E
        new["sigma_c"] = torch.full((N,), float(sigma_c), device=dev, dtype=dt)
        new["eta"] = torch.full((N,), float(eta), device=dev, dtype=dt)
        new["zeta"] = torch.full((N,), float(zeta), device=dev, dtype=dt)
        new["l0"] = torch.full((N,), float(l0_scale * self.dx), device=dev, dtype=dt)
        new["residual"] = torch.full((N,), float(residual), device=dev, dtype=dt)
        allow = torch.full((N,), bool(allow_damage), device=dev, dtype=torch.bool)
        imask = torch.zeros(N, device=dev, dtype=torch.bool)

        n_old = self.n
        n_tot = n_old + N
        S = torch.zeros((N_PLANES, _stride_for(n_tot)), device=dev, dtype=dt)
        A = torch.empty(n_tot, device=dev, dtype=torch.bool)
        IM = torch.empty(n_tot, device=dev, dtype=torch.bool)
        if n_old:
            S[:, :n_old] = self._S[:, :n_old]
            A[:n_old] = self._allow
            IM[:n_old] = self._imask
        A[n_old:] = allow
        IM[n_old:] = imask
        self._S, self._allow, self._imask = S, A, IM
        self.n = n_tot
        for name, val in new.items():
            o, k = _PLANES[name]
            if k == 1:
                S[o, n_old:n_tot] = val
            else:
                S[o:o + k, n_old:n_tot] = val.reshape(N, k).t()
        self._tag = None
        self._tag_key = None
        self._P = None
        self._ws = None
        self._graphs.clear()
        return self

    def set_radial_fibers(self, center, zero_dim: int = 1, alpha: float = -1.0):
        """anisompm.py:465-484"""
        c = torch.as_tensor(center, device=self.device, dtype=self.dtype)
        r = self.x - c
        r[:, zero_dim] = 0.0
        nrm = r.norm(dim=1, keepdim=True)
        r = torch.where(nrm > 1e-9, r / (nrm + 1e-12), torch.zeros_like(r))
        self.a0 = r
        self.alpha = torch.full((self.n,), float(alpha), device=self.device, dtype=self.dtype)
        aa = self.a0.unsqueeze(2) * self.a0.unsqueeze(1)
        eyeN = torch.eye(3, device=self.device, dtype=self.dtype).expand(self.n, 3, 3)
        self.A0 = eyeN + self.alpha.view(-1, 1, 1) * aa
        return self

    def set_structural_tensor(self, mask, A0):
        """anisompm.py:486-509"""
        mask = torch.as_tensor(mask, device=self.device).bool()
        A = torch.as_tensor(A0, device=self.device, dtype=self.dtype)
        if A.dim() == 2:
            A = A.unsqueeze(0).expand(int(mask.sum()), 3, 3)
        if A.shape[0] == int(mask.sum()):
            full = self.A0.clone()
            full[mask] = A
            A = full
        self.A0 = torch.where(mask.view(-1, 1, 1), A, self.A0)
        return self

    def set_interface_normals(self, mask, normals):
        """anisompm.py:511-529"""
        mask = torch.as_tensor(mask, device=self.device).bool()
        nrm = torch.as_tensor(normals, device=self.device, dtype=self.dtype)
        if nrm.shape[0] == int(mask.sum()):
            full = torch.zeros(self.n, 3, device=self.device, dtype=self.dtype)
            full[mask] = nrm
            nrm = full
        nrm = nrm / (nrm.norm(dim=1, keepdim=True) + 1e-12)
        self.n_interface = torch.where(mask.view(-1, 1), nrm, self.n_interface)
        self.interface_mask = self.interface_mask | mask
        return self

    def set_normal_isolation(self, mask, normals):
        """anisompm.py:531-541"""
        self.set_interface_normals(mask, normals)
        mask = torch.as_tensor(mask, device=self.device).bool()
        nn = self.n_interface.unsqueeze(2) * self.n_interface.unsqueeze(1)
        return self.set_structural_tensor(mask, nn[mask])

    # ------------------------------------------------------------------ plumbing
    def _ensure_ws(self):
        need = _lib.workspace_size(self.n, self.n_grid)
        if self._ws is None or self._ws_bytes < need:
            self._ws = torch.empty(need, dtype=torch.uint8, device=self.device)
            self._ws_bytes = need
            with torch.cuda.device(self.device):
                _lib.check(self._lib.pm_workspace_init(self._ws.data_ptr(), need, self.n, self.n_grid,
                                                       torch.cuda.current_stream().cuda_stream),
                           "pm_workspace_init")
            self._graphs.clear()

    def _descriptors(self):
        grips, calls = [], []
        for bc in self.particle_bc:
            if isinstance(bc, ParticleGrip):
                grips.append(bc)
            elif callable(bc):
                calls.append(bc)
            else:
                raise TypeError(f"particle_bc entries must be grip_bc descriptors or callables, got {type(bc)}")
        if len(grips) > _lib.PM_MAX_GRIPS:
            raise ValueError(f"at most {_lib.PM_MAX_GRIPS} grip descriptors")
        for c in self.colliders:
            if not isinstance(c, Collider):
                raise NotImplementedError("colliders must come from peel_mpm_b200.halfspace_collider / "
                                          "sphere_collider (device descriptors); arbitrary callables are not run")
        if len(self.colliders) > _lib.PM_MAX_COLLIDERS:
            raise ValueError(f"at most {_lib.PM_MAX_COLLIDERS} colliders")
        return grips, calls

    def _grip_tags(self, grips):
        key = tuple(id(g) for g in grips)
        if self._tag_key is not None and key == self._tag_key:
            return
        if not grips:
            self._tag = None
        else:
            tag = torch.full((self.n,), -1, dtype=torch.int8, device=self.device)
            for i, g in enumerate(grips):
                m = torch.as_tensor(g.mask, device=self.device)
                if m.dtype == torch.bool:
                    tag[m] = i
                else:
                    tag[m.long()] = i
            self._tag = tag
        self._tag_key = key
        self._P = None

    def _build_params(self, grips):
        key = (self.n_grid, self.grid_lim, self.dt, self._gravity_host, self.grid_damp,
               None if self.f_clamp is None else tuple(float(v) for v in self.f_clamp), self.damage_every,
               bool(self.record_stress), int(self.p2g_ctas_per_sm), int(self.grid_ctas_per_sm),
               int(self.stress_ctas_per_sm), int(self.g2p_ctas_per_sm),
               tuple((g.velocity, g.ramp) for g in grips),
               tuple((c.kind, c.mode, c.friction, c.radius, tuple(c.normal)) for c in self.colliders))
        if key == self._params_key:
            return self._params
        p = _lib.pm_params()
        p.n_grid = self.n_grid
        p.damage_every = self.damage_every
        p.grid_lim, p.dx, p.inv_dx, p.dt = self.grid_lim, self.dx, self.inv_dx, self.dt
        for a in range(3):
            p.gravity[a] = self._gravity_host[a]
        p.grid_damp = self.grid_damp
        p.use_f_clamp = int(self.f_clamp is not None)
        if self.f_clamp is not None:
            p.f_clamp_lo, p.f_clamp_hi = float(self.f_clamp[0]), float(self.f_clamp[1])
        p.record_stress = int(bool(self.record_stress))
        p.p2g_ctas_per_sm = int(self.p2g_ctas_per_sm)
        p.grid_ctas_per_sm = int(self.grid_ctas_per_sm)
        p.stress_ctas_per_sm = int(self.stress_ctas_per_sm)
        p.g2p_ctas_per_sm = int(self.g2p_ctas_per_sm)
        p.n_grips = len(grips)
        for i, g in enumerate(grips):
            for a in range(3):
                p.grips[i].vel[a] = g.velocity[a]
            p.grips[i].ramp = g.ramp
        p.n_colliders = len(self.colliders)
        for i, c in enumerate(self.colliders):
            p.colliders[i].kind = 0 if c.kind == "halfspace" else 1
            p.colliders[i].mode = 1 if c.mode == "sticky" else 0
            p.colliders[i].friction = c.friction
            p.colliders[i].radius = c.radius
            for a in range(3):
                p.colliders[i].normal[a] = c.normal[a]
        self._params, self._params_key = p, key
        self._P = None
        return p

    def _particles(self):
        if self._P is not None:
            return self._P
        P = _lib.pm_particles()
        P.n = self.n
        P.plane_stride = self._S.stride(0)
        base = self._S.data_ptr()
        st = self._S.stride(0) * 4
        for name in ("x", "v", "F", "C", "d", "lap", "D_hist", "vol0", "mass", "mu", "lam", "sigma_c", "eta",
                     "zeta", "l0", "residual", "A0", "phi"):
            setattr(P, name, base + _PLANES[name][0] * st)
        P.allow = self._allow.data_ptr()
        if self._iface_used:
            P.n_interface = base + _PLANES["n_interface"][0] * st
            P.interface_mask = self._imask.data_ptr()
            P.phi_shear = base + _PLANES["phi_shear"][0] * st
        P.grip_tag = None if self._tag is None else self._tag.data_ptr()
        P.tau_last = base + _PLANES["tau_last"][0] * st
        P.J_last = base + _PLANES["J_last"][0] * st
        self._P = P
        return P

    def _clock(self, time: float, step: int):
        clk = _lib.pm_clock()
        clk.time = float(time)
        clk.step = int(step)
        for i, c in enumerate(self.colliders):
            o = [float(v) for v in c.origin_fn(time)]
            o2 = [float(v) for v in c.origin_fn(time + 1e-4)]
            for a in range(3):
                clk.col_origin[i][a] = o[a]
                clk.col_origin_next[i][a] = o2[a]
        return clk

    # ------------------------------------------------------------------- step
    def substep(self, time: float = 0.0):
        """One MLS-MPM + AnisoMPM damage substep (anisompm.py:593-803)."""
        if self.n == 0:
            self._step += 1
            return
        grips, calls = self._descriptors()
        for bc in calls:
            bc(self, time)
        self._grip_tags(grips)
        prm = self._build_params(grips)
        self._ensure_ws()
        from . import ops
        clk = self._clock(time, self._step)
        torch.ops.peelmpm.substep(self._S, self._allow, self._imask if self._iface_used else None, self._tag,
                                  self._ws, ops.struct_bytes(prm), ops.struct_bytes(clk), self.n)
        self._step += 1

    def run_frame(self, n_sub: int, time0: float = 0.0):
        """n_sub substeps at time0 + s*dt (anisompm.py:805-807).

        With ``use_graphs`` (default) and only device descriptors in
        ``particle_bc``, the frame's substeps are captured once into a CUDA
        graph per (n_sub, parameters, storage) and replayed; each frame's
        times, step numbers and collider origins go to the device in one copy
        from pinned memory, so a frame costs one graph launch on the host."""
        n_sub = int(n_sub)
        if n_sub <= 0:
            return
        grips, calls = self._descriptors()
        if calls or not self.use_graphs or self.n == 0:
            for s in range(n_sub):
                self.substep(time0 + s * self.dt)
            return
        self._grip_tags(grips)
        prm = self._build_params(grips)
        self._ensure_ws()
        P = self._particles()
        host = torch.empty(n_sub * C.sizeof(_lib.pm_clock), dtype=torch.uint8, pin_memory=True)
        clocks = (_lib.pm_clock * n_sub).from_address(host.data_ptr())
        for s in range(n_sub):
            clocks[s] = self._clock(time0 + s * self.dt, self._step + s)
        key = (n_sub, self._params_key, id(P), self._ws.data_ptr(), self._S.data_ptr())
        entry = self._graphs.get(key)
        if entry is None:
            table = torch.empty(host.numel(), dtype=torch.uint8, device=self.device)
            _lib.check(self._lib.pm_prepare(), "pm_prepare")
            torch.cuda.synchronize(self.device)
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g):
                st = torch.cuda.current_stream().cuda_stream
                for s in range(n_sub):   # row s of the device clock table drives substep s
                    _lib.check(self._lib.pm_substep_dev_clock(C.byref(prm), C.byref(P), self._ws.data_ptr(),
                                                              self._ws_bytes, table.data_ptr(), s, st),
                               "pm_substep_dev_clock")
            entry = (g, table, prm, P)
            self._graphs[key] = entry
        g, table = entry[0], entry[1]
        table.copy_(host, non_blocking=True)
        g.replay()
        self._step += n_sub

    # ------------------------------------------------------------------ status
    def status(self) -> dict:
        """Device status counters (synchronises the current stream)."""
        self._ensure_ws()
        info = _lib.pm_status_info()
        with torch.cuda.device(self.device):
            _lib.check(self._lib.pm_read_status(self._ws.data_ptr(), self._ws_bytes, self.n, self.n_grid,
                                                C.byref(info), torch.cuda.current_stream().cuda_stream),
                       "pm_read_status")
        return {"nonfinite": int(info.nonfinite), "dense_subblocks": int(info.dense_subblocks),
                "n_active_blocks": int(info.n_active_blocks), "any_allow": int(info.any_allow)}

    def check(self):
        """Raise if any particle's position or deformation gradient went
        non-finite since the workspace was created, or if a 4^3-cell
        sub-block held more particles than the exact grid sums allow for
        (16,383: about 256 per cell)."""
        st = self.status()
        if st["nonfinite"]:
            raise FloatingPointError(f"{st['nonfinite']} particle updates produced non-finite x or F")
        if st["dense_subblocks"]:
            raise OverflowError(f"{st['dense_subblocks']} P2G sub-blocks exceeded the fixed-point headroom")
        return st


def _plane_property(name):
    def get(self):
        return self._view(name)

    def set_(self, value):
        self._set(name, value)

    return property(get, set_)


for _name in ("x", "v", "F", "C", "d", "lap", "D_hist", "vol0", "mass", "mu", "lam", "sigma_c", "eta", "zeta",
              "l0", "residual", "A0", "a0", "alpha", "phi", "phi_shear"):
    setattr(AnisoMPM, _name, _plane_property(_name))

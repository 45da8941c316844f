"""Differentiable rollouts of the plain substep through hand-written adjoint kernels.

``rollout(sim, n_steps, mu=..., lam=..., sigma_c=..., A0=..., v0=...)``
writes the given per-particle parameters (and initial velocity) into ``sim``,
advances it ``n_steps`` substeps and returns the final positions (N,3) (with
``outputs="xv"``, the final positions and velocities) as tensors that carry
the autograd graph back to those inputs.  The backward
pass never stores the whole trajectory: the forward keeps the mutable state
(x, v, F, C, d, lap, D_hist) every ``checkpoint_every`` substeps; the backward
re-runs each segment from its checkpoint while recording every substep's grid
state into a tape (``pm_substep_record``) and then walks the segment in
reverse with ``pm_substep_adjoint`` (G2P adjoint as a scatter to the grid,
grid-update adjoint, P2G adjoint as a gather fused with the constitutive,
polar, eigen-split and damage adjoints).

``material(E, nu, fibers, alpha)`` forms mu, lam and A0 with the formulas of
add_object (anisompm.py:371-372, 395-404) in differentiable torch ops, so
gradients with respect to Young's modulus and fiber directions follow by
composition.  The reference obtains the same gradients by PyTorch autograd
through its substep (anisompm.py:593-803).

Everything the substep does is differentiated: grips (gripped particles
have zero velocity adjoint, their velocity is prescribed), gravity, grid
damping, damage_every, the strain limit f_clamp (through the singular values
it limits), grid colliders (each collider's resolve rule, walked back from the
recorded pre-collider grid velocity) and the directional stress at interface
particles.
"""
from __future__ import annotations

import ctypes as C
from typing import Optional

import torch

from . import _lib
from .anisompm import _PLANES, AnisoMPM

_MUTABLE = 27          # x v F C d lap D_hist: the first 27 planes of the store


def material(E, nu: float, fibers=None, alpha: float = -1.0):
    """(mu, lam, A0) from per-particle E (N,), Poisson ratio and fibers (N,3)."""
    mu = E / (2.0 * (1.0 + nu))
    lam = E * nu / ((1.0 + nu) * (1.0 - 2.0 * nu))
    n = E.shape[0]
    eye = torch.eye(3, device=E.device, dtype=E.dtype).expand(n, 3, 3)
    if fibers is None or alpha == 0.0:
        return mu, lam, eye.clone()
    a = fibers / (fibers.norm(dim=1, keepdim=True) + 1e-12)
    A0 = eye + alpha * a.unsqueeze(2) * a.unsqueeze(1)
    return mu, lam, A0


def _state_adj(buf: torch.Tensor) -> "_lib.pm_state_adj":
    a = _lib.pm_state_adj()
    a.plane_stride = buf.stride(0)
    base, st = buf.data_ptr(), buf.stride(0) * 4
    for name in ("x", "v", "F", "C", "d", "lap", "D_hist"):
        setattr(a, name, base + _PLANES[name][0] * st)
    return a


def _particles_at(sim: AnisoMPM, P, state: torch.Tensor):
    """Copy of the descriptor P with the mutable planes in ``state``."""
    Q = _lib.pm_particles.from_buffer_copy(P)
    base, st = state.data_ptr(), state.stride(0) * 4
    for name in ("x", "v", "F", "C", "d", "lap", "D_hist"):
        setattr(Q, name, base + _PLANES[name][0] * st)
    Q.phi = None
    Q.phi_shear = None
    Q.tau_last = None
    Q.J_last = None
    return Q


def _tape_flags(sim: AnisoMPM) -> int:
    return _lib.PM_TAPE_COLLIDERS if sim.colliders else 0


class _Recorder:
    """Tape and per-substep states of one checkpoint segment."""

    def __init__(self, sim: AnisoMPM, slots: int):
        lib = _lib.load()
        self.sim, self.slots, self.lib = sim, slots, lib
        dev = sim.device
        n, stride = sim.n, sim._S.stride(0)
        grips, _ = sim._descriptors()
        sim._grip_tags(grips)
        self.prm = sim._build_params(grips)
        sim._ensure_ws()
        P = sim._particles()
        flags = _tape_flags(sim)
        self.tape_bytes = _lib.tape_size(n, sim.n_grid, slots, flags)
        self.tape = torch.empty(self.tape_bytes, dtype=torch.uint8, device=dev)
        self.stream = torch.cuda.current_stream(dev).cuda_stream
        _lib.check(lib.pm_tape_init(self.tape.data_ptr(), self.tape_bytes, n, sim.n_grid, slots, flags,
                                    self.stream), "pm_tape_init")
        self.states = torch.empty((slots + 1, _MUTABLE, stride), device=dev, dtype=torch.float32)
        self.descr = [_particles_at(sim, P, self.states[j]) for j in range(slots + 1)]

    def record(self, state0, k: int, time0: float, step0: int):
        """Run k substeps from state0 (recording slots 0..k-1); states[j] is
        the state before substep j, states[k] the final one.  Each recorded
        substep reads states[j] and writes states[j + 1] (out of place)."""
        sim, lib = self.sim, self.lib
        self.states[0].copy_(state0)
        for j in range(k):
            clk = sim._clock(time0 + j * sim.dt, step0 + j)
            _lib.check(lib.pm_substep_record(C.byref(self.prm), C.byref(self.descr[j]), C.byref(self.descr[j + 1]),
                                             sim._ws.data_ptr(), sim._ws_bytes, C.byref(clk), self.tape.data_ptr(),
                                             self.tape_bytes, self.slots, j, self.stream), "pm_substep_record")


class _Rollout(torch.autograd.Function):
    @staticmethod
    def forward(ctx, mu, lam, sigma_c, A0, v0, sim, n_steps, time0, every):
        with torch.no_grad():
            sim.mu.copy_(mu)
            sim.lam.copy_(lam)
            sim.sigma_c.copy_(sigma_c)
            sim.A0.copy_(A0)
            sim.v.copy_(v0)
        step0 = sim._step
        checkpoints = []
        want_grad = any(ctx.needs_input_grad[:5])
        rec = _Recorder(sim, min(every, n_steps)) if want_grad else None
        t = 0
        while t < n_steps:
            k = min(every, n_steps - t)
            checkpoints.append(sim._S[:_MUTABLE].clone())
            if rec is not None and t + k >= n_steps:
                # the last segment is recorded now, so the backward starts without recomputing it
                rec.record(sim._S[:_MUTABLE], k, time0 + t * sim.dt, step0 + t)
                sim._S[:_MUTABLE].copy_(rec.states[k])
                sim._step += k
            else:
                sim.run_frame(k, time0 + t * sim.dt)
            t += k
        ctx.sim = sim
        ctx.meta = (n_steps, time0, every, step0)
        ctx.checkpoints = checkpoints
        ctx.rec = rec
        return sim.x.clone(), sim.v.clone()

    @staticmethod
    def backward(ctx, gx, gv):
        sim, rec = ctx.sim, ctx.rec
        n_steps, time0, every, step0 = ctx.meta
        lib = rec.lib
        dev = sim.device
        n, stride = sim.n, sim._S.stride(0)
        a_in = torch.zeros((_MUTABLE, stride), device=dev, dtype=torch.float32)
        a_out = torch.zeros_like(a_in)
        o = _PLANES["v"][0]
        a_in[0:3, :n] = gx.t().to(torch.float32)
        a_in[o:o + 3, :n] = gv.t().to(torch.float32)
        pg = torch.zeros((12, stride), device=dev, dtype=torch.float32)   # mu lam sigma_c A0(9)
        grads = _lib.pm_param_adj()
        grads.plane_stride = stride
        pgb, pst = pg.data_ptr(), stride * 4
        grads.mu, grads.lam, grads.sigma_c, grads.A0 = pgb, pgb + pst, pgb + 2 * pst, pgb + 3 * pst
        seg_starts = list(range(0, n_steps, every))
        last = len(seg_starts) - 1
        for si in reversed(range(len(seg_starts))):
            t0 = seg_starts[si]
            k = min(every, n_steps - t0)
            if si != last:   # the forward recorded the last segment
                rec.record(ctx.checkpoints[si], k, time0 + t0 * sim.dt, step0 + t0)
            for j in reversed(range(k)):
                ai, ao = _state_adj(a_in), _state_adj(a_out)
                _lib.check(lib.pm_substep_adjoint(C.byref(rec.prm), C.byref(rec.descr[j]), C.byref(rec.descr[j + 1]),
                                                  C.byref(ai), C.byref(ao), C.byref(grads), rec.tape.data_ptr(),
                                                  rec.tape_bytes, rec.slots, j, rec.stream), "pm_substep_adjoint")
                a_in, a_out = a_out, a_in
        g_mu = pg[0, :n].clone()
        g_lam = pg[1, :n].clone()
        g_sc = pg[2, :n].clone()
        g_A0 = pg[3:12, :n].t().reshape(n, 3, 3).clone()
        g_v0 = a_in[o:o + 3, :n].t().clone()
        ctx.checkpoints = None
        ctx.rec = None
        return g_mu, g_lam, g_sc, g_A0, g_v0, None, None, None, None


def segment_bytes(sim: AnisoMPM, k: int) -> int:
    """Device bytes of a k-substep recording segment: the tape (grid and
    particle records of every substep) and the k + 1 particle states."""
    return _lib.tape_size(sim.n, sim.n_grid, k, _tape_flags(sim)) + (k + 1) * _MUTABLE * sim._S.stride(0) * 4


def auto_segment(sim: AnisoMPM, n_steps: int, memory_fraction: float = 0.5) -> int:
    """The longest segment (at most ``n_steps``) whose recording fits in
    ``memory_fraction`` of the device's free memory.  A segment as long as
    the rollout records every substep during the forward, so the backward
    recomputes nothing (1M particles on 128^3: ~0.23 GB per substep)."""
    free, _ = torch.cuda.mem_get_info(sim.device)
    budget = int(free * memory_fraction)
    lo, hi = 1, max(1, int(n_steps))
    if segment_bytes(sim, hi) <= budget:
        return hi
    while lo < hi:   # largest k with segment_bytes(k) <= budget (1 if none)
        mid = (lo + hi + 1) // 2
        if segment_bytes(sim, mid) <= budget:
            lo = mid
        else:
            hi = mid - 1
    return lo


def rollout(sim: AnisoMPM, n_steps: int, mu=None, lam=None, sigma_c=None, A0=None, v0=None,
            time0: float = 0.0, checkpoint_every=10, outputs: str = "x"):
    """Final positions after ``n_steps`` substeps, differentiable with respect
    to the given per-particle mu, lam, sigma_c, A0 and initial velocity v0
    (any left as None is taken from ``sim`` as a constant).  ``outputs``:
    "x" returns the final positions (N,3), "v" the final velocities, "xv"
    the pair (a loss may use both).

    ``checkpoint_every`` = k: the forward keeps the state every k substeps and
    records the last segment; the backward re-runs every other segment from
    its checkpoint.  ``"auto"`` takes the longest segment that fits in half
    the free device memory (``auto_segment``)."""
    if n_steps < 1:
        raise ValueError("n_steps must be >= 1")
    if checkpoint_every == "auto":
        checkpoint_every = auto_segment(sim, n_steps)
    if not isinstance(checkpoint_every, int) or checkpoint_every < 1:
        raise ValueError("checkpoint_every must be an int >= 1 or 'auto'")
    if outputs not in ("x", "v", "xv"):
        raise ValueError("outputs must be 'x', 'v' or 'xv'")
    mu = sim.mu.detach().clone() if mu is None else mu
    lam = sim.lam.detach().clone() if lam is None else lam
    sigma_c = sim.sigma_c.detach().clone() if sigma_c is None else sigma_c
    A0 = sim.A0.detach().clone() if A0 is None else A0
    v0 = sim.v.detach().clone() if v0 is None else v0
    xT, vT = _Rollout.apply(mu, lam, sigma_c, A0, v0, sim, int(n_steps), float(time0), int(checkpoint_every))
    return {"x": xT, "v": vT, "xv": (xT, vT)}[outputs]


STATE_FIELDS = ("x", "v", "F", "C", "d", "lap", "D_hist")


def substep_vjp(sim: AnisoMPM, time: float, bars: dict):
    """Advance ``sim`` by one substep and return the vector-Jacobian product
    of that substep: given adjoints ``bars[f]`` of the post-substep state
    fields (reference shapes; missing fields count as zero), the adjoints of
    the pre-substep state fields and of mu, lam, sigma_c and A0."""
    lib = _lib.load()
    n, stride, dev = sim.n, sim._S.stride(0), sim.device
    grips, calls = sim._descriptors()
    if calls:
        raise NotImplementedError("the adjoint needs grip_bc descriptors, not callables")
    sim._grip_tags(grips)
    prm = sim._build_params(grips)
    sim._ensure_ws()
    P = sim._particles()
    st = torch.cuda.current_stream(dev).cuda_stream
    flags = _tape_flags(sim)
    tape_bytes = _lib.tape_size(n, sim.n_grid, 1, flags)
    tape = torch.empty(tape_bytes, dtype=torch.uint8, device=dev)
    _lib.check(lib.pm_tape_init(tape.data_ptr(), tape_bytes, n, sim.n_grid, 1, flags, st), "pm_tape_init")
    states = torch.empty((2, _MUTABLE, stride), device=dev, dtype=torch.float32)
    states[0].copy_(sim._S[:_MUTABLE])
    pre, post = _particles_at(sim, P, states[0]), _particles_at(sim, P, states[1])
    clk = sim._clock(time, sim._step)
    _lib.check(lib.pm_substep_record(C.byref(prm), C.byref(pre), C.byref(post), sim._ws.data_ptr(), sim._ws_bytes,
                                     C.byref(clk), tape.data_ptr(), tape_bytes, 1, 0, st), "pm_substep_record")
    a_in = torch.zeros((_MUTABLE, stride), device=dev, dtype=torch.float32)
    a_out = torch.zeros_like(a_in)
    for f, val in bars.items():
        o, k = _PLANES[f]
        t = torch.as_tensor(val, device=dev, dtype=torch.float32)
        a_in[o:o + k, :n] = t.reshape(n, k).t()
    pg = torch.zeros((12, stride), device=dev, dtype=torch.float32)
    grads = _lib.pm_param_adj()
    grads.plane_stride = stride
    pgb, pst = pg.data_ptr(), stride * 4
    grads.mu, grads.lam, grads.sigma_c, grads.A0 = pgb, pgb + pst, pgb + 2 * pst, pgb + 3 * pst
    ai, ao = _state_adj(a_in), _state_adj(a_out)
    _lib.check(lib.pm_substep_adjoint(C.byref(prm), C.byref(pre), C.byref(post), C.byref(ai), C.byref(ao),
                                      C.byref(grads), tape.data_ptr(), tape_bytes, 1, 0, st), "pm_substep_adjoint")
    sim._S[:_MUTABLE].copy_(states[1])
    sim._step += 1
    out = {}
    for f in STATE_FIELDS:
        o, k = _PLANES[f]
        g = a_out[o:o + k, :n].t()
        out[f] = g[:, 0].clone() if k == 1 else (g.clone() if k == 3 else g.reshape(n, 3, 3).clone())
    par = {"mu": pg[0, :n].clone(), "lam": pg[1, :n].clone(), "sigma_c": pg[2, :n].clone(),
           "A0": pg[3:12, :n].t().reshape(n, 3, 3).clone()}
    return out, par

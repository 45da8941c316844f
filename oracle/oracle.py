"""CPU oracle driver -- TEST INFRASTRUCTURE ONLY.

ctypes wrapper around ``anisompm_oracle.c`` (built by ``oracle/Makefile`` into
``oracle/_build``).  It restates the reference solver's substep
(anisompm_py/src/anisompm.py:593-807) on the CPU so tests, the smoke check and
the CPU-baseline legs of bench.py can check and time the CUDA path.  The
product never imports this module.

``OracleSim`` mirrors the reference solver's state after ``add_object`` and
the per-particle overrides a scene applies (scenes.apply_scene), in the
reference's array-of-structs layout.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
BUILD = os.path.join(HERE, "_build")

_LIBS = {}


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def _lib(dtype):
    key = np.dtype(dtype).name
    if key not in _LIBS:
        path = os.path.join(BUILD, f"liboracle_{'f32' if key == 'float32' else 'f64'}.so")
        if not os.path.exists(path):
            build()
        lib = C.CDLL(path)
        lib.oracle_substep.restype = C.c_int
        lib.oracle_substep.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
        lib.oracle_sym_eig.restype = None
        lib.oracle_sym_eig.argtypes = [C.c_void_p, C.c_int64, C.c_int32, C.c_void_p, C.c_void_p]
        lib.oracle_bin_keys.restype = None
        lib.oracle_bin_keys.argtypes = [C.c_void_p, C.c_int64, C.c_int32, C.c_double, C.c_void_p]
        _LIBS[key] = lib
    return _LIBS[key]


class _Params(C.Structure):
    _fields_ = [
        ("n", C.c_int64), ("n_grid", C.c_int32), ("nthreads", C.c_int32),
        ("scatter_mode", C.c_int32), ("do_damage", C.c_int32),
        ("grid_lim", C.c_double), ("dx", C.c_double), ("inv_dx", C.c_double),
        ("dt", C.c_double), ("dt_dmg", C.c_double),
        ("gravity", C.c_double * 3), ("grid_damp", C.c_double),
        ("use_f_clamp", C.c_int32), ("f_clamp_lo", C.c_double), ("f_clamp_hi", C.c_double),
        ("any_interface", C.c_int32), ("n_colliders", C.c_int32), ("colliders", C.c_void_p),
        ("n_grips", C.c_int32), ("grip_tag", C.c_void_p), ("grip_vel", C.c_void_p),
    ]


_STATE_FIELDS = ["x", "v", "F", "C", "d", "lap", "D_hist", "vol0", "mass", "mu", "lam", "sigma_c",
                 "eta", "zeta", "l0", "residual", "A0", "allow", "n_interface", "interface_mask",
                 "phi", "phi_shear", "tau_last", "J_last"]


class _State(C.Structure):
    _fields_ = [(f, C.c_void_p) for f in _STATE_FIELDS]


class _Grids(C.Structure):
    _fields_ = [(f, C.c_void_p) for f in ["grid_mv", "grid_m", "grid_v", "grid_dc", "grid_dwc", "gd"]]


def _ptr(a):
    return None if a is None else a.ctypes.data


def sym_eig(A, dtype=np.float32, sweeps=5):
    """Oracle of ``sym_eig`` (anisompm.py:48-95) for a batch (N,3,3)."""
    A = np.ascontiguousarray(A, dtype=dtype)
    n = A.shape[0]
    ev = np.zeros((n, 3), dtype)
    V = np.zeros((n, 3, 3), dtype)
    _lib(dtype).oracle_sym_eig(_ptr(A), n, sweeps, _ptr(ev), _ptr(V))
    return ev, V


def bin_keys(x, n_grid, inv_dx, dtype=np.float32):
    """Cell key of every particle: ``_node_index`` of the quadratic base cell
    (anisompm.py:546-548, 586-590)."""
    x = np.ascontiguousarray(x, dtype=dtype)
    keys = np.zeros(x.shape[0], np.int64)
    _lib(dtype).oracle_bin_keys(_ptr(x), x.shape[0], int(n_grid), float(inv_dx), _ptr(keys))
    return keys


def bin_particles(x, n_grid, inv_dx, dtype=np.float32):
    """(keys, perm) with perm the stable argsort of keys."""
    keys = bin_keys(x, n_grid, inv_dx, dtype)
    return keys, np.argsort(keys, kind="stable")


def lame(E, nu):
    mu = E / (2.0 * (1.0 + nu))
    lam = E * nu / ((1.0 + nu) * (1.0 - 2.0 * nu))
    return mu, lam


class OracleSim:
    """Reference-shaped state driven by the C restatement.

    Construction follows add_object (anisompm.py:350-427) and _append (429-463)
    followed by a scene's per-particle overrides; ``substep`` follows
    anisompm.py:593-803 including the particle-BC hook (601-602) for grips and
    the collider hook (737-746)."""

    def __init__(self, scene, dtype=np.float32, nthreads=1, scatter_mode=0):
        self.dtype = np.dtype(dtype)
        self.nthreads = int(nthreads)
        self.scatter_mode = int(scatter_mode)
        sc = scene
        self.scene = sc
        dt_ = self.dtype
        n = sc.n
        self.n = n
        self.n_grid = int(sc.n_grid)
        self.grid_lim = float(sc.grid_lim)
        self.dx = self.grid_lim / self.n_grid
        self.inv_dx = 1.0 / self.dx
        self.dt = float(sc.dt)
        self.gravity = tuple(float(g) for g in sc.gravity)
        self.grid_damp = float(sc.grid_damp)
        self.f_clamp = sc.f_clamp
        self.damage_every = max(1, int(sc.damage_every))
        self._step = 0
        self.x = sc.x.astype(dt_)
        self.v = np.zeros((n, 3), dt_)
        self.F = np.tile(np.eye(3, dtype=dt_), (n, 1, 1))
        self.C = np.zeros((n, 3, 3), dt_)
        vol = sc.vol.astype(dt_)
        self.vol0 = vol.copy()
        self.mass = (vol * dt_.type(sc.rho)).astype(dt_)
        mu, lam = lame(sc.E.astype(np.float64), sc.nu)
        self.mu = mu.astype(dt_)
        self.lam = lam.astype(dt_)
        self.d = np.zeros(n, dt_) if sc.d0 is None else sc.d0.astype(dt_)
        self.lap = np.zeros(n, dt_)
        self.D_hist = np.zeros(n, dt_)
        self.n_interface = np.zeros((n, 3), dt_)
        self.interface_mask = np.zeros(n, np.uint8)
        if sc.fibers is None or sc.alpha == 0.0:
            a0 = np.zeros((n, 3), dt_)
            al = np.zeros(n, dt_)
        else:
            f = sc.fibers.astype(dt_)
            nrm = np.sqrt((f * f).sum(1, keepdims=True, dtype=dt_)).astype(dt_)
            a0 = (f / (nrm + dt_.type(1e-12))).astype(dt_)
            al = np.full(n, sc.alpha, dt_)
        aa = a0[:, :, None] * a0[:, None, :]
        self.A0 = (np.eye(3, dtype=dt_)[None] + al[:, None, None] * aa).astype(dt_)
        self.sigma_c = sc.sigma_c.astype(dt_)
        self.eta = np.full(n, sc.eta, dt_)
        self.zeta = np.full(n, sc.zeta, dt_)
        self.l0 = np.full(n, sc.l0_scale * self.dx, dt_)
        self.residual = np.full(n, sc.residual, dt_)
        self.allow = np.ones(n, np.uint8) if sc.allow is None else sc.allow.astype(np.uint8)
        if sc.interface is not None:
            m, nrm_in = sc.interface
            nr = nrm_in.astype(dt_)
            nr = (nr / (np.sqrt((nr * nr).sum(1, keepdims=True)) + dt_.type(1e-12))).astype(dt_)
            self.n_interface = np.where(m[:, None], nr, self.n_interface).astype(dt_)
            self.interface_mask = m.astype(np.uint8)
            self.A0 = np.where(m[:, None, None], self.n_interface[:, :, None] * self.n_interface[:, None, :],
                               self.A0).astype(dt_)
        self.phi = np.zeros(n, dt_)
        self.phi_shear = np.zeros(n, dt_)
        self.tau_last = np.zeros((n, 3, 3), dt_)
        self.J_last = np.zeros(n, dt_)
        self.grip_tag = np.full(n, -1, np.int32)
        for gi, g in enumerate(sc.grips):
            self.grip_tag[g.mask] = gi
        self.colliders = list(sc.colliders)

    # ------------------------------------------------------------------
    def _collider_table(self, time):
        rows = []
        for c in self.colliders:
            fn = c.origin_fn()
            o, o2 = fn(time), fn(time + 1e-4)
            nrm = np.asarray(c.normal, np.float64)
            nrm = nrm / np.linalg.norm(nrm)
            rows.append([0.0 if c.kind == "halfspace" else 1.0, 1.0 if c.mode == "sticky" else 0.0,
                         float(c.friction), float(c.radius), *nrm.tolist(), *o, *o2, 0.0, 0.0, 0.0])
        return np.asarray(rows, np.float64).reshape(-1, 16)

    def substep(self, time=0.0, grids=None):
        from peel_mpm_b200.scenes import grip_factor  # scene semantics only
        p = _Params()
        p.n = self.n
        p.n_grid = self.n_grid
        p.nthreads = self.nthreads
        p.scatter_mode = self.scatter_mode
        p.do_damage = int(bool(self.allow.any()) and (self._step % self.damage_every == 0))
        p.grid_lim, p.dx, p.inv_dx, p.dt = self.grid_lim, self.dx, self.inv_dx, self.dt
        p.dt_dmg = self.dt * self.damage_every
        p.gravity = (C.c_double * 3)(*self.gravity)
        p.grid_damp = self.grid_damp
        p.use_f_clamp = int(self.f_clamp is not None)
        if self.f_clamp is not None:
            p.f_clamp_lo, p.f_clamp_hi = float(self.f_clamp[0]), float(self.f_clamp[1])
        p.any_interface = int(bool(self.interface_mask.any()))
        col = self._collider_table(time)
        p.n_colliders = col.shape[0]
        p.colliders = _ptr(col)
        grips = self.scene.grips
        gv = np.asarray([[c * grip_factor(time, g.ramp) for c in g.velocity] for g in grips],
                        np.float64).reshape(-1, 3)
        p.n_grips = len(grips)
        p.grip_tag = _ptr(self.grip_tag)
        p.grip_vel = _ptr(gv)
        s = _State()
        for f in _STATE_FIELDS:
            setattr(s, f, _ptr(getattr(self, f)))
        g = None
        if grids is not None:
            g = _Grids()
            for f in _Grids._fields_:
                setattr(g, f[0], _ptr(grids.get(f[0])))
        rc = _lib(self.dtype).oracle_substep(C.byref(p), C.byref(s), C.byref(g) if g is not None else None)
        if rc != 0:
            raise RuntimeError("oracle_substep failed")
        self._step += 1

    def run(self, n_steps, time0=0.0, callback=None):
        for s in range(n_steps):
            self.substep(time0 + s * self.dt)
            if callback is not None:
                callback(self._step, self)

    def state(self):
        return {k: getattr(self, k).copy() for k in ("x", "v", "F", "C", "d", "lap", "D_hist")}

    def alloc_grids(self):
        G = self.n_grid ** 3
        z = lambda *s: np.zeros(s, self.dtype)
        return {"grid_mv": z(G, 3), "grid_m": z(G), "grid_v": z(G, 3), "grid_dc": z(G),
                "grid_dwc": z(G), "gd": z(G)}

"""Seeded synthetic AnisoMPM scenes.

Every scene is a jittered particle lattice inside a dense ``n_grid**3`` grid,
with per-particle material parameters, particle grips (velocity-prescribed,
damage-disabled particles) and optional grid colliders.  The generators use
only numpy's PCG64 stream, so the same seed yields the same bits on every
machine with this numpy version; the same scene feeds the reference solver,
the CPU oracle and the CUDA path.

A scene is applied to any object exposing the reference solver's setup API
(``add_object`` plus in-place writes to ``mu``/``lam``/``sigma_c``/``d``/
``allow``, ``particle_bc``, ``colliders``, ``set_normal_isolation``), which is
how the reference harnesses build theirs (peel_test.py:196-236,
test_block.py:96-113).

Particle order inside a lattice is cell-major (x slowest, z fastest), then the
sub-lattice in the same order, so the generation order is spatially coherent.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import Callable, Optional, Sequence

import numpy as np


@dataclass
class Grip:
    """Particles whose velocity is overwritten before P2G each substep.

    ``v = velocity * min(t / ramp, 1)`` (``ramp <= 0`` means no ramp), the
    gripper idiom of test_block.py:109-113 and peel_test.py:233-236."""
    mask: np.ndarray
    velocity: Sequence[float]
    ramp: float = 0.0


@dataclass
class ColliderSpec:
    """Grid collider moving linearly: origin(t) = origin + velocity * t.

    kind "halfspace" uses ``normal`` (material side), kind "sphere" uses
    ``radius``; ``mode`` is "slip" or "sticky" (anisompm.py:811-867)."""
    kind: str
    origin: Sequence[float]
    velocity: Sequence[float] = (0.0, 0.0, 0.0)
    normal: Sequence[float] = (0.0, 1.0, 0.0)
    radius: float = 0.0
    mode: str = "slip"
    friction: float = 0.0

    def origin_fn(self) -> Callable[[float], list]:
        o = [float(c) for c in self.origin]
        w = [float(c) for c in self.velocity]
        return lambda t: [o[0] + w[0] * t, o[1] + w[1] * t, o[2] + w[2] * t]


@dataclass
class Scene:
    name: str
    n_grid: int
    grid_lim: float
    dt: float
    n_steps: int
    x: np.ndarray                      # (N,3) float64 positions
    vol: np.ndarray                    # (N,) float64
    rho: float
    E: np.ndarray                      # (N,) Young's modulus
    nu: float
    fibers: Optional[np.ndarray]       # (N,3) or None
    alpha: float
    sigma_c: np.ndarray                # (N,) absolute critical stress
    l0_scale: float = 1.0
    eta: float = 1e-3
    zeta: float = 1.0
    residual: float = 1e-3
    d0: Optional[np.ndarray] = None
    allow: Optional[np.ndarray] = None  # (N,) bool
    gravity: Sequence[float] = (0.0, 0.0, 0.0)
    grid_damp: float = 1.0
    f_clamp: Optional[tuple] = None
    damage_every: int = 1
    grips: list = field(default_factory=list)
    colliders: list = field(default_factory=list)
    interface: Optional[tuple] = None  # (mask (N,) bool, normals (N,3))

    @property
    def n(self) -> int:
        return int(self.x.shape[0])

    @property
    def dx(self) -> float:
        return self.grid_lim / self.n_grid


# --------------------------------------------------------------------------- lattices
def jittered_lattice(cell_lo, n_cells, dx, ppc_dim, jitter, rng):
    """Particles on a ``ppc_dim**3`` sub-lattice of every cell in a box.

    Sub-lattice point k of a cell sits at ``(k + 0.5) / ppc_dim`` of the cell,
    plus a uniform jitter of ``+-jitter * dx`` per axis."""
    cx, cy, cz = (np.arange(n) + lo for n, lo in zip(n_cells, cell_lo))
    sub = (np.arange(ppc_dim) + 0.5) / ppc_dim
    C = np.stack(np.meshgrid(cx, cy, cz, indexing="ij"), -1).reshape(-1, 1, 3)
    S = np.stack(np.meshgrid(sub, sub, sub, indexing="ij"), -1).reshape(1, -1, 3)
    pts = ((C + S) * dx).reshape(-1, 3)
    pts = pts + rng.uniform(-jitter * dx, jitter * dx, size=pts.shape)
    return pts


def vmf_directions(mean, kappa, n, rng):
    """von Mises-Fisher samples on the sphere S^2 around ``mean``.

    For S^2 the cosine w = mean.a has the closed-form inverse CDF
    ``w = 1 + log(u + (1-u) exp(-2 kappa)) / kappa`` (Wood 1994, the p=3 case);
    the tangent direction is uniform."""
    mean = np.asarray(mean, np.float64)
    mean = mean / np.linalg.norm(mean)
    u = rng.uniform(0.0, 1.0, n)
    w = 1.0 + np.log(u + (1.0 - u) * np.exp(-2.0 * kappa)) / kappa
    w = np.clip(w, -1.0, 1.0)
    ang = rng.uniform(0.0, 2.0 * math.pi, n)
    helper = np.array([0.0, 0.0, 1.0]) if abs(mean[2]) < 0.9 else np.array([1.0, 0.0, 0.0])
    e1 = np.cross(mean, helper); e1 /= np.linalg.norm(e1)
    e2 = np.cross(mean, e1)
    s = np.sqrt(np.maximum(0.0, 1.0 - w * w))
    return (w[:, None] * mean[None] + s[:, None] * (np.cos(ang)[:, None] * e1[None]
                                                     + np.sin(ang)[:, None] * e2[None]))


def uniform_directions(n, rng):
    v = rng.normal(size=(n, 3))
    return v / np.linalg.norm(v, axis=1, keepdims=True)


# --------------------------------------------------------------------------- scenes
def plain_small(seed: int = 0) -> Scene:
    """16,384-particle bar on a 64^3 grid: left 2 cells clamped, right 2 cells
    pulled at +0.5 m/s, fibers along x with alpha=-1, sigma_c=200."""
    rng = np.random.default_rng(seed)
    ng = 64
    dx = 1.0 / ng
    lo, ext = (16, 28, 28), (32, 8, 8)
    x = jittered_lattice(lo, ext, dx, 2, 0.25, rng)
    n = x.shape[0]
    box_lo = lo[0] * dx
    box_hi = (lo[0] + ext[0]) * dx
    left = x[:, 0] < box_lo + 2 * dx
    right = x[:, 0] > box_hi - 2 * dx
    fib = np.zeros((n, 3)); fib[:, 0] = 1.0
    return Scene(
        name="plain_small", n_grid=ng, grid_lim=1.0, dt=1e-4, n_steps=200,
        x=x, vol=np.full(n, (dx / 2) ** 3), rho=1000.0, E=np.full(n, 1e4), nu=0.3,
        fibers=fib, alpha=-1.0, sigma_c=np.full(n, 200.0), l0_scale=1.0, eta=1e-3,
        allow=~(left | right),
        grips=[Grip(left, (0.0, 0.0, 0.0)), Grip(right, (0.5, 0.0, 0.0))])


def plain_1m(seed: int = 0, n_grid: int = 128, cells=(64, 32, 64), lo=(32, 16, 32)) -> Scene:
    """1,048,576-particle slab on a 128^3 grid with von Mises-Fisher fibers
    (kappa=20 about x), log-normal E, uniform sigma_c in [180, 220], initial
    damage U(0, 0.05); bottom layer clamped, one top edge pulled up at 1 m/s.
    ``cells``/``lo`` shrink it for tests (same statistics, fewer cells)."""
    rng = np.random.default_rng(seed)
    ng = n_grid
    dx = 1.0 / ng
    x = jittered_lattice(lo, cells, dx, 2, 0.25, rng)
    n = x.shape[0]
    fib = vmf_directions((1.0, 0.0, 0.0), 20.0, n, rng)
    d0 = rng.uniform(0.0, 0.05, n)
    E = 1e4 * np.exp(0.2 * rng.normal(size=n))
    sig = rng.uniform(180.0, 220.0, n)
    ylo, yhi = lo[1] * dx, (lo[1] + cells[1]) * dx
    xlo = lo[0] * dx
    bottom = x[:, 1] < ylo + dx
    top_edge = (x[:, 1] > yhi - dx) & (x[:, 0] < xlo + dx)
    return Scene(
        name="plain_1m" if cells == (64, 32, 64) else f"plain_slab_{n}",
        n_grid=ng, grid_lim=1.0, dt=5e-5, n_steps=500,
        x=x, vol=np.full(n, (dx / 2) ** 3), rho=1000.0, E=E, nu=0.3,
        fibers=fib, alpha=-1.0, sigma_c=sig, l0_scale=1.0, eta=1e-3, d0=d0,
        allow=~(bottom | top_edge),
        grips=[Grip(bottom, (0.0, 0.0, 0.0)), Grip(top_edge, (0.0, 1.0, 0.0))])


def peel_8m(seed: int = 0, scale: int = 1) -> Scene:
    """Two-layer peel slab on a 256^3 grid, 27 particles per cell: base
    128x16x128 cells (random fibers, sigma_c=400) whose top cell layer is a
    bonding band (sigma_c=40), skin 128x4x128 (fibers along x, sigma_c=400).
    Base bottom clamped; the skin's x=lo edge pulled along (1,1,0)/sqrt2 at
    1 m/s; gravity -9.8.  8,847,360 particles.  ``scale`` divides the in-plane
    extents for smaller test versions."""
    rng = np.random.default_rng(seed)
    ng = 256
    dx = 1.0 / ng
    w = 128 // scale
    lo = (64, 64, 64)
    base = jittered_lattice(lo, (w, 16, w), dx, 3, 1.0 / 6.0, rng)
    skin = jittered_lattice((lo[0], lo[1] + 16, lo[2]), (w, 4, w), dx, 3, 1.0 / 6.0, rng)
    x = np.concatenate([base, skin], 0)
    nb, ns = base.shape[0], skin.shape[0]
    n = nb + ns
    fib = np.concatenate([uniform_directions(nb, rng), np.tile([[1.0, 0.0, 0.0]], (ns, 1))], 0)
    sig = np.full(n, 400.0)
    y_bond_lo = (lo[1] + 15) * dx
    is_skin = np.arange(n) >= nb
    bond = (~is_skin) & (x[:, 1] >= y_bond_lo)
    sig[bond] = 40.0
    bottom = x[:, 1] < lo[1] * dx + dx
    edge = is_skin & (x[:, 0] < lo[0] * dx + dx)
    s2 = 1.0 / math.sqrt(2.0)
    return Scene(
        name="peel_8m" if scale == 1 else f"peel_{n}", n_grid=ng, grid_lim=1.0, dt=2e-5,
        n_steps=1000, x=x, vol=np.full(n, (dx / 3) ** 3), rho=1000.0, E=np.full(n, 1e4),
        nu=0.3, fibers=fib, alpha=-1.0, sigma_c=sig, l0_scale=1.0, eta=1e-3,
        allow=~(bottom | edge), gravity=(0.0, -9.8, 0.0),
        grips=[Grip(bottom, (0.0, 0.0, 0.0)), Grip(edge, (s2, s2, 0.0))])


def tiny_bar(seed: int = 0) -> Scene:
    """1,024-particle notched-free bar on a 32^3 grid pulled hard enough to
    damage within tens of substeps (a fast golden case)."""
    rng = np.random.default_rng(seed)
    ng = 32
    dx = 1.0 / ng
    lo, ext = (8, 14, 14), (8, 4, 4)
    x = jittered_lattice(lo, ext, dx, 2, 0.25, rng)
    n = x.shape[0]
    left = x[:, 0] < lo[0] * dx + dx
    right = x[:, 0] > (lo[0] + ext[0]) * dx - dx
    fib = np.zeros((n, 3)); fib[:, 1] = 1.0
    return Scene(
        name="tiny_bar", n_grid=ng, grid_lim=1.0, dt=1e-4, n_steps=200,
        x=x, vol=np.full(n, (dx / 2) ** 3), rho=1000.0, E=np.full(n, 1e4), nu=0.3,
        fibers=fib, alpha=-1.0, sigma_c=np.full(n, 60.0), l0_scale=1.0, eta=1e-3,
        d0=rng.uniform(0.0, 0.02, n), allow=~(left | right),
        grips=[Grip(left, (-0.5, 0.0, 0.0), ramp=2e-3), Grip(right, (1.0, 0.2, 0.0), ramp=2e-3)])


def knobs_drop(seed: int = 0) -> Scene:
    """A damaged block falling under gravity onto a slip half-space with
    friction while a sticky sphere sweeps through it; exercises grid_damp,
    f_clamp, damage_every=2 and both collider kinds (anisompm.py:622-636,
    647-649, 811-867)."""
    rng = np.random.default_rng(seed)
    ng = 32
    dx = 1.0 / ng
    lo, ext = (10, 9, 10), (10, 6, 8)
    x = jittered_lattice(lo, ext, dx, 2, 0.25, rng)
    n = x.shape[0]
    fib = uniform_directions(n, rng)
    return Scene(
        name="knobs_drop", n_grid=ng, grid_lim=1.0, dt=2e-4, n_steps=60,
        x=x, vol=np.full(n, (dx / 2) ** 3), rho=500.0, E=3e3 * np.exp(0.3 * rng.normal(size=n)),
        nu=0.35, fibers=fib, alpha=-0.8, sigma_c=rng.uniform(20.0, 40.0, n), l0_scale=0.7,
        eta=5e-3, zeta=1.3, residual=5e-3, d0=rng.uniform(0.0, 0.1, n),
        allow=np.ones(n, bool), gravity=(0.0, -9.8, 0.0), grid_damp=0.999,
        f_clamp=(0.6, 1.6), damage_every=2,
        colliders=[
            ColliderSpec("halfspace", (0.0, 9.4 * dx, 0.0), (0.0, 0.0, 0.0), normal=(0.1, 1.0, 0.0),
                         mode="slip", friction=0.4),
            ColliderSpec("sphere", (lo[0] * dx - 2 * dx, 12 * dx, 14 * dx), (3.0, 0.0, 0.0),
                         radius=2.5 * dx, mode="sticky"),
            ColliderSpec("sphere", (15 * dx, 17 * dx, 14 * dx), (0.0, -2.0, 0.0),
                         radius=2.0 * dx, mode="slip", friction=0.2),
        ])


def colliders_drop(seed: int = 0) -> Scene:
    """knobs_drop without f_clamp (grid damping, damage_every=2 and the three
    colliders: slip half-space with friction, sticky and slip spheres), with
    the half-space's origin at 9.43 dx instead of 9.4 dx.  knobs_drop's plane
    passes exactly through the grid nodes (14, 8, z), which float32 and float64
    then classify by rounding; here every node is at least 0.03 dx from it."""
    sc = knobs_drop(seed)
    dx = 1.0 / sc.n_grid
    hs = sc.colliders[0]
    sc.colliders[0] = ColliderSpec(hs.kind, (0.0, 9.43 * dx, 0.0), hs.velocity, normal=hs.normal, mode=hs.mode,
                                   friction=hs.friction)
    sc.name, sc.f_clamp = "colliders_drop", None
    return sc


def limit_drop(seed: int = 0) -> Scene:
    """colliders_drop with knobs_drop's strain limit f_clamp = (0.6, 1.6),
    which the first singular values reach after about 55 substeps."""
    sc = colliders_drop(seed)
    sc.name, sc.f_clamp = "limit_drop", (0.6, 1.6)
    return sc


def clamp_drop(seed: int = 0) -> Scene:
    """colliders_drop with a tight strain limit, f_clamp = (0.9, 1.02): about
    a hundred particles have a singular value beyond a bound at each substep
    after the first ten."""
    sc = colliders_drop(seed)
    sc.name, sc.f_clamp = "clamp_drop", (0.9, 1.02)
    return sc


def interface_peel(seed: int = 0) -> Scene:
    """Two-layer slab whose interface band carries set_normal_isolation
    normals (directional delamination stress, anisompm.py:190-227, 697-703);
    the top layer is pulled up at one end."""
    rng = np.random.default_rng(seed)
    ng = 32
    dx = 1.0 / ng
    lo, ext = (8, 10, 10), (12, 6, 8)
    x = jittered_lattice(lo, ext, dx, 2, 0.25, rng)
    n = x.shape[0]
    y = x[:, 1]
    y_if = (lo[1] + 3) * dx
    band = np.abs(y - y_if) < 0.6 * dx
    normals = np.tile([[0.0, 1.0, 0.0]], (n, 1)) + 0.05 * rng.normal(size=(n, 3))
    bottom = y < lo[1] * dx + dx
    pull = (y > (lo[1] + ext[1]) * dx - dx) & (x[:, 0] < lo[0] * dx + 2 * dx)
    return Scene(
        name="interface_peel", n_grid=ng, grid_lim=1.0, dt=1e-4, n_steps=60,
        x=x, vol=np.full(n, (dx / 2) ** 3), rho=1000.0, E=np.full(n, 1e4), nu=0.3,
        fibers=None, alpha=0.0, sigma_c=np.where(band, 30.0, 300.0), l0_scale=0.5, eta=1e-3,
        residual=5e-3, allow=~(bottom | pull),
        grips=[Grip(bottom, (0.0, 0.0, 0.0)), Grip(pull, (0.0, 1.5, 0.3), ramp=1e-3)],
        interface=(band, normals))


def batch_scenes(seed: int = 0, n_scenes: int = 64, n_lo: int = 4096, n_hi: int = 262144) -> list:
    """Independent scenes of uneven size for the batched form.

    Scene k: particle count log-uniform in [n_lo, n_hi] (8 per cell on a
    jittered 2^3 sub-lattice, so the count is 8x the box's cell count), a box
    of random aspect, a grid of 32^3-128^3 sized to the box (2x its longest
    edge plus 8 cells, rounded up to 16), E log-uniform in [1e3, 1e5],
    nu in [0.2, 0.45], one fiber direction uniform on the sphere, sigma_c in
    [50, 500], bottom layer clamped and one top edge pulled up at a velocity
    in [0.1, 2] m/s; dt = 5e-5, 300 substeps."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(n_scenes):
        target = math.exp(rng.uniform(math.log(n_lo), math.log(n_hi)))
        cells = max(1.0, target / 8.0)
        asp = np.exp(rng.uniform(-0.5, 0.5, 3)) * np.array([1.0, 0.5, 1.0])
        unit = (cells / float(np.prod(asp))) ** (1.0 / 3.0)
        ext = tuple(int(max(2, round(unit * a))) for a in asp)
        ng = int(min(128, max(32, math.ceil((2.0 * max(ext) + 8) / 16.0) * 16)))
        dx = 1.0 / ng
        lo = tuple((ng - e) // 2 for e in ext)
        x = jittered_lattice(lo, ext, dx, 2, 0.25, rng)
        n = x.shape[0]
        E = math.exp(rng.uniform(math.log(1e3), math.log(1e5)))
        nu = float(rng.uniform(0.2, 0.45))
        fib = np.tile(uniform_directions(1, rng), (n, 1))
        sig = float(rng.uniform(50.0, 500.0))
        pull = float(rng.uniform(0.1, 2.0))
        ylo, yhi = lo[1] * dx, (lo[1] + ext[1]) * dx
        bottom = x[:, 1] < ylo + dx
        top_edge = (x[:, 1] > yhi - dx) & (x[:, 0] < lo[0] * dx + dx)
        out.append(Scene(
            name=f"batch{seed}_{k}", n_grid=ng, grid_lim=1.0, dt=5e-5, n_steps=300,
            x=x, vol=np.full(n, (dx / 2) ** 3), rho=1000.0, E=np.full(n, E), nu=nu,
            fibers=fib, alpha=-1.0, sigma_c=np.full(n, sig), l0_scale=1.0, eta=1e-3,
            d0=rng.uniform(0.0, 0.05, n), allow=~(bottom | top_edge),
            grips=[Grip(bottom, (0.0, 0.0, 0.0)), Grip(top_edge, (0.0, pull, 0.0))]))
    return out


SCENES = {
    "plain_small": plain_small,
    "plain_1m": plain_1m,
    "peel_8m": peel_8m,
    "tiny_bar": tiny_bar,
    "knobs_drop": knobs_drop,
    "interface_peel": interface_peel,
}


# --------------------------------------------------------------------------- application
def lame(E, nu):
    """Lame parameters exactly as add_object forms them (anisompm.py:371-372)."""
    mu = E / (2.0 * (1.0 + nu))
    lam = E * nu / ((1.0 + nu) * (1.0 - 2.0 * nu))
    return mu, lam


def apply_scene(sim, sc: Scene, make_grip: Callable, make_collider: Callable, torch):
    """Populate a solver with ``sc`` through the reference setup API.

    ``make_grip(mask_tensor, velocity, ramp)`` and ``make_collider(spec)``
    return the boundary-condition objects the solver accepts (Python closures
    for the reference solver, device descriptors for this package)."""
    dev = sim.device
    x = torch.tensor(sc.x, dtype=torch.float64)
    vol = torch.tensor(sc.vol, dtype=torch.float64)
    fib = None if sc.fibers is None else torch.tensor(sc.fibers, dtype=torch.float64)
    sim.add_object(x, vol, rho=sc.rho, E=float(sc.E[0]), nu=sc.nu, fibers=fib, alpha=sc.alpha,
                   percentage=0.15, l0_scale=sc.l0_scale, eta=sc.eta, zeta=sc.zeta,
                   residual=sc.residual, allow_damage=True)
    if not np.all(sc.E == sc.E[0]):
        mu, lam = lame(sc.E, sc.nu)
        sim.mu[:] = torch.tensor(mu, dtype=torch.float64).to(dev)
        sim.lam[:] = torch.tensor(lam, dtype=torch.float64).to(dev)
    sim.sigma_c[:] = torch.tensor(sc.sigma_c, dtype=torch.float64).to(dev)
    if sc.d0 is not None:
        sim.d[:] = torch.tensor(sc.d0, dtype=torch.float64).to(dev)
    if sc.allow is not None:
        sim.allow[torch.tensor(~sc.allow).to(dev)] = False
    if sc.interface is not None:
        m, nrm = sc.interface
        sim.set_normal_isolation(torch.tensor(m).to(dev), torch.tensor(nrm, dtype=torch.float64)[m])
    for g in sc.grips:
        sim.particle_bc.append(make_grip(torch.tensor(g.mask).to(dev), tuple(float(c) for c in g.velocity),
                                         float(g.ramp)))
    for c in sc.colliders:
        sim.colliders.append(make_collider(c))
    return sim


def grip_factor(t: float, ramp: float) -> float:
    """Ramp factor of a grip at time t (1 when there is no ramp)."""
    return min(t / ramp, 1.0) if ramp > 0.0 else 1.0

"""Throughput of the AnisoMPM substep on B200: particle-steps/s, for the plain,
batched and differentiable forms.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--form all|plain|batched|adjoint|render] [--fd-dirs D]

Headline workload (``value``): the plain form on the 1,048,576-particle slab on
a 128^3 grid (seeded synthetic scene: vMF fibers about x with kappa=20,
log-normal E, sigma_c U(180,220), initial damage U(0,0.05), bottom clamped,
top edge pulled at 1 m/s, dt = 5e-5).  A step is one substep of the whole
scene, replayed from a captured CUDA graph of up to 100 substeps.  The
particle state (~290 MB with its grids) is larger than L2, so no flush is
needed between steps.

Beside it, in the same JSON line:
  batched     -- 64 independent scenes (log-uniform 4k-256k particles, grids
                 32^3-128^3, seeded) advanced by BatchedAnisoMPM.run_frame,
                 against the same 64 scenes advanced one after another by
                 AnisoMPM.run_frame (graph-captured too); aggregate
                 particle-steps/s of both and their ratio.
  fwd_adjoint -- differentiable.rollout on the 1M slab, 100 substeps as one
                 recorded segment sized to device memory (checkpoint_every
                 "auto": no recompute in the backward), and with checkpoints
                 every 10 (segments re-run in the backward): forward time,
                 forward+backward time and their ratio to the plain forward;
                 gradients with respect to E, fibers, sigma_c and v0 of the
                 mean squared distance to the final positions of a run with
                 E*1.2, fibers rotated 15 degrees about z and sigma_c*0.8,
                 their run-to-run spread, and an optional central-difference
                 check along random directions.
  render      -- the 1M slab's particles carrying one gaussian each
                 (positions x + F off0, covariances F cov0 F^T, damage tint)
                 and EWA-splatted to a 1280x720 image: median carry and
                 render times per frame.

Arms:
  ours       -- the sm_100a path.  ``value``: particle state resident in HBM,
                K substeps timed with CUDA events.  ``e2e``: the same substeps
                through the public API with the mutable state copied from
                pinned host memory before and back after every substep.
  reference  -- the reference algorithm on the host cores: the C oracle
                (a restatement of anisompm.py's substep) with all threads, on
                rank 0 only.

Multi-GPU: one independent replica per rank (the substep couples every
particle through the grid each step, so a single scene does not shard);
``value`` is the sum over ranks, time is the max over ranks.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "particle-steps/s at 1M pts: plain vs batched vs fwd+adjoint on 1 B200, rel err ≤1e-4"
UNIT = "particle-steps/s"
# algorithmic bytes per particle-step: mutable state x v F C d lap D_hist read
# and written (108 + 108 B) plus per-particle material read once (vol0 mass mu
# lam sigma_c eta zeta l0 residual A0 allow: 73 B)
BYTES_PER_PARTICLE = 216 + 73
# per active grid node and substep: momentum accumulate/read/v write/v read
# (16+16+12+12) + damage (8+8+4+4)
BYTES_PER_NODE = 80
# Per-launch DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) and
# warp instructions (smsp__inst_executed.sum) of the substep's kernels on this
# workload, from one ncu capture per kernel of `bench.py --form plain` (the
# command and the figures sit with the profile summaries); used for the roofline's
# `traffic` and its issue-bound floor (warp instructions / (4 schedulers x
# SMs x SM clock)).
NCU_KERNELS = {
    "k_subblocks": {"dram_bytes": 4203264, "warp_inst": 1975877},
    "k_stress": {"dram_bytes": 195174912 + 62206208, "warp_inst": 39083888},
    "k_bounds": {"dram_bytes": 4864, "warp_inst": 172},
    "k_p2g_tiles": {"dram_bytes": 96181760 + 5001984, "warp_inst": 56973418},
    "k_g2p": {"dram_bytes": 54698240 + 46928640, "warp_inst": 53436416},
}
P2G_KERNELS = ("k_subblocks", "k_stress", "k_bounds", "k_p2g_tiles")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--form", default="all", choices=["all", "plain", "batched", "adjoint", "render"])
    ap.add_argument("--fd-dirs", type=int, default=32,
                    help="central-difference directions of the adjoint check, on a pre-fracture window of the 1M "
                         "scene (the first --fd-window substeps; the forward is bit-reproducible, so the float32 "
                         "differences are not blurred by summation order)")
    ap.add_argument("--fd-window", type=int, default=3,
                    help="substeps of the central-difference window (the 1M slab's damage drive first exceeds "
                         "its threshold at substep 4)")
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-late", action="store_true", help="skip the late-run (substeps 400-420) sample")
    ap.add_argument("--adj-steps", type=int, default=100,
                    help="substeps of the differentiable rollout (the workload's 100; fewer for profiling)")
    return ap.parse_args()


# ------------------------------------------------------------------ clocks
class ClockSampler:
    """nvidia-smi samples during the timed region (median SM clock, reasons)."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            t0 = time.time()
            while not self.lines and time.time() - t0 < 3.0:   # sampling has started
                time.sleep(0.02)
        except (OSError, ValueError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, val in zip(names, f[5:9]):
                if val.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


# ------------------------------------------------------------------ helpers
def sm_count(torch):
    return torch.cuda.get_device_properties(torch.cuda.current_device()).multi_processor_count


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def build_sim(torch, device, seed):
    import peel_mpm_b200 as pm
    from peel_mpm_b200 import scenes
    sc = scenes.plain_1m(seed=seed)
    sim = pm.AnisoMPM(n_grid=sc.n_grid, grid_lim=sc.grid_lim, dt=sc.dt, gravity=tuple(sc.gravity),
                      grid_damp=sc.grid_damp, f_clamp=sc.f_clamp, damage_every=sc.damage_every, device=device)

    def mk_col(c):
        raise AssertionError("scene has no colliders")

    scenes.apply_scene(sim, sc, pm.grip_bc, mk_col, torch)
    return sim, sc


def time_kernels(torch, sim, steps, t0):
    """Per-kernel device time (ms per launch) via events around each C-ABI piece."""
    from peel_mpm_b200 import _lib
    grips, _ = sim._descriptors()
    prm = sim._build_params(grips)
    P = sim._particles()
    lib = sim._lib
    s = torch.cuda.current_stream()
    sp = s.cuda_stream
    ws, nb = sim._ws.data_ptr(), sim._ws_bytes
    names = ["bin", "p2g", "grid", "g2p"]
    acc = {k: 0.0 for k in names}
    for i in range(steps):
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(5)]
        clk = sim._clock(t0 + i * sim.dt, sim._step)
        ev[0].record(s)
        _lib.check(lib.pm_set_clock(C.byref(prm), ws, nb, sim.n, C.byref(clk), sp))
        _lib.check(lib.pm_bin(C.byref(prm), C.byref(P), ws, nb, sp))
        ev[1].record(s)
        _lib.check(lib.pm_p2g(C.byref(prm), C.byref(P), ws, nb, sp))
        ev[2].record(s)
        _lib.check(lib.pm_grid_update(C.byref(prm), ws, nb, sim.n, sp))
        ev[3].record(s)
        _lib.check(lib.pm_g2p(C.byref(prm), C.byref(P), ws, nb, sp))
        ev[4].record(s)
        sim._step += 1
        torch.cuda.synchronize()
        for k in range(4):
            acc[names[k]] += ev[k].elapsed_time(ev[k + 1])
    return {k: v / steps for k, v in acc.items()}


def cpu_baseline(torch, device, sample_steps=3):
    """The oracle port on the host cores: full 1M scene, a few substeps.
    The same substeps run on the GPU from the same initial state give the
    line's ``parity`` key (relative L2 per field after 1 + sample_steps
    substeps)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as orc
    from peel_mpm_b200 import scenes
    sc = scenes.plain_1m()
    cores = os.cpu_count() or 1
    sim = orc.OracleSim(sc, np.float32, nthreads=cores, scatter_mode=1)
    sim.substep(0.0)
    t = time.perf_counter()
    for i in range(sample_steps):
        sim.substep((i + 1) * sc.dt)
    dt = time.perf_counter() - t
    base = {"value": sc.n * sample_steps / dt, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": f"{sample_steps} substeps of the 1,048,576-particle scene after 1 warm-up, "
                      f"C oracle with OpenMP on {cores} threads"}
    gpu, _ = build_sim(torch, device, seed=0)
    for i in range(sample_steps + 1):
        gpu.substep(i * sc.dt)
    torch.cuda.synchronize()
    errs = {}
    for f in ("x", "v", "F", "C", "d", "lap", "D_hist"):
        a = getattr(sim, f).astype(np.float64).ravel()
        b = getattr(gpu, f).detach().cpu().numpy().astype(np.float64).ravel()
        errs[f] = float(np.linalg.norm(a - b) / max(np.linalg.norm(a), 1e-30))
    parity = {"substeps": sample_steps + 1, "particles": sc.n, "rel_l2_vs_oracle": errs,
              "bound": {"x v F C": 1e-5, "d lap D_hist": "ten times the oracle's own reordering envelope (tests)"},
              "full_runs": "tests/test_gpu_parity_configs.py: 1M x 500, peel 1/8 x 200, 64-scene batch x 20"}
    return base, parity


# ------------------------------------------------------------------ arms
def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as orc
    from peel_mpm_b200 import scenes
    sc = scenes.plain_1m()
    cores = os.cpu_count() or 1
    sim = orc.OracleSim(sc, np.float32, nthreads=cores, scatter_mode=1)
    for i in range(args.warmup):
        sim.substep(i * sc.dt)
    t = time.perf_counter()
    for i in range(args.steps):
        sim.substep((args.warmup + i) * sc.dt)
    el = time.perf_counter() - t
    value = sc.n * args.steps / el
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * el / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "plain AnisoMPM substep, 1,048,576 particles, 128^3 grid (seeded slab)",
                       "particles": sc.n, "n_grid": sc.n_grid, "dt": sc.dt},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
                             "sample": f"{args.steps} substeps of the full scene, C oracle, {cores} threads"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_frames(sim, steps, t0, chunk=100):
    """``steps`` substeps as graph replays of up to ``chunk`` substeps."""
    done = 0
    while done < steps:
        k = min(chunk, steps - done)
        sim.run_frame(k, t0 + done * sim.dt)
        done += k


def bench_batched(torch, device, rank=0, world=1, max_over_ranks=lambda v: v, barrier=lambda: None, seed=0,
                  n_sub=20, reps=3):
    """BatchedAnisoMPM on 64 seeded scenes vs the same scenes one by one.
    Under N ranks the scenes are bin-packed across ranks (no communication);
    times are the max over ranks."""
    import peel_mpm_b200 as pm
    from peel_mpm_b200 import autotune, scenes
    all_scs = scenes.batch_scenes(seed=seed)
    mine = pm.partition_scenes([sc.n for sc in all_scs], world)[rank]
    scs = [all_scs[k] for k in mine]

    def build(sc):
        sim = pm.AnisoMPM(n_grid=sc.n_grid, grid_lim=sc.grid_lim, dt=sc.dt, gravity=tuple(sc.gravity),
                          grid_damp=sc.grid_damp, f_clamp=sc.f_clamp, damage_every=sc.damage_every,
                          device=device)
        scenes.apply_scene(sim, sc, pm.grip_bc, None, torch)
        return sim

    solo = [build(sc) for sc in scs]
    batch = pm.BatchedAnisoMPM([build(sc) for sc in scs])
    tuned = autotune.tune(batch)
    total = sum(sc.n for sc in all_scs)
    s = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for _ in range(2):
        batch.run_frame(n_sub, 0.0)
        for sim in solo:
            sim.run_frame(n_sub, 0.0)
    torch.cuda.synchronize()
    barrier()
    e0.record(s)
    for r in range(reps):
        batch.run_frame(n_sub, [(2 + r) * n_sub * sc.dt for sc in scs])
    e1.record(s)
    torch.cuda.synchronize()
    tb = max_over_ranks(e0.elapsed_time(e1) / reps)
    barrier()
    e0.record(s)
    for r in range(reps):
        for sim, sc in zip(solo, scs):
            sim.run_frame(n_sub, (2 + r) * n_sub * sc.dt)
    e1.record(s)
    torch.cuda.synchronize()
    ts = max_over_ranks(e0.elapsed_time(e1) / reps)
    # the same scenes with eager substeps (one C call per substep, no graphs)
    for sim in solo:
        sim.use_graphs = False
    barrier()
    e0.record(s)
    for sim, sc in zip(solo, scs):
        sim.run_frame(n_sub, 5 * n_sub * sc.dt)
    e1.record(s)
    torch.cuda.synchronize()
    te = max_over_ranks(e0.elapsed_time(e1))
    st = batch.status()
    passes = _batch_passes(scs)
    return {"value": total * n_sub / (tb * 1e-3), "unit": UNIT,
            "sequential_value": total * n_sub / (ts * 1e-3), "speedup_vs_sequential": ts / tb,
            "sequential_eager_value": total * n_sub / (te * 1e-3), "speedup_vs_sequential_eager": te / tb,
            "ms_per_substep": tb / n_sub, "sequential_ms_per_substep": ts / n_sub,
            "scenes": len(all_scs), "particles": total, "grids": sorted({sc.n_grid for sc in all_scs}),
            "scenes_per_rank": len(scs), "substeps_per_frame": n_sub, "frames": reps,
            "tuned": {"knobs": tuned, "candidates_ms": autotune._CACHE[autotune.bucket(batch)]["ms"]},
            "gpu_launches_per_substep": 7 + 3 * passes,
            "nonfinite": sum(x["nonfinite"] for x in st),
            "what": "64 scenes, log-uniform 4k-256k particles, one BatchedAnisoMPM.run_frame per frame (one CUDA "
                    "graph) vs AnisoMPM.run_frame per scene (one CUDA graph each; and eager, one C call per "
                    "substep); scenes bin-packed across ranks"}


def _batch_passes(scs):
    from peel_mpm_b200 import _lib
    return _lib.batch_workspace_layout([sc.n for sc in scs], [sc.n_grid for sc in scs]).ws.sort_passes


def _smooth_field(torch, xs, gen, comps, modes=6):
    """A smooth random field over normalised positions xs (N,3) in [0,1]^3:
    per component, a sum of ``modes`` cosines with wave vectors of integer
    components 0..2 (times pi), random phases and N(0,1) amplitudes, scaled
    to unit RMS.  Returns (N, comps)."""
    dev = xs.device
    out = []
    for _ in range(comps):
        k = torch.randint(0, 3, (modes, 3), device=dev, generator=gen).to(xs.dtype) * math.pi
        ph = torch.rand(modes, device=dev, generator=gen) * (2 * math.pi)
        a = torch.randn(modes, device=dev, generator=gen)
        f = (torch.cos(xs @ k.t() + ph) * a).sum(1)
        out.append(f / f.pow(2).mean().sqrt().clamp_min(1e-12))
    return torch.stack(out, 1)


def fd_check(torch, sim, sc, S0, step0, params0, fd_dirs, fd_window, every=2):
    """Central differences of the float32 forward against the adjoint's
    directional derivatives, on the first ``fd_window`` substeps of the
    scene, before any particle reaches the damage threshold (the history
    field D_hist stays zero; its largest value over every run is reported),
    with checkpoints every ``every`` substeps so that the backward re-runs
    segments.

    The loss is linear in the final velocities with smooth weights, reduced
    in float64: L = mean_p(w_v . v_T).  The directions are smooth fields too,
    a quarter each in E (relative), the fiber directions, sigma_c (relative)
    and v0, so that the response sums coherently over the particles and
    stands far above the float32 rounding of the state (an incoherent loss,
    such as the distance to a nearby target, sums rounding noise of the same
    order as its signal).  Positions are left out of the loss: a small
    perturbation moves them by less than their float32 spacing per substep
    (5e-8 m at x ~ 0.5 for dv = 1 mm/s), so their differences come in
    rounding steps.  Each group takes its own step h (sized to its signal)
    and each derivative is Richardson-extrapolated from h and 2h,
    (4 D(h) - D(2h)) / 3, with |D(h) - D(2h)| kept as the difference's own
    error estimate.  Errors are relative to the RMS derivative of the
    direction's group."""
    from peel_mpm_b200 import differentiable as dfx
    dev = sim.device
    E0, fib0, sig0, v00 = params0
    n = sc.n
    x0 = S0[0:3, :n].t().double()
    lo, hi = x0.min(0).values, x0.max(0).values
    xs = ((x0 - lo) / (hi - lo).clamp_min(1e-12)).float()
    gen = torch.Generator(device=dev).manual_seed(0)
    w_v = _smooth_field(torch, xs, gen, 3).double()

    dh_max = [0.0]

    def run(E, fib, sig, v0):
        sim._S.copy_(S0)
        sim._step = step0
        mu, lam, A0 = dfx.material(E, sc.nu, fib, sc.alpha)
        vT = dfx.rollout(sim, fd_window, mu=mu, lam=lam, sigma_c=sig, A0=A0, v0=v0,
                         checkpoint_every=every, outputs="v")
        dh_max[0] = max(dh_max[0], float(sim.D_hist.max()))
        return (w_v * vT.double()).sum(1).mean()

    E = E0.clone().requires_grad_(True)
    fib = fib0.clone().requires_grad_(True)
    sig = sig0.clone().requires_grad_(True)
    v0 = v00.clone().requires_grad_(True)
    run(E, fib, sig, v0).backward()
    gw = (E.grad.double(), fib.grad.double(), sig.grad.double(), v0.grad.double())
    groups = ("E", "fibers", "sigma_c", "v0")
    steps = {"E": 5e-2, "fibers": 2e-2, "sigma_c": 2e-2, "v0": 1e-2}
    rows = []
    with torch.no_grad():
        dh_before = float(S0[26, :n].max())
        for k in range(fd_dirs):
            g = k % 4
            dirs = [torch.zeros_like(E0), torch.zeros_like(fib0), torch.zeros_like(sig0), torch.zeros_like(v00)]
            if g == 0:
                dirs[0] = E0 * _smooth_field(torch, xs, gen, 1)[:, 0]
            elif g == 1:
                dirs[1] = _smooth_field(torch, xs, gen, 3)
            elif g == 2:
                dirs[2] = sig0 * _smooth_field(torch, xs, gen, 1)[:, 0]
            else:
                dirs[3] = _smooth_field(torch, xs, gen, 3)
            base = (E0, fib0, sig0, v00)

            h = steps[groups[g]]

            def L(t):
                return float(run(*[b + t * d for b, d in zip(base, dirs)]))
            D1 = (L(h) - L(-h)) / (2 * h)
            D2 = (L(2 * h) - L(-2 * h)) / (4 * h)
            fdv = (4 * D1 - D2) / 3
            an = float(sum((a * d.double()).sum() for a, d in zip(gw, dirs)))
            rows.append((groups[g], an, fdv, abs(D1 - D2)))
        run(*base)
        d_grow = float((sim.d - S0[24, :n]).max())
    out = {"directions": fd_dirs, "h": steps, "window_substeps": fd_window, "checkpoint_every": every,
           "loss": "mean(w_v . v_T), smooth w_v, float64 reduction",
           "directions_kind": "smooth fields (6 cosine modes): E*f, fibers f, sigma_c*f, v0 f",
           "D_hist_max_before": dh_before, "D_hist_max_over_runs": dh_max[0],
           "d_growth_max": d_grow, "groups": {}}
    worst = 0.0
    for gname in groups:
        r = [x for x in rows if x[0] == gname]
        if not r:
            continue
        scale = math.sqrt(sum(x[2] ** 2 for x in r) / len(r))
        if scale == 0.0:
            out["groups"][gname] = {"directions": len(r), "rms_fd": 0.0,
                                    "max_abs_adjoint": max(abs(x[1]) for x in r)}
            continue
        errs = [abs(x[1] - x[2]) / scale for x in r]
        worst = max(worst, max(errs))
        out["groups"][gname] = {"directions": len(r), "rms_fd": scale, "median_rel_err": float(np.median(errs)),
                                "max_rel_err": max(errs), "fd_self_err": max(x[3] for x in r) / scale}
    out["max_rel_err"] = worst
    out["frac_below_1e-3"] = float(np.mean([abs(x[1] - x[2]) / max(out["groups"][x[0]].get("rms_fd", 0.0), 1e-300)
                                            < 1e-3 for x in rows]))
    return out


def bench_adjoint(torch, device, n_steps=100, every=10, fd_dirs=32, fd_window=3):
    """Forward and forward+backward of differentiable.rollout on the 1M slab,
    with checkpoints every ``every`` substeps (the backward re-runs the
    segments) and with one segment sized to device memory (every substep
    recorded during the forward: nothing re-run)."""
    import math
    from peel_mpm_b200 import differentiable as dfx
    sim, sc = build_sim(torch, device, seed=0)
    dev = sim.device
    f32 = torch.float32
    S0 = sim._S.clone()
    step0 = sim._step
    E0 = torch.tensor(sc.E, dtype=f32, device=dev)
    fib0 = torch.tensor(sc.fibers, dtype=f32, device=dev)
    sig0 = torch.tensor(sc.sigma_c, dtype=f32, device=dev)
    v00 = torch.zeros(sc.n, 3, dtype=f32, device=dev)

    def forward(E, fib, sig, v0, k=every, steps=n_steps):
        sim._S.copy_(S0)
        sim._step = step0
        mu, lam, A0 = dfx.material(E, sc.nu, fib, sc.alpha)
        return dfx.rollout(sim, steps, mu=mu, lam=lam, sigma_c=sig, A0=A0, v0=v0, checkpoint_every=k)

    # loss: mean squared distance of the final positions to those of a run with
    # E x 1.2, fibers rotated 15 degrees about z and sigma_c x 0.8
    t = math.radians(15.0)
    rz = torch.tensor([[math.cos(t), -math.sin(t), 0.0], [math.sin(t), math.cos(t), 0.0], [0.0, 0.0, 1.0]],
                      device=dev)
    with torch.no_grad():
        target = forward(E0 * 1.2, fib0 @ rz.t(), sig0 * 0.8, v00).clone()

    def loss_of(xT, tgt=None):
        return ((xT - (target if tgt is None else tgt)) ** 2).sum(1).mean()

    s = torch.cuda.current_stream()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]

    def timed(k):
        res = prev = None
        for rep in range(3):                      # the first two warm up (graph capture, allocations)
            E = E0.clone().requires_grad_(True)
            fib = fib0.clone().requires_grad_(True)
            sig = sig0.clone().requires_grad_(True)
            v0 = v00.clone().requires_grad_(True)
            torch.cuda.synchronize()
            ev[0].record(s)
            xT = forward(E, fib, sig, v0, k)
            loss = loss_of(xT)
            ev[1].record(s)
            loss.backward()
            ev[2].record(s)
            torch.cuda.synchronize()
            prev = None if res is None else res[2:6]
            res = (ev[0].elapsed_time(ev[1]), ev[0].elapsed_time(ev[2]), E.grad, fib.grad, sig.grad, v0.grad,
                   float(loss.detach()))
        return res, prev

    def rel(ga, gb):   # largest relative difference over the four gradients
        return max(float((a - b).norm() / max(float(b.norm()), 1e-30)) for a, b in zip(ga, gb))

    (fwd_k, tot_k, *g_k, _), g_k_prev = timed(every)
    g_k = tuple(g_k)
    k_auto = dfx.auto_segment(sim, n_steps)
    (fwd_ms, tot_ms, gE, gF, gS, gV, L0), g_prev = timed(k_auto)
    gdiff = rel((gE, gF, gS, gV), g_k)
    gspread = rel((gE, gF, gS, gV), g_prev)   # the same computation run twice
    gspread_k = rel(g_k, g_k_prev)
    # the plain forward of the same 100 substeps (no checkpoints, no tape), for the ratio
    plain = []
    for rep in range(3):
        sim._S.copy_(S0)
        sim._step = step0
        torch.cuda.synchronize()
        ev[0].record(s)
        run_frames(sim, n_steps, 0.0, chunk=n_steps)
        ev[1].record(s)
        torch.cuda.synchronize()
        plain.append(ev[0].elapsed_time(ev[1]))
    plain_ms = min(plain[1:])
    fd = fd_check(torch, sim, sc, S0, step0, (E0, fib0, sig0, v00), fd_dirs, fd_window) if fd_dirs > 0 else None
    return {"plain_forward_ms": plain_ms, "forward_ms": fwd_ms, "forward_backward_ms": tot_ms,
            "ratio": tot_ms / plain_ms, "ratio_vs_rollout_forward": tot_ms / fwd_ms,
            "value": sc.n * n_steps / (tot_ms * 1e-3), "unit": UNIT + " (forward+backward)",
            "substeps": n_steps, "checkpoint_every": k_auto,
            "segment_gb": dfx.segment_bytes(sim, k_auto) / 1e9,
            "checkpointed": {"checkpoint_every": every, "forward_ms": fwd_k, "forward_backward_ms": tot_k,
                             "ratio": tot_k / plain_ms, "segment_gb": dfx.segment_bytes(sim, every) / 1e9,
                             "grad_rel_diff_vs_one_segment": gdiff,
                             "grad_rel_diff_run_to_run": gspread_k},
            "grad_rel_diff_run_to_run": gspread,
            "particles": sc.n, "loss": L0,
            "grad_norms": {"E": float(gE.norm()), "fibers": float(gF.norm()), "sigma_c": float(gS.norm()),
                           "v0": float(gV.norm())},
            "fd_check": fd}


def bench_render(torch, device, sim, frames=10, warmup=3, width=1280, height=720):
    """Gaussian carrying + EWA splat rendering of the 1M slab: one gaussian per
    particle (isotropic, radius dx/2, coloured by height, tinted by damage),
    a 1280x720 camera facing the slab, tau from the median depth."""
    from peel_mpm_b200.render import Camera, carry_gaussians, render_gaussians, world_map
    dev = sim.device
    x = sim.x
    n = sim.n
    lo, hi = x.min(0).values, x.max(0).values
    c = (0.5 * (lo + hi)).cpu().numpy()
    ext = float((hi - lo).max())
    cam = Camera(R=np.eye(3), T=-c + np.array([0.0, 0.0, 2.0 * ext]), fx=1.6 * width, fy=1.6 * width,
                 width=width, height=height, device=dev)
    bind = torch.arange(n, dtype=torch.int32, device=dev)
    off0 = torch.zeros((n, 3), dtype=torch.float32, device=dev)
    r = 0.5 * sim.dx
    cov0 = (torch.eye(3, device=dev) * r * r).expand(n, 3, 3).contiguous()
    h = (x[:, 1] - lo[1]) / max(float(hi[1] - lo[1]), 1e-6)
    col0 = torch.stack([0.9 - 0.5 * h, 0.5 + 0.3 * h, 0.2 + 0.6 * h], 1).contiguous()
    aff = world_map(device=dev)   # built once: no host-to-device copy inside the timed calls
    s = torch.cuda.current_stream()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
    carry, render = [], []
    for f in range(warmup + frames):
        ev[0].record(s)
        pos, cov, col = carry_gaussians(sim, bind, off0, cov0, col0, aff, crack_tint=0.6, check_bind=False)
        ev[1].record(s)
        img = render_gaussians(cam, pos, cov, col, None, bg=(1.0, 1.0, 1.0), r_max=12)
        ev[2].record(s)
        torch.cuda.synchronize()
        if f >= warmup:
            carry.append(ev[0].elapsed_time(ev[1]))
            render.append(ev[1].elapsed_time(ev[2]))
    carry_ms, render_ms = statistics.median(carry), statistics.median(render)
    hbm, kind = peaks()
    carry_bytes = n * (4 + 48 + 4 + 12 + 36 + 12 + 12 + 60)   # bind, F x d, off0 cov0 color0 in; pos cov color out
    return {"gaussians": n, "width": width, "height": height, "r_max": 12,
            "carry_ms": carry_ms, "render_ms": render_ms, "frame_ms": carry_ms + render_ms,
            "value": n / ((carry_ms + render_ms) * 1e-3), "unit": "gaussians/s (carry + render)",
            "carry_roofline": {"bound": "hbm", "achieved": carry_bytes / (carry_ms * 1e-3) / 1e9, "peak": hbm,
                               "frac": carry_bytes / (carry_ms * 1e-3) / 1e9 / hbm, "unit": "GB/s",
                               "peak_kind": kind, "algorithmic_bytes": carry_bytes},
            "image_mean": float(img.mean())}


def run_ours(args):
    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    device = f"cuda:{local}"
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    def barrier():
        if world > 1:
            dist.barrier(device_ids=[local])

    def max_over_ranks(v):
        if world == 1:
            return v
        t = torch.tensor([v], device=device, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    sim, sc = build_sim(torch, device, seed=rank)
    n = sim.n
    from peel_mpm_b200 import autotune
    tuned = autotune.tune(sim)       # launch knobs for this size bucket (state restored afterwards)
    t0 = 0.0
    chunk = min(100, args.steps)
    for i in range(args.warmup):
        sim.run_frame(chunk, t0)
    torch.cuda.synchronize()
    barrier()

    s = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clocks:
        torch.cuda.synchronize()
        barrier()
        e0.record(s)
        run_frames(sim, args.steps, t0, chunk)
        e1.record(s)
        torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    barrier()
    ms_max = max_over_ranks(ms)
    value = world * n * args.steps / (ms_max * 1e-3)
    st = sim.status()
    n_active = st["n_active_blocks"] * 64

    # late-run sample: the scene's state around substep 400 of its 500 (fractured,
    # more active blocks), 20 substeps timed the same way
    late = None
    if not args.no_late:
        # a fresh copy of the scene advanced to substep 400 (the timed run above
        # went past the scene's 500 substeps)
        lsim, _ = build_sim(torch, device, seed=rank)
        for knob in autotune.KNOBS:
            setattr(lsim, knob, getattr(sim, knob))
        k = 20
        run_frames(lsim, 400 - k, 0.0, 100)
        # substeps 380-400 as one k-substep frame: captures the frame's graph
        # outside the timed region
        run_frames(lsim, k, lsim._step * lsim.dt, k)
        torch.cuda.synchronize()
        barrier()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(s)
        run_frames(lsim, k, lsim._step * lsim.dt, k)
        b.record(s)
        torch.cuda.synchronize()
        late_ms = max_over_ranks(a.elapsed_time(b))
        st_late = lsim.status()
        late = {"substeps": f"{lsim._step - k}-{lsim._step}", "ms_per_step": late_ms / k,
                "value": world * n * k / (late_ms * 1e-3), "unit": UNIT,
                "n_active_blocks": st_late["n_active_blocks"], "nonfinite": st_late["nonfinite"]}
        del lsim

    # e2e: mutable state from pinned host memory in, back out, every substep
    e2e = None
    if not args.no_e2e:
        k = min(args.steps, 20)
        nplanes = 27
        host = torch.empty((nplanes, sim._S.shape[1]), dtype=torch.float32, pin_memory=True)
        host.copy_(sim._S[:nplanes])
        for i in range(max(3, args.warmup)):   # untimed: the first eager calls set up the torch op and workspace
            sim._S[:nplanes].copy_(host, non_blocking=True)
            sim.substep(sim._step * sim.dt)
            host.copy_(sim._S[:nplanes], non_blocking=True)
        torch.cuda.synchronize()
        barrier()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(s)
        step0 = sim._step
        for i in range(k):
            sim._S[:nplanes].copy_(host, non_blocking=True)
            sim.substep((step0 + i) * sim.dt)
            host.copy_(sim._S[:nplanes], non_blocking=True)
        b.record(s)
        torch.cuda.synchronize()
        e2e_ms = max_over_ranks(a.elapsed_time(b))
        nbytes = nplanes * sim._S.shape[1] * 4
        e2e = {"value": world * n * k / (e2e_ms * 1e-3), "unit": UNIT, "h2d_bytes_per_step": nbytes,
               "d2h_bytes_per_step": nbytes, "steps": k,
               "what": "AnisoMPM.substep with x,v,F,C,d,lap,D_hist copied from pinned host before and to "
                       "pinned host after every substep"}

    # per-kernel times for the roofline (separate pass, events around each piece)
    kt = time_kernels(torch, sim, min(args.steps, 20), (sim._step) * sim.dt)
    hbm, peak_kind = peaks()
    p2g_bytes = n * (108 + 73 + 4 + 12) + n_active * 24
    g2p_bytes = n * (4 + 48 + 100) + n_active * 20
    dom = max(("p2g", "g2p"), key=lambda k: kt[k])
    alg = p2g_bytes if dom == "p2g" else g2p_bytes
    achieved = alg / (kt[dom] * 1e-3) / 1e9
    step_bytes = n * BYTES_PER_PARTICLE + n_active * BYTES_PER_NODE
    kern = P2G_KERNELS if dom == "p2g" else ("k_g2p",)
    known = all(NCU_KERNELS[k]["dram_bytes"] is not None for k in kern) and n == 1048576
    traffic = sum(NCU_KERNELS[k]["dram_bytes"] for k in kern) if known else None
    clk = clocks.summary().get("sm_mhz") or 1965.0
    floor_ms = (sum(NCU_KERNELS[k]["warp_inst"] for k in kern) / (4 * sm_count(torch) * clk * 1e6) * 1e3
                if known else None)
    roof = {"bound": "hbm",
            "kernel": " + ".join(kern) + (" (constitutive + P2G)" if dom == "p2g" else " (G2P)"),
            "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm, "peak_kind": peak_kind,
            "traffic": traffic, "traffic_over_algorithmic": (traffic / alg) if traffic else None,
            "algorithmic_bytes_per_launch": alg,
            "issue_floor": None if floor_ms is None else {
                "warp_instructions": sum(NCU_KERNELS[k]["warp_inst"] for k in kern), "floor_ms": floor_ms,
                "frac": floor_ms / kt[dom], "what": "warp instructions / (4 schedulers x SMs x SM clock)"},
            "kernel_ms": {k: round(v, 5) for k, v in kt.items()},
            "whole_step": {"achieved": step_bytes / (ms / args.steps * 1e-3) / 1e9,
                           "frac": step_bytes / (ms / args.steps * 1e-3) / 1e9 / hbm,
                           "bytes_per_step": step_bytes}}

    forms = {}
    if args.form in ("all", "batched"):   # every rank takes its share of the scenes
        forms["batched"] = bench_batched(torch, device, rank, world, max_over_ranks, barrier)
    if rank == 0 and args.form in ("all", "render"):
        forms["render"] = bench_render(torch, device, sim)
    if rank == 0 and args.form in ("all", "adjoint"):
        forms["fwd_adjoint"] = bench_adjoint(torch, device, n_steps=args.adj_steps, every=min(10, args.adj_steps),
                                             fd_dirs=args.fd_dirs, fd_window=args.fd_window)

    cpu = parity = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu, parity = cpu_baseline(torch, device)

    # clock, keys (+ first digit histogram), 3 per radix pass but the first's histogram, sub-block list,
    # stress, tiles, compact, grid, g2p
    launches_per_step = 7 + 3 * sim_passes(sim)
    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": {"workload": "plain AnisoMPM substep, 1,048,576 particles, 128^3 grid (seeded slab)",
                           "particles": n, "n_grid": sim.n_grid, "dt": sim.dt, "parallelism": f"replicas{world}",
                           "l2": "inputs larger than L2 (particle state ~290 MB)",
                           "graph_substeps": chunk},
                "tuned": {"knobs": tuned, "candidates_ms": autotune._CACHE[autotune.bucket(sim)]["ms"],
                          "substeps_per_candidate": autotune._CACHE[autotune.bucket(sim)]["substeps"]},
                "clocks": clocks.summary(), "roofline": roof, "cpu_baseline": cpu, "e2e": e2e,
                "gpu_launches": launches_per_step * args.steps, "status": st, "late_run": late,
                "parity": parity}
        line.update(forms)
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


def sim_passes(sim):
    from peel_mpm_b200 import _lib
    return _lib.workspace_layout(sim.n, sim.n_grid).sort_passes


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()

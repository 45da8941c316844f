"""Many independent AnisoMPM scenes advanced by one set of launches per substep.

``BatchedAnisoMPM(sims)`` packs the particle planes of existing ``AnisoMPM``
objects into one device tensor (scene after scene) and re-points every
scene's attribute views into it, so ``sims[k].x`` etc. keep working and show
the batched results.  A substep of the batch runs the same kernels as
``AnisoMPM.substep`` once over all scenes: one key pass, one radix sort of all
scenes' keys (each scene owns a range of sort blocks), one P2G over sorted
ranges (segments never cross scenes), one grid update over the active blocks
of all grids and one G2P whose CTAs each belong to one scene.  Each scene
keeps its own grid size, dx, dt, parameters, grips, colliders, clock and step
counter.  ``run_frame`` captures the frame in a CUDA graph whose per-scene
times come from a device table, as ``AnisoMPM.run_frame`` does.

The reference has no batch API; the batch replaces a Python loop that calls
``run_frame`` (anisompm.py:805-807) on each scene in turn.
"""
from __future__ import annotations

import ctypes as C
from typing import Optional, Sequence

import torch

from . import _lib
from .anisompm import N_PLANES, _PLANES, AnisoMPM, _stride_for


class BatchedAnisoMPM:
    def __init__(self, sims: Sequence[AnisoMPM], use_graphs: bool = True):
        sims = list(sims)
        if not sims:
            raise ValueError("a batch needs at least one scene")
        if len(sims) > _lib.PM_MAX_BATCH_SCENES:
            raise ValueError(f"at most {_lib.PM_MAX_BATCH_SCENES} scenes per batch")
        dev = sims[0].device
        for s in sims:
            if s.device != dev:
                raise ValueError("all scenes of a batch must live on one device")
            if s._batch is not None:
                raise ValueError("a scene can belong to one batch at a time")
            if s.n == 0:
                raise ValueError("every scene of a batch needs particles")
        self.sims = sims
        self.device = dev
        self.use_graphs = use_graphs
        self.p2g_ctas_per_sm = 0  # launch knobs for the whole batch (0 = library defaults)
        self.grid_ctas_per_sm = 0
        self.stress_ctas_per_sm = 0
        self.g2p_ctas_per_sm = 0
        self._lib = _lib.load()
        self._graphs = {}
        self._ws = None
        self._pack()

    # ------------------------------------------------------------------ packing
    def _knobs(self):
        return (int(self.p2g_ctas_per_sm), int(self.grid_ctas_per_sm), int(self.stress_ctas_per_sm),
                int(self.g2p_ctas_per_sm))

    def _pack(self):
        sims, dev = self.sims, self.device
        self.ns = [s.n for s in sims]
        self.grids = [s.n_grid for s in sims]
        self.pb = [0]
        for n in self.ns:
            self.pb.append(self.pb[-1] + n)
        total = self.pb[-1]
        S = torch.zeros((N_PLANES, _stride_for(total)), device=dev, dtype=torch.float32)
        A = torch.empty(total, device=dev, dtype=torch.bool)
        IM = torch.empty(total, device=dev, dtype=torch.bool)
        for k, s in enumerate(sims):
            a, b = self.pb[k], self.pb[k + 1]
            S[:, a:b] = s._S[:, :s.n]
            A[a:b] = s._allow
            IM[a:b] = s._imask
        for k, s in enumerate(sims):
            a, b = self.pb[k], self.pb[k + 1]
            s._S, s._allow, s._imask = S[:, a:b], A[a:b], IM[a:b]
            s._P = None
            s._ws = None          # a standalone substep re-creates its own workspace
            s._graphs.clear()
            s._batch = self
        self._S, self._allow, self._imask = S, A, IM
        self.n = total
        self._n_arr = (C.c_int64 * len(sims))(*self.ns)
        self._g_arr = (C.c_int32 * len(sims))(*self.grids)
        self._tag = None
        self._tag_keys = None
        self._params_keys = None
        self._prm_arr = None
        self._P = None
        need = _lib.batch_workspace_size(self.ns, self.grids)
        self._ws = torch.empty(need, dtype=torch.uint8, device=dev)
        self._ws_bytes = need
        self._ws_ready = False
        self._graphs.clear()

    def unpack(self):
        """Give every scene its own storage again (a copy of the batch's
        current state) and release the batch."""
        for k, s in enumerate(self.sims):
            n = s.n
            S = torch.zeros((N_PLANES, _stride_for(n)), device=self.device, dtype=torch.float32)
            S[:, :n] = s._S
            s._S, s._allow, s._imask = S, s._allow.clone(), s._imask.clone()
            s._P = None
            s._graphs.clear()
            s._batch = None
        self._release()
        self.sims = []

    def _release(self):
        if self._ws is not None and self._lib is not None:
            self._lib.pm_batch_workspace_release(self._ws.data_ptr())
        self._graphs.clear()
        self._ws = None

    def __del__(self):
        try:
            self._release()
        except Exception:
            pass

    # ------------------------------------------------------------------ device state
    def _sync_descriptors(self):
        """Grip tags, parameters and the particle descriptor of the batch;
        uploads parameters when a scene's changed (no graph recapture: the
        kernels read them from the workspace)."""
        grips_all = []
        for s in self.sims:
            grips, calls = s._descriptors()
            if calls:
                raise NotImplementedError("batched scenes accept grip_bc descriptors only, not callables")
            grips_all.append(grips)
        tag_keys = tuple(tuple(id(g) for g in gs) for gs in grips_all)
        if tag_keys != self._tag_keys:
            if any(grips_all):
                tag = torch.full((self.n,), -1, dtype=torch.int8, device=self.device)
                for k, (s, gs) in enumerate(zip(self.sims, grips_all)):
                    s._tag_key = None
                    s._grip_tags(gs)
                    if s._tag is not None:
                        tag[self.pb[k]:self.pb[k + 1]] = s._tag
                self._tag = tag
            else:
                self._tag = None
            self._tag_keys = tag_keys
            self._P = None
        prms = [s._build_params(gs) for s, gs in zip(self.sims, grips_all)]
        keys = tuple(s._params_key for s in self.sims) + self._knobs()
        if keys != self._params_keys or not self._ws_ready:
            arr = (_lib.pm_params * len(prms))(*prms)
            for k in range(len(prms)):
                arr[k].p2g_ctas_per_sm = int(self.p2g_ctas_per_sm)
                arr[k].grid_ctas_per_sm = int(self.grid_ctas_per_sm)
                arr[k].stress_ctas_per_sm = int(self.stress_ctas_per_sm)
                arr[k].g2p_ctas_per_sm = int(self.g2p_ctas_per_sm)
            st = torch.cuda.current_stream(self.device).cuda_stream
            if not self._ws_ready:
                _lib.check(self._lib.pm_batch_workspace_init(self._ws.data_ptr(), self._ws_bytes, len(prms),
                                                             self._n_arr, arr, st), "pm_batch_workspace_init")
                self._ws_ready = True
            else:
                _lib.check(self._lib.pm_batch_set_params(self._ws.data_ptr(), self._ws_bytes, len(prms),
                                                         self._n_arr, arr, st), "pm_batch_set_params")
            self._prm_arr = arr
            self._params_keys = keys
        iface = any(s._iface_used for s in self.sims)
        if self._P is None or self._P_iface != iface:
            P = _lib.pm_particles()
            P.n = self.n
            P.plane_stride = self._S.stride(0)
            base = self._S.data_ptr()
            st = self._S.stride(0) * 4
            for name in ("x", "v", "F", "C", "d", "lap", "D_hist", "vol0", "mass", "mu", "lam", "sigma_c", "eta",
                         "zeta", "l0", "residual", "A0", "phi", "tau_last", "J_last"):
                setattr(P, name, base + _PLANES[name][0] * st)
            P.allow = self._allow.data_ptr()
            if iface:
                P.n_interface = base + _PLANES["n_interface"][0] * st
                P.interface_mask = self._imask.data_ptr()
                P.phi_shear = base + _PLANES["phi_shear"][0] * st
            P.grip_tag = None if self._tag is None else self._tag.data_ptr()
            self._P, self._P_iface = P, iface
        return self._P

    def _times(self, time0, n_sub):
        if isinstance(time0, (int, float)):
            t0 = [float(time0)] * len(self.sims)
        else:
            t0 = [float(t) for t in time0]
            if len(t0) != len(self.sims):
                raise ValueError("one start time per scene")
        return [[t0[k] + i * s.dt for k, s in enumerate(self.sims)] for i in range(n_sub)]

    def _clock_table(self, times):
        """Pinned host table of pm_clock, row i = substep i of every scene."""
        S = len(self.sims)
        rows = len(times)
        host = torch.empty(rows * S * C.sizeof(_lib.pm_clock), dtype=torch.uint8, pin_memory=True)
        clocks = (_lib.pm_clock * (rows * S)).from_address(host.data_ptr())
        for i, row in enumerate(times):
            for k, s in enumerate(self.sims):
                clocks[i * S + k] = s._clock(row[k], s._step + i)
        return host

    # ------------------------------------------------------------------ stepping
    def _launch(self, P, table_ptr, stream):
        _lib.check(self._lib.pm_batch_substep(len(self.sims), self._n_arr, self._g_arr, C.byref(P),
                                              self._ws.data_ptr(), self._ws_bytes, table_ptr, stream),
                   "pm_batch_substep")

    def substep(self, time=0.0):
        """One substep of every scene; ``time`` is one float for all scenes
        or one per scene."""
        self.run_frame(1, time, _graph=False)

    def run_frame(self, n_sub: int, time0=0.0, _graph: Optional[bool] = None):
        """n_sub substeps of every scene, scene k at time0[k] + i * dt_k."""
        n_sub = int(n_sub)
        if n_sub <= 0:
            return
        P = self._sync_descriptors()
        host = self._clock_table(self._times(time0, n_sub))
        use_graph = self.use_graphs if _graph is None else _graph
        row_bytes = len(self.sims) * C.sizeof(_lib.pm_clock)
        if not use_graph:
            table = torch.empty(host.numel(), dtype=torch.uint8, device=self.device)
            table.copy_(host, non_blocking=True)
            st = torch.cuda.current_stream(self.device).cuda_stream
            for i in range(n_sub):
                self._launch(P, table.data_ptr() + i * row_bytes, st)
            # keep the pinned source and device table alive until the copy and kernels ran
            self._eager_keep = (host, table)
        else:
            key = (n_sub, id(P), self._ws.data_ptr(), self._S.data_ptr()) + self._knobs()
            entry = self._graphs.get(key)
            if entry is None:
                table = torch.empty(host.numel(), dtype=torch.uint8, device=self.device)
                _lib.check(self._lib.pm_prepare(), "pm_prepare")
                torch.cuda.synchronize(self.device)
                g = torch.cuda.CUDAGraph()
                with torch.cuda.graph(g):
                    st = torch.cuda.current_stream().cuda_stream
                    for i in range(n_sub):
                        self._launch(P, table.data_ptr() + i * row_bytes, st)
                entry = (g, table, P)
                self._graphs[key] = entry
            g, table = entry[0], entry[1]
            table.copy_(host, non_blocking=True)
            g.replay()
            self._host_keep = host
        for s in self.sims:
            s._step += n_sub

    # ------------------------------------------------------------------ status
    def status(self):
        """Per-scene status counters (synchronises the current stream)."""
        S = len(self.sims)
        out = (_lib.pm_status_info * S)()
        if not self._ws_ready:
            self._sync_descriptors()
        st = torch.cuda.current_stream(self.device).cuda_stream
        _lib.check(self._lib.pm_batch_read_status(self._ws.data_ptr(), self._ws_bytes, S, self._n_arr, self._g_arr,
                                                  out, st), "pm_batch_read_status")
        return [{"nonfinite": int(o.nonfinite), "dense_subblocks": int(o.dense_subblocks),
                 "n_active_blocks": int(o.n_active_blocks),
                 "any_allow": int(o.any_allow)} for o in out]

    def check(self):
        st = self.status()
        bad = [k for k, s in enumerate(st) if s["nonfinite"]]
        if bad:
            raise FloatingPointError(f"scenes {bad} produced non-finite x or F")
        dense = [k for k, s in enumerate(st) if s["dense_subblocks"]]
        if dense:
            raise OverflowError(f"scenes {dense} exceeded the fixed-point headroom of their P2G sub-blocks")
        return st


def partition_scenes(sizes, world: int):
    """Assign scenes to ``world`` ranks by greedy bin packing on particle
    counts (largest first onto the least-loaded rank).  Returns one list of
    scene indices per rank, each in ascending order; scenes are independent,
    so ranks need no communication while they run."""
    if world < 1:
        raise ValueError("world must be >= 1")
    loads = [0] * world
    parts = [[] for _ in range(world)]
    for k in sorted(range(len(sizes)), key=lambda i: (-int(sizes[i]), i)):
        r = min(range(world), key=lambda j: (loads[j], j))
        parts[r].append(k)
        loads[r] += int(sizes[k])
    return [sorted(p) for p in parts]

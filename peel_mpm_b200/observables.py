"""Per-frame observables of the experiment loop, reduced on the device.

The reference's peel harness (peel_test.py:263-307) reads back, after every
frame, the peak damage drive phi per particle group (interface, flesh, peel),
the peak shear drive, mean / max damage and the broken fraction per group,
the mean height of a cap group, a NaN flag, and it detects the delamination
onset (first frame where more than 5% of the interface has d > 0.5) and
snapshots the state there.  Each of those reads synchronises the host with
the GPU.  ``FrameObservables.update(frame)`` enqueues the same reductions
(``pm_observe``: three kernel launches) into a per-frame device table and
the onset snapshot is taken on the device; ``read()`` synchronises once and
returns everything.

    obs = FrameObservables(sim, {"interface": m_if, "flesh": m_fl, "peel": m_pe},
                           max_frames=frames, onset_group="interface")
    for f in range(frames):
        sim.run_frame(n_sub, f / fps)
        obs.update(f)
    r = obs.read()     # r["table"][f]["interface"]["phi_max"], r["onset_frame"], ...
"""
from __future__ import annotations

import ctypes as C
from typing import Dict, Optional

import numpy as np
import torch

from . import _lib
from .anisompm import AnisoMPM

_FIELDS = ("phi_max", "phi_shear_max", "d_sum", "d_max", "n_broken", "count", "y_sum")


class FrameObservables:
    def __init__(self, sim: AnisoMPM, groups: Dict[str, torch.Tensor], max_frames: int,
                 d_threshold: float = 0.5, onset_group: Optional[str] = None, onset_fraction: float = 0.05,
                 snapshot: bool = True, per_particle_peaks: bool = True):
        if not 1 <= len(groups) <= _lib.PM_OBS_MAX_GROUPS:
            raise ValueError(f"1 to {_lib.PM_OBS_MAX_GROUPS} groups")
        self.sim = sim
        self.names = list(groups)
        dev = sim.device
        tag = torch.full((sim.n,), -1, dtype=torch.int8, device=dev)
        for g, name in enumerate(self.names):
            m = torch.as_tensor(groups[name], device=dev)
            if m.dtype == torch.bool:
                tag[m] = g
            else:
                tag[m.long()] = g
        self.group = tag
        self.max_frames = int(max_frames)
        self.table = torch.zeros((self.max_frames, len(self.names), _lib.PM_OBS_VALUES), dtype=torch.float32,
                                 device=dev)
        self.status = torch.tensor([-1, 0], dtype=torch.int32, device=dev)
        self.d_threshold = float(d_threshold)
        self.onset_group = -1 if onset_group is None else self.names.index(onset_group)
        self.onset_fraction = float(onset_fraction)
        n = sim.n
        self.phi_peak = torch.zeros(n, dtype=torch.float32, device=dev) if per_particle_peaks else None
        self.phi_shear_peak = torch.zeros(n, dtype=torch.float32, device=dev) if per_particle_peaks else None
        self.snap_d = torch.zeros(n, dtype=torch.float32, device=dev) if snapshot else None
        self.snap_x = torch.zeros((3, n), dtype=torch.float32, device=dev) if snapshot else None
        self._lib = _lib.load()

    def update(self, frame: int):
        """Enqueue the reductions of the current state into row ``frame``."""
        if not 0 <= frame < self.max_frames:
            raise IndexError("frame outside the table")
        sim = self.sim
        P = sim._particles()
        ptr = lambda t: None if t is None else t.data_ptr()
        with torch.cuda.device(sim.device):
            st = torch.cuda.current_stream().cuda_stream
            _lib.check(self._lib.pm_observe(C.byref(P), self.group.data_ptr(), len(self.names), self.d_threshold,
                                            self.table[frame].data_ptr(), ptr(self.phi_peak),
                                            ptr(self.phi_shear_peak), self.status.data_ptr(), self.onset_group,
                                            self.onset_fraction, int(frame), ptr(self.snap_d), ptr(self.snap_x),
                                            sim.n, st), "pm_observe")

    def read(self, frames: Optional[int] = None) -> dict:
        """Synchronise once and return the per-frame table, peaks, onset and
        snapshot.  Per group and frame: phi_max, phi_shear_max, d_mean,
        d_max, broken (fraction with d above the threshold), y_mean."""
        torch.cuda.synchronize(self.sim.device)
        t = self.table.cpu().numpy()
        nf = self.max_frames if frames is None else int(frames)
        rows = []
        for f in range(nf):
            row = {}
            for g, name in enumerate(self.names):
                v = dict(zip(_FIELDS, t[f, g, :7].tolist()))
                cnt = max(v["count"], 1.0)
                row[name] = {"phi_max": v["phi_max"], "phi_shear_max": v["phi_shear_max"],
                             "d_mean": v["d_sum"] / cnt, "d_max": v["d_max"], "broken": v["n_broken"] / cnt,
                             "y_mean": v["y_sum"] / cnt, "count": int(v["count"])}
            rows.append(row)
        status = self.status.cpu().numpy()
        peak = {name: float(t[:nf, g, 0].max()) if nf else 0.0 for g, name in enumerate(self.names)}
        return {"table": rows, "phi_peak_per_group": peak, "onset_frame": int(status[0]),
                "nonfinite": int(status[1]), "phi_peak": self.phi_peak, "phi_shear_peak": self.phi_shear_peak,
                "snap_d": self.snap_d if status[0] >= 0 else None,
                "snap_x": None if self.snap_x is None or status[0] < 0 else self.snap_x.t()}

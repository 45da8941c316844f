"""The C ABI exposed as torch ops: ``torch.ops.peelmpm.*``.

Registered with ``torch.library.custom_op`` so that the substep, the
eigensolver and the binning appear to PyTorch as ordinary operators (with
fake implementations for shape propagation and tracing), while the work is
done by ``libpeelmpm.so``:

* ``peelmpm::sym_eig(A, sweeps) -> (evals, evecs)`` -- anisompm.py:48-95;
* ``peelmpm::bin_sort(x, n_grid, inv_dx) -> (keys, perm)`` -- the reference's
  ``_node_index`` of the quadratic base cell, sorted, and its stable argsort;
* ``peelmpm::substep(planes!, allow, interface_mask?, grip_tag?, workspace!,
  params, clock, n)`` -- one ``AnisoMPM.substep`` (anisompm.py:593-803) on the
  solver's particle planes; ``params`` and ``clock`` are the ``pm_params`` /
  ``pm_clock`` structures as CPU byte tensors.
"""
from __future__ import annotations

import ctypes as C
from typing import Optional, Tuple

import torch
from torch import Tensor

from . import _lib

# plane offsets of the particle store, as AnisoMPM lays it out
from .anisompm import _PLANES


def _stream(dev) -> int:
    return torch.cuda.current_stream(dev).cuda_stream


@torch.library.custom_op("peelmpm::sym_eig", mutates_args=())
def sym_eig(A: Tensor, sweeps: int) -> Tuple[Tensor, Tensor]:
    lib = _lib.load()
    A = A.to(torch.float32).contiguous()
    n = A.shape[0]
    ev = torch.empty((n, 3), dtype=torch.float32, device=A.device)
    V = torch.empty((n, 3, 3), dtype=torch.float32, device=A.device)
    with torch.cuda.device(A.device):
        _lib.check(lib.pm_sym_eig(A.data_ptr(), n, int(sweeps), ev.data_ptr(), V.data_ptr(), _stream(A.device)),
                   "pm_sym_eig")
    return ev, V


@sym_eig.register_fake
def _(A, sweeps):
    return A.new_empty((A.shape[0], 3), dtype=torch.float32), A.new_empty((A.shape[0], 3, 3), dtype=torch.float32)


@torch.library.custom_op("peelmpm::bin_sort", mutates_args=())
def bin_sort(x: Tensor, n_grid: int, inv_dx: float) -> Tuple[Tensor, Tensor]:
    lib = _lib.load()
    n = x.shape[0]
    if x.stride(0) != 1:
        x = x.t().contiguous().t()
    ps = x.stride(1)
    need = _lib.bin_workspace_size(n, n_grid)   # the sort buffers only, no grids
    ws = torch.empty(need, dtype=torch.uint8, device=x.device)
    keys = torch.empty(n, dtype=torch.int32, device=x.device)
    perm = torch.empty(n, dtype=torch.int32, device=x.device)
    with torch.cuda.device(x.device):
        _lib.check(lib.pm_bin_sort(x.data_ptr(), n, ps, int(n_grid), float(inv_dx), keys.data_ptr(), perm.data_ptr(),
                                   ws.data_ptr(), need, _stream(x.device)), "pm_bin_sort")
    return keys.to(torch.int64), perm.to(torch.int64)


@bin_sort.register_fake
def _(x, n_grid, inv_dx):
    n = x.shape[0]
    return x.new_empty((n,), dtype=torch.int64), x.new_empty((n,), dtype=torch.int64)


def particles_struct(planes: Tensor, n: int, allow: Tensor, imask: Optional[Tensor], tag: Optional[Tensor]):
    """pm_particles over the solver's float32 planes (64 x stride)."""
    P = _lib.pm_particles()
    P.n = n
    P.plane_stride = planes.stride(0)
    base, st = planes.data_ptr(), planes.stride(0) * 4
    for name in ("x", "v", "F", "C", "d", "lap", "D_hist", "vol0", "mass", "mu", "lam", "sigma_c", "eta", "zeta",
                 "l0", "residual", "A0", "phi"):
        setattr(P, name, base + _PLANES[name][0] * st)
    P.allow = allow.data_ptr()
    if imask is not None:
        P.n_interface = base + _PLANES["n_interface"][0] * st
        P.interface_mask = imask.data_ptr()
        P.phi_shear = base + _PLANES["phi_shear"][0] * st
    P.grip_tag = None if tag is None else tag.data_ptr()
    P.tau_last = base + _PLANES["tau_last"][0] * st
    P.J_last = base + _PLANES["J_last"][0] * st
    return P


@torch.library.custom_op("peelmpm::substep", mutates_args=("planes", "workspace"))
def substep(planes: Tensor, allow: Tensor, interface_mask: Optional[Tensor], grip_tag: Optional[Tensor],
            workspace: Tensor, params: Tensor, clock: Tensor, n: int) -> None:
    lib = _lib.load()
    prm = _lib.pm_params.from_buffer_copy(params.numpy().tobytes())
    clk = _lib.pm_clock.from_buffer_copy(clock.numpy().tobytes())
    P = particles_struct(planes, n, allow, interface_mask, grip_tag)
    with torch.cuda.device(planes.device):
        _lib.check(lib.pm_substep(C.byref(prm), C.byref(P), workspace.data_ptr(), workspace.numel(), C.byref(clk),
                                  _stream(planes.device)), "pm_substep")


@substep.register_fake
def _(planes, allow, interface_mask, grip_tag, workspace, params, clock, n):
    return None


def struct_bytes(s) -> Tensor:
    """A ctypes structure as a CPU uint8 tensor (the op's params / clock)."""
    return torch.frombuffer(bytearray(bytes(s)), dtype=torch.uint8)

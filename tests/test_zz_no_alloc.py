"""The allocation-free binning entry point, pm_bin_sort_static.

It is for callers that cannot allocate device memory -- a host application
that owns every device allocation and hands a plugin only its input and
output buffers, or a latency-bound loop that must not call cudaMalloc/cudaFree
(they can synchronise the whole device).  Its sort scratch is a static array
inside libpeelmpm.so, so the call takes only positions and the two outputs.

This file is collected last on purpose: it runs after every other GPU test and
also passes on its own in a fresh process (the first call on the device sets
up the scratch address).
"""
import ctypes as C

import numpy as np
import pytest
import torch

from peel_mpm_b200 import _lib
import peel_mpm_b200 as pm

pytestmark = pytest.mark.gpu


def _static_bin(x_planes, n_grid, inv_dx):
    lib = _lib.load()
    n = x_planes.shape[1]
    keys = torch.empty(n, dtype=torch.int32, device=x_planes.device)
    perm = torch.empty(n, dtype=torch.int32, device=x_planes.device)
    rc = lib.pm_bin_sort_static(x_planes.data_ptr(), n, x_planes.stride(0), n_grid, inv_dx, keys.data_ptr(),
                                perm.data_ptr(), torch.cuda.current_stream().cuda_stream)
    return rc, keys, perm


@pytest.mark.parametrize("n_grid", [128, 36, 1024])
def test_static_binning_matches_workspace_binning_on_two_calls(n_grid):
    # the grids give keys of 21, 16 and 30 bits: 3, 2 and 4 radix passes, so
    # the result ends in either half of the static scratch
    # two calls in a row on different inputs: the second reuses the scratch the
    # first left behind and must still match the workspace entry point exactly
    for seed, n in ((11, 200_003), (12, _lib.PM_BIN_STATIC_MAX_N)):
        rng = np.random.default_rng(seed)
        x = torch.tensor(rng.uniform(-0.02, 1.02, size=(n, 3)).astype(np.float32), device="cuda")
        keys_ref, perm_ref = pm.bin_particles(x, n_grid, float(n_grid))
        rc, keys, perm = _static_bin(x.t().contiguous(), n_grid, float(n_grid))
        assert rc == _lib.PM_OK, _lib.load().pm_last_error()
        torch.cuda.synchronize()
        assert torch.equal(keys.to(torch.int64), keys_ref)     # integer output: bit-exact
        assert torch.equal(perm.to(torch.int64), perm_ref)


def test_static_binning_rejects_sizes_beyond_its_maximum():
    lib = _lib.load()
    n = _lib.PM_BIN_STATIC_MAX_N + 1
    x = torch.zeros(3, n, device="cuda")
    rc, _, _ = _static_bin(x, 64, 64.0)
    assert rc == _lib.PM_ERR_ARG
    assert b"PM_BIN_STATIC_MAX_N" in lib.pm_last_error()

"""The C-ABI library loads without a GPU, exports every entry point
include/peelmpm.h declares, and its structs match the ctypes binding."""
import ctypes as C
import os
import re

import pytest

from peel_mpm_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    src = open(os.path.join(ROOT, "include", "peelmpm.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(pm_\w+)\s*\(", src)))


def test_library_exports_every_declared_function():
    lib = _lib.load()
    declared = header_functions()
    assert len(declared) >= 15
    for name in declared:
        assert hasattr(lib, name), name
    assert set(declared) == set(_lib.EXPORTS)


def test_struct_layouts_match_binding():
    for name, (py, c) in _lib.check_layout().items():
        assert py == c, (name, py, c)


def test_abi_version():
    assert _lib.load().pm_abi_version() == 1


@pytest.mark.parametrize("n,ng", [(0, 4), (1, 8), (16384, 64), (1 << 20, 128), (8_847_360, 256), (1000, 96)])
def test_workspace_layout_is_aligned_and_disjoint(n, ng):
    L = _lib.workspace_layout(n, ng)
    offs = [L.ctrl, L.keys_a, L.keys_b, L.vals_a, L.vals_b, L.hist, L.block_mask, L.block_list, L.g_mom, L.g_dmg,
            L.g_vel, L.g_gd, L.payload, L.inv_perm, L.total]
    assert all(o % 256 == 0 for o in offs)
    assert offs == sorted(offs) and len(set(offs)) == len(offs)
    nn = max(n, 1)
    G = ng ** 3
    assert L.keys_b - L.keys_a >= 4 * nn and L.g_dmg - L.g_mom >= 16 * G and L.payload - L.g_gd >= 4 * G and L.inv_perm - L.payload >= 80 * nn and L.total - L.inv_perm >= 4 * nn
    assert L.sort_passes == 3 if ng >= 64 else L.sort_passes >= 1
    assert _lib.workspace_size(n, ng) == L.total


def test_argument_errors_without_device():
    lib = _lib.load()
    out = C.c_size_t(0)
    assert lib.pm_workspace_size(-1, 64, C.byref(out)) == _lib.PM_ERR_ARG
    assert b"bad" in lib.pm_last_error()
    assert lib.pm_workspace_size(10, 2, C.byref(out)) == _lib.PM_ERR_ARG
    assert lib.pm_workspace_size(10, 2048, C.byref(out)) == _lib.PM_ERR_ARG
    assert lib.pm_struct_size(99) == 0
    with pytest.raises(_lib.PeelMPMError):
        _lib.check(lib.pm_workspace_size(-5, 64, C.byref(out)), "size")

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
    assert _lib.load().pm_abi_version() == 2


@pytest.mark.parametrize("n,ng", [(0, 4), (1, 8), (16384, 64), (1 << 20, 128), (8_847_360, 256), (1000, 96)])
def test_workspace_layout_is_aligned_and_disjoint(n, ng):
    L = _lib.workspace_layout(n, ng)
    offs = [L.ctrl, L.keys_a, L.keys_b, L.vals_a, L.vals_b, L.hist, L.block_mask, L.block_list, L.g_mom, L.g_dmg,
            L.g_vel, L.g_gd, L.payload, L.inv_perm, L.work, L.total]
    assert all(o % 256 == 0 for o in offs)
    assert offs == sorted(offs) and len(set(offs)) == len(offs)
    nn = max(n, 1)
    G = ng ** 3
    # int64 fixed-point accumulators: 4 per node for momentum and mass, 2 for the damage sums
    assert L.keys_b - L.keys_a >= 4 * nn and L.g_dmg - L.g_mom >= 32 * G and L.g_vel - L.g_dmg >= 16 * G
    assert L.payload - L.g_gd >= 4 * G and L.inv_perm - L.payload >= 80 * nn and L.work - L.inv_perm >= 4 * nn
    assert L.total - L.work >= 4 * nn
    assert _lib.bin_workspace_size(n, ng) == L.block_mask
    key_bits = max(max(_bits(ng ** 3), 1), _bits(((ng + 7) // 8) ** 3) + 9)
    assert L.sort_passes == _radix_passes(key_bits)
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


def _bits(v):
    b = 0
    while (1 << b) < v:
        b += 1
    return b


def _radix_passes(key_bits):
    """LSD passes of the sort: 8-bit digits, the last one 9 bits wide when
    exactly 9 bits remain."""
    p, rem = 0, max(key_bits, 1)
    while rem > 0:
        rem -= 9 if rem == 9 else 8
        p += 1
    return p


@pytest.mark.parametrize("ns,gs", [([1000, 0, 5000, 70000], [32, 64, 48, 128]), ([1], [4]),
                                   ([4096] * 64, [32 + 16 * (k % 7) for k in range(64)])])
def test_batch_layout_packs_scenes(ns, gs):
    L = _lib.batch_workspace_layout(ns, gs)
    assert L.n_total == sum(ns)
    assert L.n_nodes == sum(g ** 3 for g in gs)
    assert L.n_grid_blocks == sum(((g + 3) // 4) ** 3 for g in gs)
    assert L.n_sort_blocks == sum(((g + 7) // 8) ** 3 for g in gs)
    assert L.n_g2p_ctas == sum((n + 255) // 256 for n in ns)
    assert L.ws.sort_passes == _radix_passes(_bits(L.n_sort_blocks) + 9)
    w = L.ws
    offs = [w.ctrl, w.keys_a, w.keys_b, w.vals_a, w.vals_b, w.hist, w.block_mask, w.block_list, w.g_mom, w.g_dmg,
            w.g_vel, w.g_gd, w.payload, w.inv_perm, w.work, L.params, L.tables, w.total]
    assert all(o % 256 == 0 for o in offs)
    assert offs == sorted(offs) and len(set(offs)) == len(offs)
    assert w.keys_a - w.ctrl >= 224 * len(ns)                      # one control block per scene
    assert w.g_dmg - w.g_mom >= 32 * L.n_nodes and w.block_list - w.block_mask >= L.n_grid_blocks
    assert L.tables - L.params >= C.sizeof(_lib.pm_params) * len(ns)
    assert w.total - L.tables >= 5 * 8 * (len(ns) + 1)
    assert _lib.batch_workspace_size(ns, gs) == w.total


def test_batch_argument_errors_without_device():
    lib = _lib.load()
    out = C.c_size_t(0)
    n1, g1 = (C.c_int64 * 1)(10), (C.c_int32 * 1)(32)
    assert lib.pm_batch_workspace_size(0, n1, g1, C.byref(out)) == _lib.PM_ERR_ARG
    assert lib.pm_batch_workspace_size(_lib.PM_MAX_BATCH_SCENES + 1, n1, g1, C.byref(out)) == _lib.PM_ERR_ARG
    assert lib.pm_batch_workspace_size(1, (C.c_int64 * 1)(-1), g1, C.byref(out)) == _lib.PM_ERR_ARG
    assert lib.pm_batch_workspace_size(1, n1, (C.c_int32 * 1)(2), C.byref(out)) == _lib.PM_ERR_ARG
    assert lib.pm_batch_workspace_size(2, (C.c_int64 * 2)(1 << 30, 1 << 30), (C.c_int32 * 2)(32, 32),
                                       C.byref(out)) == _lib.PM_ERR_ARG
    assert lib.pm_batch_workspace_size(1, None, g1, C.byref(out)) == _lib.PM_ERR_ARG
    assert lib.pm_batch_workspace_size(1, n1, g1, C.byref(out)) == _lib.PM_OK and out.value > 0


def test_tape_size_grows_by_the_pre_collider_grid_per_slot():
    """With PM_TAPE_COLLIDERS every slot also keeps the grid velocity before
    the colliders (16 bytes per node); unknown flag bits are rejected."""
    lib = _lib.load()
    src = open(os.path.join(ROOT, "include", "peelmpm.h")).read()
    assert re.search(r"#define PM_TAPE_COLLIDERS 1\b", src) and _lib.PM_TAPE_COLLIDERS == 1
    n, ng = 100_000, 64
    for slots in (1, 3):
        plain = _lib.tape_size(n, ng, slots, 0)
        col = _lib.tape_size(n, ng, slots, _lib.PM_TAPE_COLLIDERS)
        assert col - plain == slots * 16 * ng ** 3
    out = C.c_size_t(0)
    assert lib.pm_tape_size(n, ng, 1, 2, C.byref(out)) == _lib.PM_ERR_ARG


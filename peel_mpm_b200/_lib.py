"""ctypes binding of the C ABI in include/peelmpm.h (libpeelmpm.so).

The structures mirror the header field for field; ``check_layout`` compares
their sizes with the library's own ``sizeof``.  Loading needs no GPU; every
compute entry point does.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libpeelmpm.so")

PM_MAX_GRIPS = 32
PM_MAX_COLLIDERS = 8
PM_OK, PM_ERR_ARG, PM_ERR_CUDA, PM_ERR_WORKSPACE, PM_ERR_UNSUPPORTED = 0, 1, 2, 3, 4

EXPORTS = (
    "pm_abi_version", "pm_last_error", "pm_struct_size", "pm_prepare", "pm_workspace_size", "pm_workspace_init",
    "pm_workspace_layout", "pm_grid_sums", "pm_substep", "pm_substep_dev_clock", "pm_set_clock", "pm_bin", "pm_p2g",
    "pm_grid_update", "pm_g2p", "pm_read_status", "pm_sym_eig", "pm_bin_workspace_size", "pm_bin_sort",
    "pm_bin_sort_static",
    "pm_batch_workspace_size", "pm_batch_workspace_layout", "pm_batch_workspace_init", "pm_batch_set_params",
    "pm_batch_workspace_release", "pm_batch_substep", "pm_batch_read_status",
    "pm_tape_size", "pm_tape_init", "pm_substep_record", "pm_substep_adjoint", "pm_observe",
    "pm_render_workspace_size", "pm_render_gaussians", "pm_carry_gaussians",
)
PM_OBS_MAX_GROUPS, PM_OBS_VALUES = 8, 8
PM_MAX_BATCH_SCENES = 4096
PM_BIN_STATIC_MAX_N = 262144


class pm_grip(C.Structure):
    _fields_ = [("vel", C.c_double * 3), ("ramp", C.c_double)]


class pm_collider(C.Structure):
    _fields_ = [("kind", C.c_int32), ("mode", C.c_int32), ("friction", C.c_double), ("radius", C.c_double),
                ("normal", C.c_double * 3)]


class pm_params(C.Structure):
    _fields_ = [
        ("n_grid", C.c_int32), ("damage_every", C.c_int32),
        ("grid_lim", C.c_double), ("dx", C.c_double), ("inv_dx", C.c_double), ("dt", C.c_double),
        ("gravity", C.c_double * 3), ("grid_damp", C.c_double),
        ("use_f_clamp", C.c_int32), ("record_stress", C.c_int32),
        ("f_clamp_lo", C.c_double), ("f_clamp_hi", C.c_double),
        ("n_grips", C.c_int32), ("n_colliders", C.c_int32), ("p2g_ctas_per_sm", C.c_int32),
        ("grid_ctas_per_sm", C.c_int32), ("stress_ctas_per_sm", C.c_int32), ("g2p_ctas_per_sm", C.c_int32),
        ("grips", pm_grip * PM_MAX_GRIPS), ("colliders", pm_collider * PM_MAX_COLLIDERS),
    ]


class pm_clock(C.Structure):
    _fields_ = [("time", C.c_double), ("step", C.c_int64),
                ("col_origin", (C.c_double * 3) * PM_MAX_COLLIDERS),
                ("col_origin_next", (C.c_double * 3) * PM_MAX_COLLIDERS)]


PARTICLE_FIELDS = ("x", "v", "F", "C", "d", "lap", "D_hist", "vol0", "mass", "mu", "lam", "sigma_c", "eta",
                   "zeta", "l0", "residual", "A0", "allow", "n_interface", "interface_mask", "grip_tag", "phi",
                   "phi_shear", "tau_last", "J_last")


class pm_particles(C.Structure):
    _fields_ = [("n", C.c_int64), ("plane_stride", C.c_int64)] + [(f, C.c_void_p) for f in PARTICLE_FIELDS]


class pm_status_info(C.Structure):
    _fields_ = [("nonfinite", C.c_uint32), ("dense_subblocks", C.c_uint32), ("n_active_blocks", C.c_uint32),
                ("any_allow", C.c_int32)]


class pm_ws_layout(C.Structure):
    _fields_ = [(f, C.c_size_t) for f in ("ctrl", "keys_a", "keys_b", "vals_a", "vals_b", "hist", "block_mask",
                                          "block_list", "g_mom", "g_dmg", "g_vel", "g_gd", "payload", "inv_perm",
                                          "work", "total")] + \
               [("sort_passes", C.c_int32), ("n_tiles", C.c_int32)]


class pm_batch_layout(C.Structure):
    _fields_ = [("ws", pm_ws_layout), ("params", C.c_size_t), ("tables", C.c_size_t)] + \
               [(f, C.c_int64) for f in ("n_total", "n_nodes", "n_grid_blocks", "n_sort_blocks", "n_g2p_ctas")]


class pm_state_adj(C.Structure):
    _fields_ = [("plane_stride", C.c_int64)] + [(f, C.c_void_p) for f in ("x", "v", "F", "C", "d", "lap", "D_hist")]


class pm_param_adj(C.Structure):
    _fields_ = [("plane_stride", C.c_int64)] + [(f, C.c_void_p) for f in ("mu", "lam", "sigma_c", "A0")]


class pm_camera(C.Structure):
    _fields_ = [("R", C.c_float * 9), ("T", C.c_float * 3), ("fx", C.c_float), ("fy", C.c_float),
                ("width", C.c_int32), ("height", C.c_int32)]


class pm_render_params(C.Structure):
    _fields_ = [("bg", C.c_float * 3), ("scale_modifier", C.c_float), ("r_max", C.c_int32), ("tau", C.c_float),
                ("near", C.c_float), ("max_raw_radius", C.c_float)]


STRUCTS = (pm_params, pm_particles, pm_clock, pm_status_info, pm_ws_layout, pm_grip, pm_collider, pm_batch_layout,
           pm_state_adj, pm_param_adj, pm_camera, pm_render_params)

_lib = None


class PeelMPMError(RuntimeError):
    pass


def load():
    """Load libpeelmpm.so (built by ``python -m peel_mpm_b200.build``)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with `python -m peel_mpm_b200.build` "
                          "(there is no fallback path)")
    lib = C.CDLL(LIB_PATH)
    vp, i32, i64, sz = C.c_void_p, C.c_int32, C.c_int64, C.c_size_t
    sig = {
        "pm_abi_version": (C.c_int, []),
        "pm_last_error": (C.c_char_p, []),
        "pm_struct_size": (sz, [i32]),
        "pm_prepare": (C.c_int, []),
        "pm_workspace_size": (C.c_int, [i64, i32, C.POINTER(sz)]),
        "pm_workspace_init": (C.c_int, [vp, sz, i64, i32, vp]),
        "pm_workspace_layout": (C.c_int, [i64, i32, C.POINTER(pm_ws_layout)]),
        "pm_grid_sums": (C.c_int, [vp, sz, i64, i32, vp, vp, vp]),
        "pm_substep": (C.c_int, [C.POINTER(pm_params), C.POINTER(pm_particles), vp, sz, C.POINTER(pm_clock), vp]),
        "pm_substep_dev_clock": (C.c_int, [C.POINTER(pm_params), C.POINTER(pm_particles), vp, sz, vp, i32, vp]),
        "pm_set_clock": (C.c_int, [C.POINTER(pm_params), vp, sz, i64, C.POINTER(pm_clock), vp]),
        "pm_bin": (C.c_int, [C.POINTER(pm_params), C.POINTER(pm_particles), vp, sz, vp]),
        "pm_p2g": (C.c_int, [C.POINTER(pm_params), C.POINTER(pm_particles), vp, sz, vp]),
        "pm_grid_update": (C.c_int, [C.POINTER(pm_params), vp, sz, i64, vp]),
        "pm_g2p": (C.c_int, [C.POINTER(pm_params), C.POINTER(pm_particles), vp, sz, vp]),
        "pm_read_status": (C.c_int, [vp, sz, i64, i32, C.POINTER(pm_status_info), vp]),
        "pm_sym_eig": (C.c_int, [vp, i64, i32, vp, vp, vp]),
        "pm_bin_workspace_size": (C.c_int, [i64, i32, C.POINTER(sz)]),
        "pm_bin_sort": (C.c_int, [vp, i64, i64, i32, C.c_double, vp, vp, vp, sz, vp]),
        "pm_bin_sort_static": (C.c_int, [vp, i64, i64, i32, C.c_double, vp, vp, vp]),
        "pm_batch_workspace_size": (C.c_int, [i32, vp, vp, C.POINTER(sz)]),
        "pm_batch_workspace_layout": (C.c_int, [i32, vp, vp, C.POINTER(pm_batch_layout)]),
        "pm_batch_workspace_init": (C.c_int, [vp, sz, i32, vp, C.POINTER(pm_params), vp]),
        "pm_batch_set_params": (C.c_int, [vp, sz, i32, vp, C.POINTER(pm_params), vp]),
        "pm_batch_workspace_release": (C.c_int, [vp]),
        "pm_batch_substep": (C.c_int, [i32, vp, vp, C.POINTER(pm_particles), vp, sz, vp, vp]),
        "pm_batch_read_status": (C.c_int, [vp, sz, i32, vp, vp, C.POINTER(pm_status_info), vp]),
        "pm_tape_size": (C.c_int, [i64, i32, i32, i32, C.POINTER(sz)]),
        "pm_tape_init": (C.c_int, [vp, sz, i64, i32, i32, i32, vp]),
        "pm_substep_record": (C.c_int, [C.POINTER(pm_params), C.POINTER(pm_particles), C.POINTER(pm_particles), vp,
                                        sz, C.POINTER(pm_clock), vp, sz, i32, i32, vp]),
        "pm_render_workspace_size": (C.c_int, [i64, i32, i32, i32, C.POINTER(sz)]),
        "pm_carry_gaussians": (C.c_int, [C.POINTER(pm_particles), vp, vp, vp, vp, i64, vp, C.c_float, vp, vp, vp,
                                         vp]),
        "pm_render_gaussians": (C.c_int, [C.POINTER(pm_camera), C.POINTER(pm_render_params), vp, vp, vp, i64, vp, vp,
                                          sz, vp]),
        "pm_observe": (C.c_int, [C.POINTER(pm_particles), vp, i32, C.c_float, vp, vp, vp, vp, i32, C.c_float, i32,
                                 vp, vp, i64, vp]),
        "pm_substep_adjoint": (C.c_int, [C.POINTER(pm_params), C.POINTER(pm_particles), C.POINTER(pm_particles),
                                         C.POINTER(pm_state_adj), C.POINTER(pm_state_adj), C.POINTER(pm_param_adj),
                                         vp, sz, i32, i32, vp]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if lib.pm_abi_version() != 2:
        raise ImportError("libpeelmpm.so ABI version mismatch; rebuild it")
    _lib = lib
    return lib


def check(rc: int, what: str = "peelmpm"):
    """Raise PeelMPMError for a non-zero status, with pm_last_error()."""
    if rc != PM_OK:
        msg = _lib.pm_last_error().decode() if _lib is not None else ""
        raise PeelMPMError(f"{what} failed with status {rc}: {msg}")


def check_layout():
    """Sizes of the ctypes structures versus the library's sizeof (no GPU)."""
    lib = load()
    return {s.__name__: (C.sizeof(s), int(lib.pm_struct_size(i))) for i, s in enumerate(STRUCTS)}


def workspace_size(n: int, n_grid: int) -> int:
    lib = load()
    out = C.c_size_t(0)
    check(lib.pm_workspace_size(int(n), int(n_grid), C.byref(out)), "pm_workspace_size")
    return int(out.value)


def bin_workspace_size(n: int, n_grid: int) -> int:
    lib = load()
    out = C.c_size_t(0)
    check(lib.pm_bin_workspace_size(int(n), int(n_grid), C.byref(out)), "pm_bin_workspace_size")
    return int(out.value)


def workspace_layout(n: int, n_grid: int) -> pm_ws_layout:
    lib = load()
    lay = pm_ws_layout()
    check(lib.pm_workspace_layout(int(n), int(n_grid), C.byref(lay)), "pm_workspace_layout")
    return lay


def _scene_arrays(ns, grids):
    S = len(ns)
    if S != len(grids):
        raise ValueError("one n_grid per scene")
    n_arr = (C.c_int64 * S)(*[int(v) for v in ns])
    g_arr = (C.c_int32 * S)(*[int(v) for v in grids])
    return S, n_arr, g_arr


def batch_workspace_size(ns, grids) -> int:
    lib = load()
    S, n_arr, g_arr = _scene_arrays(ns, grids)
    out = C.c_size_t(0)
    check(lib.pm_batch_workspace_size(S, n_arr, g_arr, C.byref(out)), "pm_batch_workspace_size")
    return int(out.value)


def batch_workspace_layout(ns, grids) -> pm_batch_layout:
    lib = load()
    S, n_arr, g_arr = _scene_arrays(ns, grids)
    lay = pm_batch_layout()
    check(lib.pm_batch_workspace_layout(S, n_arr, g_arr, C.byref(lay)), "pm_batch_workspace_layout")
    return lay


PM_TAPE_COLLIDERS = 1


def tape_size(n: int, n_grid: int, slots: int, flags: int = 0) -> int:
    lib = load()
    out = C.c_size_t(0)
    check(lib.pm_tape_size(int(n), int(n_grid), int(slots), int(flags), C.byref(out)), "pm_tape_size")
    return int(out.value)

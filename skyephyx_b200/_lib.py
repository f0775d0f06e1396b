"""Loads the in-tree CUDA library ``libavbd.so`` and declares its C-ABI.

There is no CPU fallback: if the library is missing or no CUDA device is
present, loading or creating a world fails with an exception.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
# AVBD_CHECKS=1 selects the debug build with device index checks
LIB_PATH = os.path.join(HERE, "libavbd_checks.so" if os.environ.get("AVBD_CHECKS") == "1" else "libavbd.so")

STATUS = {0: "ok", 1: "exploded", 2: "nan", 3: "capacity", 4: "timeout"}


class AvbdError(RuntimeError):
    pass


class AvbdParams(C.Structure):
    """AvbdParams (include/avbd.h); same names/defaults as solver.hpp:69-84."""
    _fields_ = [
        ("num_iterations", C.c_int32),
        ("step_value", C.c_float),
        ("alpha", C.c_float),
        ("beta", C.c_float),
        ("gamma", C.c_float),
        ("on_penetration_penalty", C.c_float),
        ("post_stabilization", C.c_int32),
        ("projection_mode", C.c_int32),
        ("trust_region_rho", C.c_float),
    ]


class AvbdServedRequest(C.Structure):
    """AvbdServedRequest (include/avbd.h): one finished served request."""
    _fields_ = [("request", C.c_int32), ("status", C.c_int32), ("steps", C.c_int32), ("bodies", C.c_int32),
                ("arrival_s", C.c_double), ("admitted_s", C.c_double), ("finished_s", C.c_double)]


class AvbdServerStats(C.Structure):
    _fields_ = [(n, C.c_int64) for n in ("submitted", "admitted", "completed", "ticks", "body_iterations",
                                         "uploaded_bytes", "pending", "active", "resident_dynamic",
                                         "device_us", "wait_us", "regrown", "catchup_us", "stage_us",
                                         "retire_us", "issue_us")]


class AvbdTimings(C.Structure):
    _fields_ = [(n, C.c_float) for n in ("broad_phase_ms", "warmstart_ms", "colouring_ms", "prediction_ms",
                                         "primal_dual_ms", "velocity_update_ms", "post_stab_ms",
                                         "total_substep_ms")]


_lib = None

# (name, argtypes, restype) of every exported entry point
_F = C.POINTER(C.c_float)
_I = C.POINTER(C.c_int32)
_U = C.POINTER(C.c_uint32)
_V = C.c_void_p
SIGNATURES = [
    ("avbd_default_params", [C.POINTER(AvbdParams)], None),
    ("avbd_status_string", [C.c_int32], C.c_char_p),
    ("avbd_world_create", [C.POINTER(AvbdParams), C.c_int32, C.POINTER(_V)], C.c_int32),
    ("avbd_world_destroy", [_V], C.c_int32),
    ("avbd_world_clear", [_V], C.c_int32),
    ("avbd_set_params", [_V, C.POINTER(AvbdParams)], C.c_int32),
    ("avbd_get_params", [_V, C.POINTER(AvbdParams)], C.c_int32),
    ("avbd_add_body", [_V, C.c_int32, C.c_float, C.c_float, _F, _F, _F, _F, _F, C.c_int32], C.c_int32),
    ("avbd_add_bodies", [_V, C.c_int32, C.c_int32, _F, _F, _F, _F, _F, _F, _F, _I], C.c_int32),
    ("avbd_add_particle", [_V, C.c_float, C.c_float, _F, _F, C.c_int32], C.c_int32),
    ("avbd_set_body_static", [_V, C.c_int32, C.c_int32], C.c_int32),
    ("avbd_add_spring", [_V, C.c_int32, _F, C.c_int32, _F, C.c_float, C.c_float, C.c_int32, C.c_float], C.c_int32),
    ("avbd_add_joint", [_V, C.c_int32, _F, C.c_int32, _F, _F, _F], C.c_int32),
    ("avbd_add_neohookean_tet", [_V, _I, C.c_float, C.c_float], C.c_int32),
    ("avbd_add_stvk_tri", [_V, _I, C.c_float, C.c_float], C.c_int32),
    ("avbd_make_tet_volume", [_V, C.c_float, C.c_float, C.c_float, C.c_int32, C.c_int32, C.c_int32, C.c_float,
                              C.c_float, C.c_float, C.c_float, C.c_float, C.c_int32], C.c_int32),
    ("avbd_make_stvk_tet_volume", [_V, C.c_float, C.c_float, C.c_float, C.c_int32, C.c_int32, C.c_int32, C.c_float,
                              C.c_float, C.c_float, C.c_float, C.c_float, C.c_int32], C.c_int32),
    ("avbd_add_stvk_tet", [_V, _I, C.c_float, C.c_float], C.c_int32),
    ("avbd_set_body_color", [_V, C.c_int32, _F], C.c_int32),
    ("avbd_export_instances", [_V, _V, C.c_int32, _I, _I], C.c_int32),
    ("avbd_batch_export_instances", [_V, C.c_int32, _V, C.c_int32, _I, _I], C.c_int32),
    ("avbd_batch_scene_snapshot_bytes", [_V, C.c_int32], C.c_int64),
    ("avbd_batch_scene_snapshot", [_V, C.c_int32, _V, C.c_int64], C.c_int32),
    ("avbd_batch_scene_restore", [_V, _V, C.c_int64], C.c_int32),
    ("avbd_make_tet_sphere", [_V, C.c_float, C.c_float, C.c_float, C.c_float, C.c_float, C.c_float, C.c_float,
                              C.c_float, C.c_float], C.c_int32),
    ("avbd_remove_body", [_V, C.c_int32], C.c_int32),
    ("avbd_remove_force", [_V, C.c_int32], C.c_int32),
    ("avbd_remove_neohookean_tet", [_V, C.c_int32], C.c_int32),
    ("avbd_remove_stvk_tri", [_V, C.c_int32], C.c_int32),
    ("avbd_snapshot_bytes", [_V], C.c_int64),
    ("avbd_snapshot", [_V, _V, C.c_int64], C.c_int32),
    ("avbd_restore", [_V, _V, C.c_int64], C.c_int32),
    ("avbd_step", [_V], C.c_int32),
    ("avbd_step_dt", [_V, C.c_float, C.c_int32], C.c_int32),
    ("avbd_num_bodies", [_V], C.c_int32),
    ("avbd_num_dynamic_bodies", [_V], C.c_int32),
    ("avbd_emergency_stop", [_V], C.c_int32),
    ("avbd_force_live", [_V, C.c_int32], C.c_int32),
    ("avbd_get_state", [_V, _F, _F, _F, _F], C.c_int32),
    ("avbd_set_state", [_V, _F, _F, _F, _F], C.c_int32),
    ("avbd_get_contacts", [_V, C.c_int32, _I, _I, _U, _F], C.c_int32),
    ("avbd_get_colours", [_V, _I], C.c_int32),
    ("avbd_get_timings", [_V, C.POINTER(AvbdTimings)], C.c_int32),
    ("avbd_collide", [_V, C.c_int32, C.c_int32, _U, _F], C.c_int32),
    ("avbd_collide_noalloc", [_V, C.c_int32, _I, _I, _U, _F, _I], C.c_int32),
    ("avbd_batch_create", [C.POINTER(AvbdParams), C.c_int32, C.POINTER(_V)], C.c_int32),
    ("avbd_batch_destroy", [_V], C.c_int32),
    ("avbd_batch_add_scene", [_V, _V], C.c_int32),
    ("avbd_batch_reserve", [_V, C.c_int64, C.c_int64, C.c_int64, C.c_int64, C.c_int32], C.c_int32),
    ("avbd_batch_scene_body_offset", [_V, C.c_int32], C.c_int32),
    ("avbd_batch_remove_scene", [_V, C.c_int32], C.c_int32),
    ("avbd_batch_prepare", [_V], C.c_int32),
    ("avbd_batch_uploaded_bytes", [_V], C.c_int64),
    ("avbd_host_alloc_pinned", [C.c_int32, C.c_int64, C.POINTER(C.c_void_p)], C.c_int32),
    ("avbd_host_free_pinned", [_V], C.c_int32),
    ("avbd_batch_step", [_V, C.c_int32], C.c_int32),
    ("avbd_batch_num_scenes", [_V], C.c_int32),
    ("avbd_batch_scene_status", [_V, C.c_int32], C.c_int32),
    ("avbd_batch_scene_bodies", [_V, C.c_int32], C.c_int32),
    ("avbd_batch_scene_info", [_V, C.c_int32, _I], C.c_int32),
    ("avbd_batch_dynamic_bodies", [_V], C.c_int64),
    ("avbd_batch_get_state", [_V, C.c_int32, _F, _F, _F, _F], C.c_int32),
    ("avbd_batch_get_all_poses", [_V, _F, _F, C.c_int64], C.c_int32),
    ("avbd_scene_footprint_bytes", [_V], C.c_int64),
    ("avbd_batch_set_launch", [_V, C.c_int32, C.c_int32], C.c_int32),
    ("avbd_batch_get_launch", [_V, _I, _I], C.c_int32),
    ("avbd_batch_set_kernel", [_V, C.c_int32], C.c_int32),
    ("avbd_batch_set_team_work", [_V, C.c_int32], C.c_int32),
    ("avbd_batch_set_fem_team_work", [_V, C.c_int32], C.c_int32),
    ("avbd_batch_set_grid_broadphase", [_V, C.c_int32], C.c_int32),
    ("avbd_batch_set_cluster", [_V, C.c_int32, C.c_int32], C.c_int32),
    ("avbd_batch_set_scene_timing", [_V, C.c_int32], C.c_int32),
    ("avbd_batch_set_queue_weight", [_V, C.c_int32], C.c_int32),
    ("avbd_batch_read_poses", [_V, _F, _F, C.c_int64], C.c_int32),
    ("avbd_batch_read_poses_wait", [_V], C.c_int32),
    ("avbd_check_word", [_V, C.POINTER(C.c_int32)], C.c_int32),
    ("avbd_batch_check_word", [_V, C.POINTER(C.c_int32)], C.c_int32),
    ("avbd_batch_scene_times", [_V, C.POINTER(C.c_int64), C.c_int32], C.c_int32),
    ("avbd_batch_last_ms", [_V], C.c_float),
    ("avbd_batch_set_groups", [_V, C.c_int32, C.c_int32], C.c_int32),
    ("avbd_set_group", [_V, C.c_int32], C.c_int32),
    ("avbd_server_create", [C.POINTER(AvbdParams), C.c_int32, C.c_int64, C.c_int32, C.POINTER(_V)], C.c_int32),
    ("avbd_server_destroy", [_V], C.c_int32),
    ("avbd_server_batch", [_V], _V),
    ("avbd_server_submit", [_V, _V, C.c_int32, C.c_double, C.c_int32], C.c_int32),
    ("avbd_server_tick", [_V, C.c_double], C.c_int32),
    ("avbd_server_drain", [_V, C.c_double], C.c_int32),
    ("avbd_server_poll", [_V, C.POINTER(AvbdServedRequest)], C.c_int32),
    ("avbd_server_result", [_V, C.c_int32, _F, _F, _F, _F], C.c_int32),
    ("avbd_server_release", [_V, C.c_int32], C.c_int32),
    ("avbd_server_stats", [_V, C.POINTER(AvbdServerStats)], C.c_int32),
]


def load(path: str = LIB_PATH):
    """Returns the loaded library (building it first if it is absent)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        from . import build as _build
        _build.build(checks=path.endswith("libavbd_checks.so"))
    if not os.path.exists(path):
        raise AvbdError(f"CUDA library not found at {path}; build it with `python -m skyephyx_b200.build`")
    lib = C.CDLL(path)
    for name, args, res in SIGNATURES:
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = res
    _lib = lib
    return lib


def check(code: int, what: str = "") -> int:
    if code < 0:
        msg = load().avbd_status_string(code).decode()
        raise AvbdError(f"{what}: {msg} ({code})")
    return code


def default_params(**overrides) -> AvbdParams:
    p = AvbdParams()
    load().avbd_default_params(C.byref(p))
    for k, v in overrides.items():
        setattr(p, k, v)
    return p

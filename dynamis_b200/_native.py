"""ctypes binding of libdynamis_cuda.so (the C ABI declared in include/dynamis_cuda.h).

The library is built in-tree by dynamis_b200.build. There is no fallback: if the library is
missing or fails to load, importing this module raises.
"""
from __future__ import annotations

import ctypes
from pathlib import Path

LIBRARY = Path(__file__).resolve().parent / "libdynamis_cuda.so"

P = ctypes.c_void_p
U32 = ctypes.c_uint32
I32 = ctypes.c_int32
F32 = ctypes.c_float
PU32 = ctypes.POINTER(ctypes.c_uint32)
PF32 = ctypes.POINTER(ctypes.c_float)

# name -> (restype, argtypes); every symbol include/dynamis_cuda.h declares
SIGNATURES = {
    "dyn_abi_version": (U32, []),
    "dyn_status_string": (ctypes.c_char_p, [I32]),
    "dyn_config_default": (None, [P]),
    "dyn_collider_desc_default": (None, [P]),
    "dyn_body_desc_default": (None, [P]),
    "dyn_world_create": (I32, [P, P, I32, ctypes.POINTER(P)]),
    "dyn_world_destroy": (I32, [P]),
    "dyn_last_error": (ctypes.c_char_p, [P]),
    "dyn_world_set_stream": (I32, [P, P]),
    "dyn_add_hull": (I32, [P, P, U32, PU32]),
    "dyn_add_hull_from_mesh": (I32, [P, P, U32, P, U32, PU32]),
    "dyn_add_hull_mesh": (I32, [P, P, U32, P, U32, PU32]),
    "dyn_hull_info": (I32, [P, U32, PU32, PU32, PF32, P]),
    "dyn_spawn_bodies": (I32, [P, P, U32, P, U32, P]),
    "dyn_upload_bodies": (I32, [P, P, P, U32, P, P, U32]),
    "dyn_upload_states": (I32, [P, P, U32]),
    "dyn_stream_capacity": (I32, [P, PU32, PU32]),
    "dyn_scene_sizes": (I32, [P, PU32, PU32, PU32, PU32, PU32]),
    "dyn_export_scene": (I32, [P, P, P, P, P, P, P]),
    "dyn_step_params_for": (I32, [P, F32, P]),
    "dyn_step": (I32, [P, F32]),
    "dyn_sync": (I32, [P]),
    "dyn_device_status": (I32, [P, PU32]),
    "dyn_download_states": (I32, [P, P, U32]),
    "dyn_read_state": (I32, [P, U32, P]),
    "dyn_read_counters": (I32, [P, P, U32]),
    "dyn_debug_aabbs": (I32, [P, P, U32, PU32]),
    "dyn_debug_entries": (I32, [P, P, P, U32, PU32]),
    "dyn_debug_pairs": (I32, [P, P, P, U32, PU32]),
    "dyn_debug_contacts": (I32, [P, P, U32, PU32]),
    "dyn_debug_islands": (I32, [P, P, U32, PU32]),
    "dyn_debug_resting": (I32, [P, P, U32, PU32]),
    "dyn_query": (I32, [P, P, U32, P, U32]),
    "dyn_hull_triangles": (I32, [P, U32, P, U32, PU32]),
    "dyn_set_timing": (I32, [P, I32]),
    "dyn_set_solver_guard": (I32, [P, U32]),
    "dyn_set_ccd": (I32, [P, U32, I32]),
    "dyn_set_launch_config": (I32, [P, P]),
    "dyn_get_launch_config": (I32, [P, P]),
    "dyn_autotune": (I32, [P, ctypes.c_float, U32, P, P]),
    "dyn_snapshot_take": (I32, [P, P]),
    "dyn_snapshot_restore": (I32, [P, P]),
    "dyn_snapshot_free": (I32, [P]),
    "dyn_step_kernel_count": (U32, [P]),
    "dyn_stage_count": (U32, []),
    "dyn_stage_name": (ctypes.c_char_p, [U32]),
    "dyn_stage_timings": (I32, [P, P, U32]),
    "dyn_radix_sort": (I32, [P, P, P, P, U32, U32, U32]),
    "dyn_radix_sort_static": (I32, [P, P, P, U32, U32, U32, P]),
    "dyn_radix_sort_static_status": (I32, [P, PU32]),
    "dyn_clear_device_status": (I32, [P]),
    "dyn_debug_sort_fault": (I32, [P, U32, U32]),
    "dyn_tape_begin": (I32, [P, U32]),
    "dyn_tape_end": (I32, [P]),
    "dyn_tape_steps": (I32, [P, PU32, PU32]),
    "dyn_step_backward": (I32, [P, P, P, U32]),
    "dyn_backward": (I32, [P, P, P, U32, U32]),
    "dyn_param_grads": (I32, [P, P, P, U32, P, U32]),
    "dyn_set_mass_properties": (I32, [P, P, P, U32]),
    "dyn_set_friction": (I32, [P, P, U32]),
    "dyn_set_body_worlds": (I32, [P, P, U32]),
    "dyn_edit_bodies": (I32, [P, P, P, U32]),
    "dyn_remove_bodies": (I32, [P, P, U32]),
    "dyn_observe_bodies": (I32, [P, P, U32]),
    "dyn_stop_observing": (I32, [P]),
    "dyn_poll": (I32, [P]),
    "dyn_try_state": (I32, [P, U32, P, P]),
    "dyn_try_counters": (I32, [P, P, U32, P]),
    "dyn_export_body_worlds": (I32, [P, P]),
    "dyn_add_ball_joint": (I32, [P, U32, U32, P, P, PU32]),
    "dyn_add_constraints": (I32, [P, P, U32, PU32]),
    "dyn_constraint_count": (I32, [P, PU32]),
    "dyn_read_constraints": (I32, [P, P, U32]),
    "dyn_export_constraints": (I32, [P, P, P, P]),
    "dyn_joint_plan": (I32, [P, P, P, P, PU32, PU32]),
}


class DynamisError(RuntimeError):
    """A C ABI call returned a non-zero dyn_status."""

    def __init__(self, status: int, message: str):
        super().__init__(f"dynamis status {status}: {message}")
        self.status = status


def _load() -> ctypes.CDLL:
    if not LIBRARY.exists():
        raise ImportError(
            f"{LIBRARY} is missing: build it with `python dynamis_b200/build.py` (nvcc, sm_100a); "
            "there is no CPU fallback")
    lib = ctypes.CDLL(str(LIBRARY))
    for name, (restype, argtypes) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = restype
        fn.argtypes = argtypes
    return lib


class _Library:
    """libdynamis_cuda.so, loaded at the first call through it (so that the scene descriptions and
    record dtypes import without it); a missing library raises ImportError there, with no fallback."""

    _cdll = None

    def __getattr__(self, name):
        if _Library._cdll is None:
            _Library._cdll = _load()
        return getattr(_Library._cdll, name)


lib = _Library()


def check(status: int, world=None) -> None:
    if status != 0:
        detail = lib.dyn_last_error(world).decode() if world else ""
        raise DynamisError(status, f"{lib.dyn_status_string(status).decode()}: {detail}")


def ptr(array) -> int | None:
    """Address of a numpy array's buffer (None for None)."""
    if array is None:
        return None
    return array.ctypes.data

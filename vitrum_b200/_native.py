"""ctypes binding of libvitrum_pt.so (the C ABI declared in include/vitrum_pt.h).

The library is required: importing a symbol from here raises if the shared
object is missing or fails to load.  There is no CPU fallback.
"""
from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libvitrum_pt.so")

VT_OK = 0
STATUS_NAMES = {
    0: "VT_OK", 1: "VT_ERR_INVALID_ARGUMENT", 2: "VT_ERR_RANGE", 3: "VT_ERR_CUDA", 4: "VT_ERR_OUT_OF_MEMORY",
    5: "VT_ERR_STATE", 6: "VT_ERR_BUILD", 7: "VT_ERR_TIMEOUT",
}


class VtError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


class BuildOptions(ctypes.Structure):
    _fields_ = [("position_stride", ctypes.c_int32), ("index_stride", ctypes.c_int32),
                ("max_leaf_triangles", ctypes.c_int32), ("bin_count", ctypes.c_int32),
                ("max_depth", ctypes.c_int32), ("traversal_tree", ctypes.c_int32)]


class BvhInfo(ctypes.Structure):
    _fields_ = [("triangle_count", ctypes.c_int64), ("binary_node_count", ctypes.c_int64),
                ("wide_node_count", ctypes.c_int64), ("wide_depth", ctypes.c_int32),
                ("binary_depth", ctypes.c_int32), ("build_ms", ctypes.c_double)]


class LightTreeEmitter(ctypes.Structure):
    _fields_ = [("power", ctypes.c_double), ("centroid", ctypes.c_double * 3), ("aabb_min", ctypes.c_double * 3),
                ("aabb_max", ctypes.c_double * 3), ("cone_axis", ctypes.c_double * 3), ("cone_theta_o", ctypes.c_double),
                ("cone_theta_e", ctypes.c_double), ("oriented", ctypes.c_int32)]


class BvhProof(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int64) for n in ("node_count", "root_count", "interior_node_count", "leaf_node_count",
                                               "max_depth", "max_traversal_stack_entries",
                                               "traversal_stack_capacity", "triangle_count")]


class WideProof(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int64) for n in ("node_count", "internal_slots", "leaf_slots", "triangle_count",
                                               "depth", "stack_entries")]


class WatertightResult(ctypes.Structure):
    _fields_ = [("hit", ctypes.c_int32), ("t", ctypes.c_float), ("bary", ctypes.c_float * 3),
                ("side", ctypes.c_int32), ("zero_edge_mask", ctypes.c_int32)]


_lib = None

P = ctypes.c_void_p
SZ = ctypes.c_size_t
I32 = ctypes.c_int32

# name -> argtypes; every entry returns vt_status unless listed in _RESTYPE
SIGNATURES = {
    "vt_last_error": [],
    "vt_version": [],
    "vt_bvh_build": [I32, P, SZ, P, SZ, P, P],
    "vt_bvh_build_device": [I32, P, SZ, P, SZ, P, P, P],
    "vt_bvh_get_info": [P, P],
    "vt_bvh_export_binary": [P, P, SZ, P, SZ],
    "vt_bvh_trace_closest_device": [P, P, SZ, P, P],
    "vt_bvh_trace_any_device": [P, P, SZ, P, P],
    "vt_bvh_trace_closest": [P, P, SZ, P],
    "vt_bvh_trace_any": [P, P, SZ, P],
    "vt_bvh_destroy": [P],
    "vt_bvh_set_trace_order": [P, I32],
    "vt_engine_autotune_bvh": [P, P, P, P, SZ, P],
    "vt_tlas_build": [P, SZ, I32, I32, I32, P, SZ, P, SZ, P],
    "vt_validate_bvh_encoding": [P, SZ, SZ, P, SZ, ctypes.c_int64, I32, P],
    "vt_light_tree_build": [P, SZ, P, SZ, P],
    "vt_light_tree_select_device": [P, SZ, ctypes.c_uint32, P, P, P, SZ, P, P, P],
    "vt_bvh_validate": [P, P],
    "vt_engine_export_tlas": [P, P, SZ, P, SZ, P],
    "vt_bvh_trace_closest_noalloc": [P, P, SZ, P],
    "vt_watertight_eval_device": [I32, P, SZ, P, P],
    "vt_create": [I32, P, P],
    "vt_set_scene": [P, P],
    "vt_render_frame": [P, P, P],
    "vt_profile_frame": [P, P, P, P],
    "vt_capture": [P, P, SZ],
    "vt_capture_output": [P, P, P, SZ],
    "vt_update_instances": [P, P, SZ, I32],
    "vt_update_mesh": [P, SZ, P, I32],
    "vt_get_capabilities": [P, P],
    "vt_bake_preetham_sky": [P, I32, I32, P, SZ],
    "vt_capture_moments": [P, P, P, SZ],
    "vt_engine_export_scene": [P, P, SZ, P, SZ, P, P],
    "vt_bvh_export_wide": [P, P, SZ, P, SZ, P, P],
    "vt_capture_luminance_moments": [P, P, SZ],
    "vt_capture_aux": [P, I32, P, SZ],
    "vt_set_previous_camera": [P, P, P],
    "vt_pick": [P, ctypes.c_float, ctypes.c_float, P],
    "vt_trace_rays": [P, P, SZ, P, P],
    "vt_set_nrc": [P, P],
    "vt_batch_create": [I32, P, P],
    "vt_batch_set_scenes": [P, P, P, SZ],
    "vt_batch_render": [P, P],
    "vt_batch_capture": [P, SZ, P, SZ],
    "vt_batch_set_tuning": [P, P],
    "vt_batch_get_tuning": [P, P],
    "vt_batch_autotune": [P, P, SZ, P],
    "vt_batch_destroy": [P],
    "vt_engine_autotune": [P, P, P, SZ, P],
    "vt_engine_get_tuning": [P, P],
    "vt_engine_set_tuning": [P, P],
    "vt_nrc_create": [I32, P, P],
    "vt_nrc_destroy": [P],
    "vt_nrc_query": [P, P, SZ, P],
    "vt_nrc_train": [P, P, SZ, P],
    "vt_nrc_gradients": [P, P, SZ, P, P, P],
    "vt_nrc_get_params": [P, P, P],
    "vt_nrc_set_params": [P, P, P],
    "vt_nrc_query_device": [P, P, SZ, P, P],
    "vt_nrc_train_device": [P, P, SZ, P],
    "vt_engine_set_wait_limit": [P, ctypes.c_int64],
    "vt_debug_fail_device_allocation": [ctypes.c_int64],
    "vt_reset": [P],
    "vt_engine_get_stats": [P, P],
    "vt_destroy": [P],
}
_RESTYPE = {"vt_last_error": ctypes.c_char_p, "vt_version": ctypes.c_char_p}


def lib():
    """Load libvitrum_pt.so (raises OSError when it is missing: no fallback)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise OSError(f"{LIB_PATH} is missing; build it with `python -m vitrum_b200.build`")
        L = ctypes.CDLL(LIB_PATH)
        for name, args in SIGNATURES.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = _RESTYPE.get(name, ctypes.c_int32)
        _lib = L
    return _lib


def check(status: int) -> None:
    if status != VT_OK:
        raise VtError(status, lib().vt_last_error().decode())


def call(name: str, *args) -> None:
    check(getattr(lib(), name)(*args))

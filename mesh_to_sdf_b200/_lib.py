"""ctypes binding of libm2s.so (the C ABI of include/m2s.h)."""
from __future__ import annotations

import ctypes
import os
import threading

_HERE = os.path.dirname(os.path.abspath(__file__))
# M2S_BUILD=fast selects the fast build (fused multiply-adds in the distance
# arithmetic; distances within 4 ulp or 1e-6 of the bbox diagonal of the
# strict build, same Raycast signs).  The default is the strict build.
FAST = os.environ.get("M2S_BUILD", "strict") == "fast"
LIB_PATH = os.path.join(_HERE, "libm2s_fast.so" if FAST else "libm2s.so")
_lock = threading.Lock()
_lib = None

P = ctypes.c_void_p
U64 = ctypes.c_uint64
I = ctypes.c_int

# name -> (restype, argtypes); every function declared in include/m2s.h
SIGNATURES = {
    "m2s_generate_sdf": (I, [P, U64, P, U64, I, I, P, U64, I, I, P, P, P]),
    "m2s_generate_grid_sdf": (I, [P, U64, P, U64, I, I, P, P, P, I, P, P, P]),
    "m2s_build_sdf_acceleration": (I, [P, U64, P, U64, I, I, I, I, P, P]),
    "m2s_query_sdf": (I, [P, P, U64, P, P, P]),
    "m2s_query_vector_to_closest_point": (I, [P, P, U64, P, P, P, P]),
    "m2s_mesh_free": (None, [P]),
    "m2s_mesh_triangle_count": (U64, [P]),
    "m2s_mesh_accel": (I, [P]),
    "m2s_query_sdf_device": (I, [P, P, U64, P, P, P]),
    "m2s_grid_sdf_device": (I, [P, P, P, P, I, P, P, P]),
    "m2s_grid_sdf_batch_device": (I, [P, ctypes.c_uint32, P, P, P, I, P, P, P]),
    "m2s_grid_plan_create": (I, [P, ctypes.c_uint32, P, P, P, I, P, P, P, P]),
    "m2s_grid_plan_run": (I, [P, P]),
    "m2s_grid_plan_autotune": (I, [P, P, P]),
    "m2s_grid_plan_cells": (U64, [P]),
    "m2s_grid_plan_device_bytes": (U64, [P]),
    "m2s_grid_plan_blocks": (ctypes.c_uint32, [P]),
    "m2s_grid_plan_free": (None, [P]),
    "m2s_clear_grid_autotune": (None, []),
    "m2s_set_grid_tuning": (None, [I, ctypes.c_uint32, U64, I]),
    "m2s_set_grid_bound_filter": (None, [I]),
    "m2s_last_grid_filter_stats": (I, [P]),
    "m2s_pool_usage": (I, [P]),
    "m2s_set_fp64_audit": (None, [I]),
    "m2s_last_grid_audit": (I, [P]),
    "m2s_last_query_audit": (I, [P]),
    "m2s_grid_plan_waves": (ctypes.c_uint32, [P]),
    "m2s_radix_sort_pairs_device": (I, [P, P, U64, I, P]),
    "m2s_sort_cells_by_distance_device": (I, [P, U64, P, P, P]),
    "m2s_sort_cells_by_distance": (I, [P, U64, P, P, P]),
    "m2s_serialize_generic": (I, [P, U64, P, U64, P, U64, P]),
    "m2s_serialize_grid": (I, [P, P, P, P, U64, P, U64, P]),
    "m2s_deserialize": (I, [P, U64, P, P, P, P, P, P, P, P]),
    "m2s_check_mesh_triangle_list": (I, [P, U64, P, U64, P, P, P]),
    "m2s_server_create": (I, [U64, ctypes.c_uint32, P]),
    "m2s_server_free": (None, [P]),
    "m2s_server_submit_upload": (I, [P, P, U64, P, U64, I, I, I, I, P, P]),
    "m2s_server_submit_points": (I, [P, ctypes.c_uint32, P, U64, P, P]),
    "m2s_server_submit_grid": (I, [P, ctypes.c_uint32, P, P, P, I, P, P]),
    "m2s_server_wait": (I, [P, U64, ctypes.c_double, P, P]),
    "m2s_server_remove_mesh": (I, [P, ctypes.c_uint32]),
    "m2s_server_stats": (I, [P, P]),
    "m2s_generate_sdf_none_noalloc": (I, [P, U64, P, U64, I, I, P, U64, I, P, P]),
    "m2s_last_grid_stats": (I, [P]),
    "m2s_last_query_stats": (I, [P]),
    "m2s_query_autotune": (I, [P, P, U64, P, P, P]),
    "m2s_test_grid_barrier": (I, [ctypes.c_uint32, ctypes.c_uint32, P]),
    "m2s_set_profiling": (None, [I]),
    "m2s_last_grid_phase_ms": (I, [P]),
    "m2s_last_grid_round_log": (ctypes.c_uint32, [P, ctypes.c_uint32]),
    "m2s_set_query_budget": (None, [ctypes.c_uint32]),
    "m2s_query_budget": (ctypes.c_uint32, []),
    "m2s_status_string": (ctypes.c_char_p, [I]),
    "m2s_last_error": (ctypes.c_char_p, []),
    "m2s_device_available": (I, []),
    "m2s_version": (I, []),
}


class LibraryMissing(RuntimeError):
    pass


def lib():
    """Loads libm2s.so (building it if the sources are newer).  Raises if it cannot be built."""
    global _lib
    with _lock:
        if _lib is None:
            from . import build as _build

            if not _build.up_to_date(FAST) and LIB_PATH == _build.lib_path(FAST):
                try:
                    _build.build(fast=FAST)
                except Exception as e:  # no nvcc: the prebuilt library must exist
                    if not os.path.exists(LIB_PATH):
                        raise LibraryMissing(f"libm2s.so is missing and cannot be built: {e}") from e
            L = ctypes.CDLL(LIB_PATH)
            for name, (res, args) in SIGNATURES.items():
                f = getattr(L, name)
                f.restype = res
                f.argtypes = args
            _lib = L
    return _lib

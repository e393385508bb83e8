"""ctypes bindings of libmlods.so (the C ABI in include/mlods.h).

The library is loaded from ``mlodsurfaces_b200/_lib/libmlods.so``.  There is
no fallback: if the library is missing the import fails with the build
command to run.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

# MLODS_LIBRARY selects another build of the same library (e.g. a variant
# compiled with different tuning constants); the default is the in-tree build.
LIB_PATH = Path(os.environ.get("MLODS_LIBRARY", Path(__file__).resolve().parent / "_lib" / "libmlods.so"))

MLODS_OK = 0
MLODS_ERR_INVALID = 1
MLODS_ERR_CUDA = 2
MLODS_ERR_STATE = 3
MLODS_ERR_CAPACITY = 4
MLODS_ERR_TIMEOUT = 5

GAUSSIAN = 0
SINGULAR = 1
GAUSSIAN_MULTIPLE = 2
INLINE_SIGMAS = 16
MAX_KNN = 32

MODE_MLOD = 0
MODE_GLOBAL = 1
MODE_KNN = 2
MODE_BALL = 3

BLEND_GPU = 0
BLEND_CPU = 1

CONVERGE_OFF = 0
CONVERGE_EXACT = 1
CONVERGE_TOL = 2

NOALLOC_MAX_QUERIES = 524288
PARAMS_FILE_BYTES = 134


class mlods_kernel(C.Structure):
    _fields_ = [
        ("type", C.c_int32),
        ("sigma", C.c_float),
        ("exponent", C.c_float),
        ("constant_shift", C.c_float),
        ("n_sigmas", C.c_int32),
        ("sigmas", C.c_float * INLINE_SIGMAS),
        ("sigmas_ext", C.POINTER(C.c_float)),
    ]


class mlods_params(C.Structure):
    _fields_ = [
        ("cutoff", C.c_float),
        ("min_depth", C.c_int32),
        ("mode", C.c_int32),
        ("knn", C.c_int32),
        ("ball_radius", C.c_float),
        ("blend_rule", C.c_int32),
        ("reorder", C.c_int32),
        ("prune_tol", C.c_float),
        ("converge", C.c_int32),
        ("converge_tol", C.c_float),
        ("local_output", C.c_int32),
        ("queries_per_warp", C.c_int32),
    ]


class mlods_scene_params(C.Structure):
    _fields_ = [
        ("cam_quat", C.c_float * 4),
        ("cam_translation", C.c_float * 3),
        ("cam_dist", C.c_float),
        ("sigma", C.c_float),
        ("fixed_sigmas", C.c_float * 5),
        ("beginning_sigma", C.c_float),
        ("factor", C.c_float),
        ("constant_shift", C.c_float),
        ("exponent", C.c_float),
        ("cutoff", C.c_float),
        ("n_computed_sigmas", C.c_uint32),
        ("max_iterations", C.c_uint32),
        ("max_depth", C.c_uint32),
        ("min_depth", C.c_uint32),
        ("fast_method", C.c_uint32),
        ("kernel_type", C.c_int32),
        ("computed_sigma", C.c_uint8),
        ("cut", C.c_uint8),
        ("n_points", C.c_uint32),
        ("max_upsamples", C.c_uint32),
        ("offset", C.c_float * 6),
    ]


class mlods_server_config(C.Structure):
    _fields_ = [
        ("n_streams", C.c_int32),
        ("max_batch_requests", C.c_int32),
        ("max_batch_queries", C.c_int64),
        ("max_device_bytes", C.c_int64),
        ("max_pending_bytes", C.c_int64),
        ("max_wait_us", C.c_int32),
        ("reserved", C.c_int32),
    ]


class mlods_batch_schedule(C.Structure):
    _fields_ = [
        ("queries_per_warp", C.c_int32),
        ("reorder", C.c_int32),
        ("grid_pct", C.c_int32),
        ("line_order", C.c_int32),
        ("solo_min_queries", C.c_int64),
    ]


class mlods_tree_info(C.Structure):
    _fields_ = [
        ("n_points", C.c_int64),
        ("n_nodes", C.c_int64),
        ("n_extra", C.c_int64),
        ("depth", C.c_int32),
        ("max_depth", C.c_int32),
        ("n_ties", C.c_int64),
        ("bbox_min", C.c_float * 3),
        ("bbox_max", C.c_float * 3),
        ("origin", C.c_double * 3),
        ("device_bytes", C.c_int64),
    ]


class MlodsError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"mlods error {code}: {msg}")
        self.code = code


_P = C.c_void_p
_F = C.POINTER(C.c_float)
_D = C.POINTER(C.c_double)
_I32 = C.POINTER(C.c_int32)
_I64 = C.POINTER(C.c_int64)

# name -> (restype, argtypes); the full exported surface of include/mlods.h
SIGNATURES = {
    "mlods_last_error": (C.c_char_p, []),
    "mlods_version": (C.c_int, []),
    "mlods_tree_build": (C.c_int, [_P, _P, C.c_int64, C.c_int32, _P, C.POINTER(_P)]),
    "mlods_tree_build_device": (C.c_int, [_P, _P, C.c_int64, C.c_int32, _P, C.POINTER(_P)]),
    "mlods_tree_free": (C.c_int, [_P]),
    "mlods_tree_get_info": (C.c_int, [_P, C.POINTER(mlods_tree_info)]),
    "mlods_tree_export": (C.c_int, [_P] + [_P] * 12),
    "mlods_set_kernel": (C.c_int, [_P, C.POINTER(mlods_kernel)]),
    "mlods_default_params": (None, [C.POINTER(mlods_params)]),
    "mlods_set_params": (C.c_int, [_P, C.POINTER(mlods_params)]),
    "mlods_queries_create": (C.c_int, [C.POINTER(_P)]),
    "mlods_queries_destroy": (C.c_int, [_P]),
    "mlods_queries_upload": (C.c_int, [_P, C.c_int64, _P, _P]),
    "mlods_project": (C.c_int, [_P, _P, C.c_int64, C.c_int32, C.c_float, _P, _P, _P]),
    "mlods_queries_free": (C.c_int, [_P]),
    "mlods_project_device": (C.c_int, [_P, C.c_int64, _P, _P, _P, C.c_int32, C.c_float, _P]),
    "mlods_queries_reorganize": (C.c_int, [_P, C.c_int64, _P, C.c_uint32, _P]),
    "mlods_project_host": (C.c_int, [_P, C.c_int64, _P, _P, _P, C.c_int32, C.c_float, C.c_int32, _P]),
    "mlods_last_stats": (C.c_int, [_P, _I64, _I64, _I32, _I64, C.POINTER(C.c_float)]),
    "mlods_last_iterations": (C.c_int, [_P, _I64]),
    "mlods_last_walk_counts": (C.c_int, [_P, _I64, _I64]),
    "mlods_tune_schedule": (C.c_int, [_P, C.c_int64, _P, C.c_int32, _P, C.POINTER(C.c_int32),
                                      C.POINTER(C.c_float)]),
    "mlods_tune_schedule_host": (C.c_int, [_P, C.c_int64, _P, C.c_int32, _I32, C.POINTER(C.c_float)]),
    "mlods_kernel_launches": (C.c_int64, []),
    "mlods_release_scratch": (C.c_int, []),
    "mlods_knn": (C.c_int, [_P, C.c_int64, _P, C.c_int32, _P, _P, _P]),
    "mlods_knn_host": (C.c_int, [_P, C.c_int64, _P, C.c_int32, _P, _P]),
    "mlods_dcgrid_from_points": (C.c_int, [_P, C.c_int64, C.c_int32, _P, _P, C.POINTER(_P)]),
    "mlods_dcgrid_from_points_device": (C.c_int, [_P, C.c_int64, C.c_int32, _P, _P, _P, C.POINTER(_P)]),
    "mlods_dcgrid_info": (C.c_int, [_P, _I64, _I32]),
    "mlods_dcgrid_cells": (C.c_int, [_P, _P]),
    "mlods_dcgrid_free": (C.c_int, [_P]),
    "mlods_dc_evaluate": (C.c_int, [_P, C.c_int64, _P, C.c_int32, _P, C.c_int32, _P, _P, _P, _I64, _P]),
    "mlods_dc_evaluate_device": (C.c_int, [_P, C.c_int64, _P, C.c_int32, _P, C.c_int32, _P, _P, _P, _I64, _P]),
    "mlods_batch_create": (C.c_int, [_P, C.c_int32, C.POINTER(_P)]),
    "mlods_batch_free": (C.c_int, [_P]),
    "mlods_batch_project": (C.c_int, [_P, _P, _P, _P, _P, C.c_int32, C.c_int32, _P]),
    "mlods_batch_tune": (C.c_int, [_P, _P, _P, _P, _P, C.c_int32, _P]),
    "mlods_batch_stats": (C.c_int, [_P, _I64, _I64, _I64, C.POINTER(C.c_float), _I64, _I32]),
    "mlods_batch_get_schedule": (C.c_int, [_P, C.POINTER(mlods_batch_schedule)]),
    "mlods_batch_set_schedule": (C.c_int, [_P, C.POINTER(mlods_batch_schedule)]),
    "mlods_batch_tune_results": (C.c_int, [_P, C.c_int32, C.POINTER(mlods_batch_schedule), C.POINTER(C.c_float),
                                           _I32]),
    "mlods_project_device_noalloc": (C.c_int, [_P, C.c_int64, _P, _P, _P, C.c_int32, C.c_float, _P]),
    "mlods_dcgrid_adaptive": (C.c_int, [_P, C.c_int32, C.c_int32, _P, C.POINTER(_P)]),
    "mlods_dcgrid_xform": (C.c_int, [_P, _P, _I64]),
    "mlods_dc_extract": (C.c_int, [C.c_int64, _P, _P, _P, C.POINTER(_P)]),
    "mlods_mesh_info": (C.c_int, [_P, _I64, _I64]),
    "mlods_mesh_get": (C.c_int, [_P, _P, _P, _P]),
    "mlods_mesh_device_arrays": (C.c_int, [_P, C.POINTER(_P), C.POINTER(_P), C.POINTER(_P)]),
    "mlods_mesh_transform": (C.c_int, [_P, _P]),
    "mlods_mesh_smooth": (C.c_int, [_P]),
    "mlods_mesh_subdivide": (C.c_int, [_P]),
    "mlods_mesh_project": (C.c_int, [_P, _P, C.c_int32, _P]),
    "mlods_mesh_free": (C.c_int, [_P]),
    "mlods_mesh_stage_ms": (C.c_int, [_P, _P]),
    "mlods_dc_mesh": (C.c_int, [_P, _P, C.c_int32, C.c_int32, _P, C.POINTER(_P)]),
    "mlods_server_default_config": (None, [C.POINTER(mlods_server_config)]),
    "mlods_server_create": (C.c_int, [_P, C.c_int32, C.POINTER(mlods_server_config), C.POINTER(_P)]),
    "mlods_server_submit": (C.c_int, [_P, C.c_int32, C.c_int64, _P, _P, _P, C.c_int32, C.POINTER(mlods_kernel),
                                      C.POINTER(C.c_uint64)]),
    "mlods_server_wait": (C.c_int, [_P, C.c_uint64, C.c_int32, C.POINTER(C.c_double)]),
    "mlods_server_stats": (C.c_int, [_P, _I64, _I64, _I64, _I64, C.POINTER(C.c_double)]),
    "mlods_server_free": (C.c_int, [_P]),
    "mlods_server_memory": (C.c_int, [_P, _I64, _I64, _I64, _I64, _I64]),
    "mlods_server_batch_bytes": (C.c_int64, [C.c_int64, C.c_int64]),
    "mlods_cloud_load": (C.c_int, [C.c_char_p, C.c_int32, C.POINTER(_P)]),
    "mlods_cloud_info": (C.c_int, [_P, _I64, _I32, _P, C.POINTER(C.c_float)]),
    "mlods_cloud_get": (C.c_int, [_P, _P, _P]),
    "mlods_cloud_free": (C.c_int, [_P]),
    "mlods_cloud_save": (C.c_int, [C.c_char_p, _P, _P, C.c_int64, _P, C.c_float]),
    "mlods_cloud_normalize": (C.c_int, [_P, C.c_int64, _P, _P, C.POINTER(C.c_float)]),
    "mlods_cloud_morton_order": (C.c_int, [_P, C.c_int64, C.c_int32, _P]),
    "mlods_cloud_sample_around": (C.c_int, [_P, _P, C.c_int64, C.c_int64, C.c_float, C.c_uint64, _P, _P]),
    "mlods_sample_cells_device": (C.c_int, [_P, C.c_int64, C.c_int64, C.c_uint64, _P, _P, _P]),
    "mlods_params_file_load": (C.c_int, [C.c_char_p, C.POINTER(mlods_scene_params)]),
    "mlods_params_file_save": (C.c_int, [C.c_char_p, C.POINTER(mlods_scene_params)]),
}

_lib = None


def load() -> C.CDLL:
    """Load libmlods.so once; raise if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise ImportError(
            f"{LIB_PATH} is missing: build it with `python -m mlodsurfaces_b200.build` "
            "(there is no CPU fallback)"
        )
    lib = C.CDLL(os.fspath(LIB_PATH))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def check(rc: int) -> None:
    if rc != MLODS_OK:
        msg = load().mlods_last_error().decode(errors="replace")
        raise MlodsError(rc, msg)


def ptr(a) -> C.c_void_p:
    """Address of a numpy array or torch tensor (None -> NULL)."""
    if a is None:
        return C.c_void_p(0)
    if hasattr(a, "data_ptr"):
        return C.c_void_p(a.data_ptr())
    return C.c_void_p(a.ctypes.data)

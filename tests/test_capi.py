"""libmlods.so loads, exports every entry point include/mlods.h declares, and
validates arguments before touching the GPU (no device needed)."""
import ctypes as C
import re
from pathlib import Path

import pytest

from mlodsurfaces_b200 import _capi as capi

HEADER = Path(__file__).resolve().parents[1] / "include" / "mlods.h"


def declared_functions():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(mlods_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_entry_points():
    names = declared_functions()
    assert "mlods_tree_build" in names and "mlods_project" in names
    assert len(names) >= 15


def test_library_exports_every_declared_symbol():
    lib = capi.load()
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_python_bindings_cover_the_header():
    assert set(declared_functions()) == set(capi.SIGNATURES)


def test_null_handles_are_rejected_without_a_gpu():
    lib = capi.load()
    assert lib.mlods_set_kernel(None, None) == capi.MLODS_ERR_INVALID
    assert b"null" in lib.mlods_last_error()
    assert lib.mlods_project(None, None, 10, 1, -1.0, None, None, None) == capi.MLODS_ERR_INVALID
    assert lib.mlods_queries_upload(None, 10, None, None) == capi.MLODS_ERR_INVALID
    assert lib.mlods_queries_destroy(None) == capi.MLODS_OK
    assert lib.mlods_tree_build(None, None, 0, 12, None, C.byref(C.c_void_p())) == capi.MLODS_ERR_INVALID
    assert lib.mlods_tree_free(None) == capi.MLODS_OK


def test_default_params_follow_the_reference():
    lib = capi.load()
    p = capi.mlods_params()
    lib.mlods_default_params(C.byref(p))
    assert p.cutoff == pytest.approx(2.0)  # GPUUtils.h:63
    assert p.min_depth == 0
    assert p.knn == 20 and p.ball_radius == pytest.approx(0.1)
    assert p.blend_rule == capi.BLEND_GPU and p.mode == capi.MODE_MLOD


def test_error_raises():
    with pytest.raises(capi.MlodsError):
        capi.check(capi.load().mlods_set_params(None, None))


def test_apss_lifecycle_methods_without_a_gpu():
    """APSS::stop is a no-op here; eraseAndRestart leaves an empty octree
    (GPUUtils.cu:394-404)."""
    from mlodsurfaces_b200 import APSSOctree, Fastapss

    t = APSSOctree()
    f = Fastapss(t)
    f.stop()
    f.eraseAndRestart()
    assert isinstance(f.CPU(), APSSOctree) and f.CPU() is not t


def test_new_entry_points_reject_null_handles_without_a_gpu():
    lib = capi.load()
    ci = C.c_int32(0)
    assert lib.mlods_tune_schedule(None, 10, None, 1, None, C.byref(ci), None) == capi.MLODS_ERR_INVALID
    assert lib.mlods_tune_schedule_host(None, 10, None, 1, C.byref(ci), None) == capi.MLODS_ERR_INVALID
    assert lib.mlods_last_walk_counts(None, None, None) == capi.MLODS_ERR_INVALID
    sched = capi.mlods_batch_schedule(2, 1, 100, 0, 0)
    assert lib.mlods_batch_set_schedule(None, C.byref(sched)) == capi.MLODS_ERR_INVALID
    assert lib.mlods_batch_get_schedule(None, C.byref(sched)) == capi.MLODS_ERR_INVALID
    assert lib.mlods_batch_tune_results(None, 0, None, None, C.byref(ci)) == capi.MLODS_ERR_INVALID
    assert lib.mlods_batch_stats(None, None, None, None, None, None, None) == capi.MLODS_ERR_INVALID
    assert lib.mlods_batch_create(None, 0, C.byref(C.c_void_p())) == capi.MLODS_ERR_INVALID
    assert lib.mlods_batch_free(None) == capi.MLODS_OK


def test_server_batch_footprint_grows_with_the_batch():
    """mlods_server_batch_bytes is host arithmetic: a batch's device bytes
    grow with its queries and requests."""
    lib = capi.load()
    small = lib.mlods_server_batch_bytes(4096, 1)
    assert small > 4096 * 36
    assert lib.mlods_server_batch_bytes(8192, 1) > small
    assert lib.mlods_server_batch_bytes(4096, 64) > small

"""Point-set and parameter files of the reference application.

* :func:`load_cloud` / :func:`save_cloud` -- Pn::load / Pn::save
  (sources/apss/Pn.cpp:102-241): ``.pn`` raw float32 records and ``.ply``
  vertex elements, optional Pn::normalize (Pn.cpp:262-290);
* :func:`load_params` / :func:`save_params` -- the 134-byte ``.params`` file
  of scene::loadParameters (sources/scene/scene.cpp:1183-1250);
* :func:`kernel_from_params` -- the kernel those parameters describe, with
  the sigmas scaled by the tree's box radius as the loader does
  (Kernel::updateSigmas, sources/apss/Kernel.cpp:172-190).

The file work runs in libmlods (host code).
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import _capi as capi
from .apss import Kernel


def _path(p) -> bytes:
    return os.fsencode(os.fspath(p))


def load_cloud(path, normalize: bool = True):
    """(points (n, 3) float32, normals (n, 3) or None, offset (3,), norme)."""
    lib = capi.load()
    h = C.c_void_p(0)
    capi.check(lib.mlods_cloud_load(_path(path), 1 if normalize else 0, C.byref(h)))
    try:
        n = C.c_int64(0)
        hn = C.c_int32(0)
        off = np.zeros(3, np.float32)
        norme = C.c_float(1.0)
        capi.check(lib.mlods_cloud_info(h, C.byref(n), C.byref(hn), capi.ptr(off), C.byref(norme)))
        pts = np.empty((n.value, 3), np.float32)
        nrm = np.empty((n.value, 3), np.float32) if hn.value else None
        capi.check(lib.mlods_cloud_get(h, capi.ptr(pts), capi.ptr(nrm)))
        return pts, nrm, off, float(norme.value)
    finally:
        lib.mlods_cloud_free(h)


def save_cloud(path, points, normals=None, offset=None, norme: float = 1.0) -> None:
    """Writes points * norme + offset (and normals) as Pn::save does."""
    lib = capi.load()
    p = np.ascontiguousarray(np.asarray(points, np.float32).reshape(-1, 3))
    n = None if normals is None else np.ascontiguousarray(np.asarray(normals, np.float32).reshape(-1, 3))
    o = None if offset is None else np.ascontiguousarray(np.asarray(offset, np.float32).reshape(3))
    capi.check(lib.mlods_cloud_save(_path(path), capi.ptr(p), capi.ptr(n), len(p), capi.ptr(o), float(norme)))


def normalize(points):
    """Pn::normalize of an array: (points, offset, norme)."""
    lib = capi.load()
    p = np.ascontiguousarray(np.asarray(points, np.float32).reshape(-1, 3))
    out = np.empty_like(p)
    off = np.zeros(3, np.float32)
    norme = C.c_float(0)
    capi.check(lib.mlods_cloud_normalize(capi.ptr(p), len(p), capi.ptr(out), capi.ptr(off), C.byref(norme)))
    return out, off, float(norme.value)


def morton_order(points, grid: int = 64) -> np.ndarray:
    """Pn::order: the permutation that sorts the points by Morton code on a
    grid^3 lattice (ties keep their input order)."""
    lib = capi.load()
    p = np.ascontiguousarray(np.asarray(points, np.float32).reshape(-1, 3))
    perm = np.empty(len(p), np.uint32)
    capi.check(lib.mlods_cloud_morton_order(capi.ptr(p), len(p), int(grid), capi.ptr(perm)))
    return perm


def sample_around(points, normals, n: int, factor: float = 1.0, seed: int = 0):
    """Pn::initialize(n, pointSetToFit, factor): n queries near the points
    (random tangent-disk offsets of radius meanGap), with their normals."""
    lib = capi.load()
    p = np.ascontiguousarray(np.asarray(points, np.float32).reshape(-1, 3))
    nv = np.ascontiguousarray(np.asarray(normals, np.float32).reshape(-1, 3))
    out_p = np.empty((int(n), 3), np.float32)
    out_n = np.empty((int(n), 3), np.float32)
    capi.check(lib.mlods_cloud_sample_around(capi.ptr(p), capi.ptr(nv), len(p), int(n), float(factor),
                                             C.c_uint64(seed), capi.ptr(out_p), capi.ptr(out_n)))
    return out_p, out_n


def sample_cells(cells, n: int, seed: int = 0, device=None, stream=None):
    """scene::generateFromOctree (scene.cpp:733-756) on the device: n points
    in cells {depth, x, y, z} of the [-1, 1]^3 octree drawn uniformly, each at
    its cell centre plus a uniform offset in [-2, 2)^3 / 2^depth; the normals
    are the points.  Returns two (n, 3) float32 CUDA tensors.  Asynchronous on
    `stream` (default: torch's current stream)."""
    import torch

    lib = capi.load()
    dev = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
    c = torch.as_tensor(np.ascontiguousarray(np.asarray(cells, np.int32).reshape(-1, 4))) \
        if not isinstance(cells, torch.Tensor) else cells.to(torch.int32).reshape(-1, 4).contiguous()
    c = c.to(dev)
    out_p = torch.empty((int(n), 3), dtype=torch.float32, device=dev)
    out_n = torch.empty((int(n), 3), dtype=torch.float32, device=dev)
    s = stream if stream is not None else torch.cuda.current_stream(dev).cuda_stream
    capi.check(lib.mlods_sample_cells_device(capi.ptr(c), int(c.shape[0]), int(n), C.c_uint64(seed),
                                             capi.ptr(out_p), capi.ptr(out_n), C.c_void_p(s)))
    return out_p, out_n


_ARRAYS = {"cam_quat": 4, "cam_translation": 3, "fixed_sigmas": 5, "offset": 6}


def load_params(path) -> dict:
    lib = capi.load()
    p = capi.mlods_scene_params()
    capi.check(lib.mlods_params_file_load(_path(path), C.byref(p)))
    out = {}
    for name, _ in capi.mlods_scene_params._fields_:
        v = getattr(p, name)
        out[name] = [float(x) for x in v] if name in _ARRAYS else v
    return out


def save_params(path, params: dict) -> None:
    lib = capi.load()
    p = capi.mlods_scene_params()
    for name, _ in capi.mlods_scene_params._fields_:
        if name not in params:
            continue
        if name in _ARRAYS:
            arr = getattr(p, name)
            for i, x in enumerate(params[name]):
                arr[i] = float(x)
        else:
            setattr(p, name, params[name])
    capi.check(lib.mlods_params_file_save(_path(path), C.byref(p)))


def kernel_from_params(params: dict, radius: float) -> Kernel:
    """The weight kernel a .params file describes, scaled by the box radius."""
    k = Kernel()
    k.type = int(params["kernel_type"])
    k.sigma = float(params["sigma"])
    k.fixedSigmas = list(params["fixed_sigmas"])
    k.beginningSigma = float(params["beginning_sigma"])
    k.factor = float(params["factor"])
    k.constant_shift = float(params["constant_shift"])
    k.exponent = float(params["exponent"])
    k.nbOfComputedSigmas = int(params["n_computed_sigmas"])
    k.updateSigmas(bool(params["computed_sigma"]), radius)
    return k

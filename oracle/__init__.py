"""Test infrastructure: the CPU checkers of the projection path.

* ``liboracle`` -- oracle/mlods_oracle.c, an FP64 restatement of the
  reference's algorithm (tree build, MLoD traversal with both blend rules,
  sphere fit, global/kNN/ball APSS, DC corner field and vertex).
* ``libref`` -- the reference's own CPU code (sources/apss/CPUUtils.cpp,
  Kernel.cpp, kdTreeNN.h) compiled by oracle/Makefile behind ref_shim.cpp.

Only tests, the smoke test and the benchmark's CPU-baseline/reference arms
use this module; the library never does.
"""
from __future__ import annotations

import ctypes as C
import os
import shutil
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ORACLE_SO = HERE / "_build" / "libmlods_oracle.so"
REF_SO = HERE / "_ref" / "libmlods_ref.so"
# The reference project's root (sources/, lib/, data/), from $MLODS_REF_ROOT;
# the compiled checkers under _ref/ are used without it.
REF_ROOT = Path(os.environ["MLODS_REF_ROOT"]) if os.environ.get("MLODS_REF_ROOT") else None
REFDC_SO = HERE / "_ref" / "libmlods_refdc.so"
REF_DATA = HERE / "_ref" / "data"

_P = C.c_void_p
_orc = None
_ref = None


def build(with_ref: bool = True, ref_root=None) -> None:
    """Compile the oracle, and the reference checkers when the reference
    project is at ``ref_root`` (default $MLODS_REF_ROOT)."""
    root = Path(ref_root) if ref_root else REF_ROOT
    targets = ["oracle"]
    if with_ref and root is not None and (root / "sources" / "apss").is_dir():
        targets += ["ref", "refdc", "refdata"]
        if shutil.which("nvcc"):  # the reference's own GPU path, for the GPU-side pins
            targets.append("refgpu")
    args = [f"REF_ROOT={root}"] if root is not None else []
    subprocess.run(["make", "-s", "-C", str(HERE)] + args + targets, check=True)


def ref_available() -> bool:
    return REF_SO.exists()


def _ptr(a):
    return C.c_void_p(0) if a is None else C.c_void_p(a.ctypes.data)


def orc() -> C.CDLL:
    global _orc
    if _orc is None:
        if not ORACLE_SO.exists():
            build(with_ref=False)
        lib = C.CDLL(os.fspath(ORACLE_SO))
        lib.orc_tree_build.restype = _P
        lib.orc_tree_build.argtypes = [_P, _P, C.c_int64, C.c_int]
        lib.orc_tree_free.argtypes = [_P]
        lib.orc_tree_num_nodes.restype = C.c_int64
        lib.orc_tree_num_nodes.argtypes = [_P]
        lib.orc_tree_num_ties.restype = C.c_int64
        lib.orc_tree_num_ties.argtypes = [_P]
        lib.orc_tree_radius.restype = C.c_double
        lib.orc_tree_radius.argtypes = [_P]
        lib.orc_tree_export.argtypes = [_P] + [_P] * 12
        lib.orc_project_mlod.argtypes = [_P, _P, C.c_int64, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double,
                                         _P, C.c_int, C.c_int, C.c_double, C.c_int, C.c_double, _P, _P, _P]
        lib.orc_project_global.argtypes = [_P, _P, C.c_int64, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double,
                                           _P, C.c_int, C.c_double, _P, _P]
        lib.orc_knn.argtypes = [_P, C.c_int64, _P, C.c_int64, C.c_int, _P, _P, _P]
        lib.orc_project_apss.argtypes = [_P, _P, C.c_int64, _P, C.c_int64, C.c_int, C.c_int, C.c_int, C.c_double,
                                         C.c_int, C.c_double, C.c_double, C.c_double, _P, C.c_int, C.c_double, _P, _P]
        lib.orc_dc_field.argtypes = [_P, _P, _P, C.c_int64, _P]
        lib.orc_dc_vertex.argtypes = [_P, C.c_double, _P, _P, _P]
        _orc = lib
    return _orc


def ref() -> C.CDLL:
    global _ref
    if _ref is None:
        if not REF_SO.exists():
            raise FileNotFoundError(f"{REF_SO} not built (needs the reference sources)")
        lib = C.CDLL(os.fspath(REF_SO))
        lib.ref_tree_build.restype = _P
        lib.ref_tree_build.argtypes = [_P, _P, C.c_int64, C.c_int, C.c_uint]
        lib.ref_tree_free.argtypes = [_P]
        lib.ref_tree_num_nodes.restype = C.c_int64
        lib.ref_tree_num_nodes.argtypes = [_P]
        lib.ref_tree_depth.restype = C.c_int
        lib.ref_tree_depth.argtypes = [_P]
        lib.ref_tree_export.argtypes = [_P] + [_P] * 12
        lib.ref_project.restype = C.c_double
        lib.ref_project.argtypes = [_P, _P, _P, _P, C.c_int64, C.c_int, C.c_int, C.c_float, C.c_float, C.c_float, _P,
                                    C.c_int, C.c_float, C.c_int, C.c_float, C.c_int, C.c_int, C.c_float, C.c_int]
        lib.ref_kdtree_knn.argtypes = [_P, C.c_int64, _P, C.c_int64, C.c_int, _P, _P]
        _ref = lib
    return _ref


def _kargs(kernel):
    """(type, sigma, exponent, shift, sigmas float64 array, nsig) of a Kernel-like object."""
    sig = np.ascontiguousarray(np.asarray(kernel.sigmas if len(kernel.sigmas) else [0.0], np.float64))
    return int(kernel.type), float(kernel.sigma), float(kernel.exponent), float(kernel.constant_shift), sig, \
        len(kernel.sigmas)


def _f32(a):
    return np.ascontiguousarray(np.asarray(a, np.float32))


EXPORT_KEYS = ["depth", "parent", "first_child", "n_children", "next_brother", "leaf_off", "leaf_cnt", "perm",
               "bmin", "bmax"]


class OracleTree:
    """FP64 restatement of APSSOctree (oracle/mlods_oracle.c)."""

    def __init__(self, pts, nrm, max_depth: int = 12):
        self.pts = _f32(pts)
        self.nrm = _f32(nrm)
        self._h = orc().orc_tree_build(_ptr(self.pts), _ptr(self.nrm), len(self.pts), int(max_depth))
        if not self._h:
            raise ValueError("oracle tree build failed")

    def __del__(self):
        if getattr(self, "_h", None):
            orc().orc_tree_free(self._h)
            self._h = None

    @property
    def n_nodes(self) -> int:
        return int(orc().orc_tree_num_nodes(self._h))

    @property
    def n_ties(self) -> int:
        return int(orc().orc_tree_num_ties(self._h))

    @property
    def radius(self) -> float:
        return float(orc().orc_tree_radius(self._h))

    def export(self) -> dict:
        nn, n = self.n_nodes, len(self.pts)
        out = {k: np.empty(nn, np.int32) for k in EXPORT_KEYS[:7]}
        out["perm"] = np.empty(n, np.int32)
        out["bmin"] = np.empty((nn, 3), np.float32)
        out["bmax"] = np.empty((nn, 3), np.float32)
        out["mom"] = np.empty((nn, 9), np.float64)
        out["area"] = np.empty(n, np.float64)
        keys = EXPORT_KEYS + ["mom", "area"]
        orc().orc_tree_export(self._h, *[_ptr(out[k]) for k in keys])
        return out

    def project_mlod(self, q, n_iter, kernel, rule=0, cutoff=2.0, min_depth=0, step_max=-1.0, visited=False):
        q = _f32(q)
        n = len(q)
        op = np.empty((n, 3), np.float64)
        on = np.empty((n, 3), np.float64)
        vis = np.empty(n, np.int64) if visited else None
        t, s, e, sh, sig, ns = _kargs(kernel)
        orc().orc_project_mlod(self._h, _ptr(q), n, int(n_iter), t, s, e, sh, _ptr(sig), ns, int(rule),
                               float(cutoff), int(min_depth), float(step_max), _ptr(op), _ptr(on), _ptr(vis))
        return (op, on, vis) if visited else (op, on)

    def project_global(self, q, n_iter, kernel, step_max=-1.0):
        q = _f32(q)
        n = len(q)
        op = np.empty((n, 3), np.float64)
        on = np.empty((n, 3), np.float64)
        t, s, e, sh, sig, ns = _kargs(kernel)
        orc().orc_project_global(self._h, _ptr(q), n, int(n_iter), t, s, e, sh, _ptr(sig), ns, float(step_max),
                                 _ptr(op), _ptr(on))
        return op, on


def knn(pts, q, k):
    """Exact kNN (brute force, kdTreeNN distance arithmetic); (idx, d2, tie)."""
    pts, q = _f32(pts), _f32(q)
    idx = np.empty((len(q), k), np.int32)
    d2 = np.empty((len(q), k), np.float64)
    tie = np.empty(len(q), np.int32)
    orc().orc_knn(_ptr(pts), len(pts), _ptr(q), len(q), int(k), _ptr(idx), _ptr(d2), _ptr(tie))
    return idx, d2, tie


def project_apss(pts, nrm, q, n_iter, kernel, mode, k=20, ball_r=0.1, step_max=1.0):
    """kNN (mode 0) / ball (mode 1) APSS restatement (CPUUtils.cpp:690-737)."""
    pts, nrm, q = _f32(pts), _f32(nrm), _f32(q)
    op = np.empty((len(q), 3), np.float64)
    on = np.empty((len(q), 3), np.float64)
    t, s, e, sh, sig, ns = _kargs(kernel)
    orc().orc_project_apss(_ptr(pts), _ptr(nrm), len(pts), _ptr(q), len(q), int(n_iter), int(mode), int(k),
                           float(ball_r), t, s, e, sh, _ptr(sig), ns, float(step_max), _ptr(op), _ptr(on))
    return op, on


class RefTree:
    """The reference's own APSSOctree, built and run on the CPU (oracle/_ref)."""

    def __init__(self, pts, nrm, max_depth: int = 12, seed: int = 0):
        self.pts = _f32(pts)
        self.nrm = _f32(nrm)
        self._h = ref().ref_tree_build(_ptr(self.pts), _ptr(self.nrm), len(self.pts), int(max_depth), int(seed))

    def __del__(self):
        if getattr(self, "_h", None):
            ref().ref_tree_free(self._h)
            self._h = None

    @property
    def n_nodes(self) -> int:
        return int(ref().ref_tree_num_nodes(self._h))

    @property
    def depth(self) -> int:
        return int(ref().ref_tree_depth(self._h))

    def export(self) -> dict:
        nn, n = self.n_nodes, len(self.pts)
        out = {k: np.empty(nn, np.int32) for k in EXPORT_KEYS[:7]}
        out["perm"] = np.empty(n, np.int32)
        out["bmin"] = np.empty((nn, 3), np.float32)
        out["bmax"] = np.empty((nn, 3), np.float32)
        out["stats"] = np.empty((nn, 9), np.float32)
        out["area"] = np.empty(n, np.float32)
        keys = EXPORT_KEYS + ["stats", "area"]
        ref().ref_tree_export(self._h, *[_ptr(out[k]) for k in keys])
        return out

    def cpu_sphere(self, q, kernel, k=20):
        """APSSOctree::cpuSphere at each query: (n, 5) of (u0, u123, u4)."""
        q = _f32(q)
        out = np.empty((len(q), 5), np.float32)
        sig = np.ascontiguousarray(np.asarray(kernel.sigmas if len(kernel.sigmas) else [0.0], np.float32))
        lib = ref()
        lib.ref_cpu_sphere.argtypes = [_P, _P, C.c_int64, C.c_int, C.c_int, C.c_float, C.c_float, C.c_float, _P,
                                       C.c_int, _P]
        lib.ref_cpu_sphere(self._h, _ptr(q), len(q), int(k), int(kernel.type), float(kernel.sigma),
                           float(kernel.exponent), float(kernel.constant_shift), _ptr(sig), len(kernel.sigmas),
                           _ptr(out))
        return out

    def project(self, q, n_iter, kernel, cutoff=2.0, min_depth=0, step_max=-1.0, mode=0, k=20, ball_r=0.1,
                nthreads=0):
        """Returns (points, normals, seconds) from APSSOctree::projectCPU."""
        q = _f32(q)
        n = len(q)
        op = np.empty((n, 3), np.float32)
        on = np.empty((n, 3), np.float32)
        sig = np.ascontiguousarray(np.asarray(kernel.sigmas if len(kernel.sigmas) else [0.0], np.float32))
        secs = ref().ref_project(self._h, _ptr(q), _ptr(op), _ptr(on), n, int(n_iter), int(kernel.type),
                                 float(kernel.sigma), float(kernel.exponent), float(kernel.constant_shift), _ptr(sig),
                                 len(kernel.sigmas), float(cutoff), int(min_depth), float(step_max), int(mode),
                                 int(k), float(ball_r), int(nthreads))
        return op, on, secs


def ref_kdtree_knn(pts, q, k):
    pts, q = _f32(pts), _f32(q)
    idx = np.empty((len(q), k), np.int32)
    d2 = np.empty((len(q), k), np.float64)
    ref().ref_kdtree_knn(_ptr(pts), len(pts), _ptr(q), len(q), int(k), _ptr(idx), _ptr(d2))
    return idx, d2


REFGPU_SO = HERE / "_ref" / "libmlods_refgpu.so"
_refgpu = None


def refgpu_available() -> bool:
    return REFGPU_SO.exists()


def refgpu() -> C.CDLL:
    global _refgpu
    if _refgpu is None:
        if not REFGPU_SO.exists():
            raise FileNotFoundError(f"{REFGPU_SO} not built (needs the reference sources and nvcc)")
        lib = C.CDLL(os.fspath(REFGPU_SO))
        lib.refgpu_create.restype = _P
        lib.refgpu_create.argtypes = [_P, _P, C.c_int64, C.c_int, C.c_int, C.c_float, C.c_float, C.c_float, _P,
                                      C.c_int, C.c_float, C.c_int, C.c_char_p, C.c_int]
        lib.refgpu_project.restype = C.c_double
        lib.refgpu_project.argtypes = [_P, _P, C.c_int64, C.c_int, C.c_int, C.c_float, _P, _P]
        lib.refgpu_free.argtypes = [_P]
        lib.refgpu_set_kernel.argtypes = [_P, C.c_int, C.c_float, C.c_float, C.c_float, _P, C.c_int]
        lib.refgpu_global_create.restype = _P
        lib.refgpu_global_create.argtypes = [_P, _P, C.c_int64, C.c_int, C.c_int, C.c_float, C.c_float, C.c_float,
                                             _P, C.c_int]
        lib.refgpu_global_project.restype = C.c_double
        lib.refgpu_global_project.argtypes = [_P, _P, C.c_int64, C.c_int, C.c_float, _P, _P]
        lib.refgpu_global_free.argtypes = [_P]
        _refgpu = lib
    return _refgpu


class RefGpu:
    """The reference's own Fastapss (GPU) on the reference's host-built tree.
    Refuses trees of depth >= 12 (the reference kernel would index its
    per-depth array out of bounds there)."""

    def __init__(self, pts, nrm, kernel, cutoff=2.0, min_depth=0, max_depth=12):
        self.pts = _f32(pts)
        self.nrm = _f32(nrm)
        sig = np.ascontiguousarray(np.asarray(kernel.sigmas if len(kernel.sigmas) else [0.0], np.float32))
        err = C.create_string_buffer(256)
        self._h = refgpu().refgpu_create(_ptr(self.pts), _ptr(self.nrm), len(self.pts), int(max_depth),
                                         int(kernel.type), float(kernel.sigma), float(kernel.exponent),
                                         float(kernel.constant_shift), _ptr(sig), len(kernel.sigmas), float(cutoff),
                                         int(min_depth), err, 256)
        if not self._h:
            raise ValueError(err.value.decode())

    def __del__(self):
        if getattr(self, "_h", None):
            refgpu().refgpu_free(self._h)
            self._h = None

    def set_kernel(self, kernel):
        """APSS::updateKernel with a new kernel (the tree stays)."""
        sig = np.ascontiguousarray(np.asarray(kernel.sigmas if len(kernel.sigmas) else [0.0], np.float32))
        refgpu().refgpu_set_kernel(self._h, int(kernel.type), float(kernel.sigma), float(kernel.exponent),
                                   float(kernel.constant_shift), _ptr(sig), len(kernel.sigmas))

    def project(self, q, calls=10, iters_per_call=1, step_max=-1.0):
        """(points, normals, device milliseconds of the project calls)."""
        q = _f32(q)
        op = np.empty((len(q), 3), np.float32)
        on = np.empty((len(q), 3), np.float32)
        ms = refgpu().refgpu_project(self._h, _ptr(q), len(q), int(calls), int(iters_per_call), float(step_max),
                                     _ptr(op), _ptr(on))
        if ms < 0:
            raise ValueError("query count out of the reference's launch range")
        return op, on, ms


class RefGpuGlobal:
    """The reference's own GlobalAPSS (GPU, all points per query)."""

    def __init__(self, pts, nrm, kernel, max_depth=12):
        self.pts = _f32(pts)
        self.nrm = _f32(nrm)
        sig = np.ascontiguousarray(np.asarray(kernel.sigmas if len(kernel.sigmas) else [0.0], np.float32))
        self._h = refgpu().refgpu_global_create(_ptr(self.pts), _ptr(self.nrm), len(self.pts), int(max_depth),
                                                int(kernel.type), float(kernel.sigma), float(kernel.exponent),
                                                float(kernel.constant_shift), _ptr(sig), len(kernel.sigmas))

    def __del__(self):
        if getattr(self, "_h", None):
            refgpu().refgpu_global_free(self._h)
            self._h = None

    def project(self, q, calls=10, step_max=-1.0):
        """(points, normals, device milliseconds of `calls` one-step calls)."""
        q = _f32(q)
        op = np.empty((len(q), 3), np.float32)
        on = np.empty((len(q), 3), np.float32)
        ms = refgpu().refgpu_global_project(self._h, _ptr(q), len(q), int(calls), float(step_max), _ptr(op),
                                            _ptr(on))
        if ms < 0:
            raise ValueError("query count out of the reference's launch range")
        return op, on, ms


# ---------------------------------------------------------------- reference DC
# The reference's own dual-contouring and point-set code (oracle/_ref/
# libmlods_refdc.so, built from scene/upsample.cpp, dual-contouring/octree.h,
# dual_contouring.h and apss/Pn.cpp).  Every projection it asks for is made by
# a Python callable project(pts (n,3) float32, iters, step_max, cpu_rule) ->
# (points, normals), so a test can hand it the projections of the library
# under test and compare everything else bit for bit.
REFDC_PROJECT_FN = C.CFUNCTYPE(None, C.c_void_p, C.c_int64, C.POINTER(C.c_float), C.POINTER(C.c_float), C.c_int32,
                               C.c_float, C.c_int32)
_refdc = None


def refdc_available() -> bool:
    return REFDC_SO.exists()


def refdc() -> C.CDLL:
    global _refdc
    if _refdc is None:
        if not REFDC_SO.exists():
            raise FileNotFoundError(f"{REFDC_SO} not built (needs the reference sources)")
        lib = C.CDLL(os.fspath(REFDC_SO))
        lib.refdc_grid_adaptive.restype = _P
        lib.refdc_grid_adaptive.argtypes = [REFDC_PROJECT_FN, _P, C.c_int32, C.c_int32]
        lib.refdc_grid_points.restype = _P
        lib.refdc_grid_points.argtypes = [_P, C.c_int64, C.c_int32]
        lib.refdc_grid_size.restype = C.c_int64
        lib.refdc_grid_size.argtypes = [_P]
        lib.refdc_grid_max_depth.restype = C.c_int32
        lib.refdc_grid_max_depth.argtypes = [_P]
        lib.refdc_grid_projected.restype = C.c_int64
        lib.refdc_grid_projected.argtypes = [_P]
        lib.refdc_grid_cells.argtypes = [_P, _P]
        lib.refdc_grid_xform.argtypes = [_P, _P]
        lib.refdc_grid_free.argtypes = [_P]
        lib.refdc_mesh.restype = _P
        lib.refdc_mesh.argtypes = [_P, REFDC_PROJECT_FN, _P, C.c_int32]
        lib.refdc_mesh_sizes.argtypes = [_P] + [C.POINTER(C.c_int64)] * 5
        lib.refdc_mesh_get.argtypes = [_P] * 8
        lib.refdc_mesh_free.argtypes = [_P]
        lib.refpn_load.restype = _P
        lib.refpn_load.argtypes = [C.c_char_p, C.c_int32, C.POINTER(C.c_int64)]
        lib.refpn_get.argtypes = [_P, _P, _P, C.POINTER(C.c_int64), _P, _P]
        lib.refpn_free.argtypes = [_P]
        lib.refpn_order.argtypes = [_P, C.c_int64, C.c_int32, _P]
        _refdc = lib
    return _refdc


def _refdc_callback(project):
    def cb(_ctx, n, pts, nrm, iters, step_max, cpu_rule):
        try:
            p = np.ctypeslib.as_array(pts, shape=(int(n), 3))
            nn = np.ctypeslib.as_array(nrm, shape=(int(n), 3))
            op, on = project(p.copy(), int(iters), float(step_max), int(cpu_rule))
            p[:] = op
            nn[:] = on
        except BaseException as e:  # an exception cannot cross the C frames
            _refdc_callback.error = e
    return REFDC_PROJECT_FN(cb)


def _refdc_raise():
    err = getattr(_refdc_callback, "error", None)
    _refdc_callback.error = None
    if err is not None:
        raise err


class RefDCGrid:
    """A DC grid made by the reference's OctreeGenerator and uniformize*."""

    def __init__(self, handle):
        self._h = handle

    @classmethod
    def adaptive(cls, project, max_depth: int, cut: bool = False) -> "RefDCGrid":
        """OctreeGenerator::generate + uniformize (scene.cpp:155-167, :1297)."""
        cb = _refdc_callback(project)
        h = refdc().refdc_grid_adaptive(cb, None, int(max_depth), int(bool(cut)))
        _refdc_raise()
        return cls(h)

    @classmethod
    def from_points(cls, pts, max_depth: int) -> "RefDCGrid":
        """generateFromPoints + uniformizeFromPoints over [-1, 1]^3."""
        pts = _f32(pts)
        return cls(refdc().refdc_grid_points(_ptr(pts), len(pts), int(max_depth)))

    def __del__(self):
        if getattr(self, "_h", None):
            refdc().refdc_grid_free(self._h)
            self._h = None

    def cells(self) -> np.ndarray:
        out = np.empty((int(refdc().refdc_grid_size(self._h)), 4), np.int32)
        refdc().refdc_grid_cells(self._h, _ptr(out))
        return out

    @property
    def max_depth(self) -> int:
        return int(refdc().refdc_grid_max_depth(self._h))

    @property
    def projected(self) -> int:
        return int(refdc().refdc_grid_projected(self._h))

    def xform(self) -> np.ndarray:
        out = np.empty(12, np.float32)
        refdc().refdc_grid_xform(self._h, _ptr(out))
        return out

    def mesh(self, project, refine_rounds: int = 2) -> dict:
        """scene::computeDualContouring after the grid: corner field (one
        projection per corner slot), extraction, transform, projection and
        refine_rounds x (smooth, subdivide, project)."""
        cb = _refdc_callback(project)
        lib = refdc()
        h = lib.refdc_mesh(self._h, cb, None, int(refine_rounds))
        _refdc_raise()
        try:
            sz = [C.c_int64() for _ in range(5)]
            lib.refdc_mesh_sizes(h, *[C.byref(s) for s in sz])
            nc, nev, nei, nv, ni = (int(s.value) for s in sz)
            out = {"corner_keys": np.empty((nc, 3), np.int32), "corner_vals": np.empty(nc, np.float32),
                   "ext_vertices": np.empty((nev, 3), np.float32), "ext_indices": np.empty(nei, np.uint32),
                   "vertices": np.empty((nv, 3), np.float32), "normals": np.empty((nv, 3), np.float32),
                   "indices": np.empty(ni, np.uint32)}
            lib.refdc_mesh_get(h, *[_ptr(out[k]) for k in ("corner_keys", "corner_vals", "ext_vertices",
                                                             "ext_indices", "vertices", "normals", "indices")])
        finally:
            lib.refdc_mesh_free(h)
        return out


def refpn_load(path, normalize: bool = True) -> dict:
    """Pn::load (Pn.cpp:102-164) with Pn::normalize (Pn.cpp:262-290)."""
    lib = refdc()
    n = C.c_int64()
    h = lib.refpn_load(os.fsencode(str(path)), int(bool(normalize)), C.byref(n))
    try:
        pts = np.empty((int(n.value), 3), np.float32)
        nrm = np.empty((int(n.value), 3), np.float32)
        nn = C.c_int64()
        off = np.empty(3, np.float32)
        norme = np.empty(1, np.float32)
        lib.refpn_get(h, _ptr(pts), _ptr(nrm), C.byref(nn), _ptr(off), _ptr(norme))
    finally:
        lib.refpn_free(h)
    return {"pts": pts, "nrm": nrm[: int(nn.value)], "offset": off, "norme": float(norme[0])}


def refpn_order(pts, grid: int = 64) -> np.ndarray:
    """The positions after Pn::order(grid) (Pn.cpp:388-445)."""
    pts = _f32(pts)
    out = np.empty_like(pts)
    refdc().refpn_order(_ptr(pts), len(pts), int(grid), _ptr(out))
    return out


def ref_data(name: str):
    """Path of a copy of one of the reference's shipped files (data/), or None."""
    p = REF_DATA / name
    return p if p.exists() else None

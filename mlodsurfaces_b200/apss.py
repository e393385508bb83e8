"""Python mirror of the reference's projection API over libmlods.so.

Class and method names follow the reference's C++ classes so that code (and
tests) written against them read the same:

* :class:`Kernel` -- ``class Kernel`` (sources/apss/Kernel.h:24-60)
* :class:`APSSOctree` -- ``class APSSOctree`` (sources/apss/CPUUtils.h:166-229);
  ``build`` runs on the device.
* :class:`APSS`, :class:`Fastapss` -- ``class APSS`` (sources/apss/GPUUtils.h:22-67)
  and ``class Fastapss`` (sources/apss/Fastapss.h:32-51): upload queries,
  project them in place ``n_iterations`` steps per call, copy back on demand.

Arrays are numpy ``float32`` arrays of shape (n, 3) on the host.  Errors raise
:class:`~mlodsurfaces_b200._capi.MlodsError` (the reference exits the process).
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import _capi as capi


def _f32x3(a, name: str) -> np.ndarray:
    a = np.ascontiguousarray(np.asarray(a, dtype=np.float32))
    if a.ndim != 2 or a.shape[1] != 3:
        raise ValueError(f"{name} must have shape (n, 3)")
    return a


class Kernel:
    """Weight kernel value type (Kernel.h:24-60, Kernel.cpp:76-190)."""

    GAUSSIAN = capi.GAUSSIAN
    SINGULAR = capi.SINGULAR
    GAUSSIAN_MULTIPLE = capi.GAUSSIAN_MULTIPLE

    def __init__(self):
        # Kernel::Kernel(), Kernel.cpp:76-79
        self.type = Kernel.GAUSSIAN
        self.sigma = 2.0
        self.exponent = 1.0
        self.constant_shift = 0.0
        self.sigmas: list[float] = []
        self.fixedSigmas: list[float] = []
        self.beginningSigma = 0.0
        self.factor = 0.0
        self.nbOfComputedSigmas = 1

    def copy(self) -> "Kernel":
        k = Kernel()
        k.__dict__.update({key: (list(v) if isinstance(v, list) else v) for key, v in self.__dict__.items()})
        return k

    def updateSigmas(self, computedSigmas: bool = True, radius: float = 1.0) -> None:
        """Kernel::updateSigmas (Kernel.cpp:172-190), float arithmetic."""
        f32 = np.float32
        if computedSigmas:
            s = [f32(self.beginningSigma)]
            for _ in range(1, self.nbOfComputedSigmas):
                s.append(f32(s[-1] * f32(self.factor)))
            self.sigmas = [float(v) for v in s]
        else:
            self.sigmas = list(self.fixedSigmas)
        self.sigma = float(f32(self.sigma) * f32(radius))
        self.sigmas = [float(f32(v) * f32(radius)) for v in self.sigmas]

    def w(self, p, eta) -> float:
        """Kernel::w (Kernel.cpp:64-83), evaluated in double on the host."""
        d2 = float(sum((float(a) - float(b)) ** 2 for a, b in zip(p, eta)))
        if self.type == Kernel.GAUSSIAN_MULTIPLE:
            s = sum(math.exp(-d2 / (2.0 * sg * sg)) / (sg * sg * sg) for sg in self.sigmas)
            return s if s != 0 else self.constant_shift
        if self.type == Kernel.GAUSSIAN:
            return math.exp(-d2 / (2.0 * self.sigma * self.sigma)) + self.constant_shift
        if self.type == Kernel.SINGULAR:
            v = max(self.constant_shift, 1e-4)
            return v**self.exponent / (d2 + self.constant_shift) ** self.exponent
        return 1.0

    def to_c(self) -> capi.mlods_kernel:
        """The C kernel value.  Sigma lists longer than the inline array
        (the reference's files go up to 30 terms) travel through
        ``sigmas_ext``; the array is kept alive on the returned structure."""
        k = capi.mlods_kernel()
        k.type = int(self.type)
        k.sigma = float(self.sigma)
        k.exponent = float(self.exponent)
        k.constant_shift = float(self.constant_shift)
        k.n_sigmas = len(self.sigmas)
        if len(self.sigmas) > capi.INLINE_SIGMAS:
            ext = (C.c_float * len(self.sigmas))(*[float(s) for s in self.sigmas])
            k._sigmas_keepalive = ext
            k.sigmas_ext = C.cast(ext, C.POINTER(C.c_float))
        else:
            for i, s in enumerate(self.sigmas):
                k.sigmas[i] = float(s)
        return k


class APSSOctree:
    """Device-resident octree with per-node weighted moments (CPUUtils.h:166-229)."""

    def __init__(self):
        self._h = C.c_void_p(0)
        self._lib = capi.load()
        self.m_scalingProtectionSphere = 2.0  # CPUUtils.h:206
        self.m_minDepth = 0
        self.m_knnMode = False
        self.m_knn = 20
        self.m_ballMode = False
        self.m_ballRadius = 0.1
        self._info = None

    # -- lifetime
    def build(self, points, normals, updateRootBoundingBox: bool = True, maxDepth: int = 12,
              maxNumberOfPointsPerLeaf: int = 1, stream=None) -> None:
        """APSSOctree::build (CPUUtils.cpp:540-569), on the device."""
        if not updateRootBoundingBox:
            raise ValueError("a fixed root box is not supported (the reference never uses it)")
        if maxNumberOfPointsPerLeaf != 1:
            raise ValueError("only one point per leaf is supported (the reference's only setting)")
        pts = _f32x3(points, "points")
        nrm = _f32x3(normals, "normals")
        if len(pts) != len(nrm) or len(pts) == 0:
            raise ValueError("points and normals must be non-empty and of equal length")
        self.free()
        h = C.c_void_p(0)
        capi.check(self._lib.mlods_tree_build(capi.ptr(pts), capi.ptr(nrm), len(pts), int(maxDepth),
                                              C.c_void_p(stream or 0), C.byref(h)))
        self._h = h
        self._info = None
        self._host = (pts, nrm)  # the reference keeps m_points / m_normals on the host too

    def build_device(self, d_points, d_normals, maxDepth: int = 12, stream=None) -> None:
        """Build from device tensors (torch CUDA float32, shape (n, 3))."""
        self.free()
        h = C.c_void_p(0)
        capi.check(self._lib.mlods_tree_build_device(capi.ptr(d_points), capi.ptr(d_normals), int(d_points.shape[0]),
                                                     int(maxDepth), C.c_void_p(stream or 0), C.byref(h)))
        self._host = None
        self._h = h
        self._info = None

    def free(self) -> None:
        if self._h:
            self._lib.mlods_tree_free(self._h)
            self._h = C.c_void_p(0)

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass

    @property
    def handle(self) -> C.c_void_p:
        if not self._h:
            raise RuntimeError("tree not built")
        return self._h

    # -- queries
    def info(self) -> capi.mlods_tree_info:
        if self._info is None:
            inf = capi.mlods_tree_info()
            capi.check(self._lib.mlods_tree_get_info(self.handle, C.byref(inf)))
            self._info = inf
        return self._info

    def getBoundingBox(self):
        inf = self.info()
        return np.array(inf.bbox_min[:], np.float32), np.array(inf.bbox_max[:], np.float32)

    def radius(self) -> float:
        """BBOX::radius of the root box, float arithmetic (CPUUtils.h:85)."""
        bb, BB = self.getBoundingBox()
        d = (BB - bb).astype(np.float32)
        d2 = np.float32(np.float32(d[0] * d[0] + d[1] * d[1]) + d[2] * d[2])
        return float(np.float32(np.sqrt(d2)) / np.float32(2.0))

    def nbOfNodes(self) -> int:
        return int(self.info().n_nodes)

    def computeDepth(self) -> int:
        return int(self.info().depth)

    def numTies(self) -> int:
        return int(self.info().n_ties)

    def getScalingProtectionSphere(self) -> float:
        return self.m_scalingProtectionSphere

    def setScalingProtectionSphere(self, val: float) -> None:
        self.m_scalingProtectionSphere = float(val)

    def getMinDepth(self) -> int:
        return self.m_minDepth

    def setMinDepth(self, val: int) -> None:
        self.m_minDepth = int(val)

    def knnMode(self, setMode: bool, knn: int = 20) -> None:
        """CPUUtils.cpp:674-680."""
        self.m_knnMode = bool(setMode)
        if self.m_knnMode:
            self.m_ballMode = False
        self.m_knn = int(knn)

    def ballMode(self, setMode: bool, ballRadius: float = 0.1) -> None:
        """CPUUtils.cpp:682-688."""
        self.m_ballMode = bool(setMode)
        if self.m_ballMode:
            self.m_knnMode = False
        self.m_ballRadius = float(ballRadius)

    def isAPSS(self) -> bool:
        return self.m_knnMode or self.m_ballMode

    def knearest(self, queries, k: int):
        """k nearest neighbours of host queries (kdTree::knearest semantics,
        kdTreeNN.h:590-600): (indices int32 (n, k), squared distances float32)."""
        import torch

        q = torch.from_numpy(_f32x3(queries, "queries")).cuda()
        idx = torch.empty((len(q), k), dtype=torch.int32, device=q.device)
        d2 = torch.empty((len(q), k), dtype=torch.float32, device=q.device)
        capi.check(self._lib.mlods_knn(self.handle, len(q), capi.ptr(q), int(k), capi.ptr(idx), capi.ptr(d2),
                                       C.c_void_p(torch.cuda.current_stream().cuda_stream)))
        torch.cuda.current_stream().synchronize()
        return idx.cpu().numpy(), d2.cpu().numpy()

    def cpuSphere(self, qStart, kernel: Kernel | None = None):
        """APSSOctree::cpuSphere (CPUUtils.cpp:638-663): the algebraic sphere
        u0 + u123.x + u4 |x|^2 fitted to the m_knn nearest points of qStart
        with weights kernel.w (unweighted by area), summed in float in world
        coordinates as the reference does.  Returns (u0, u123, u4).  Needs
        the host arrays given to build()."""
        host = getattr(self, "_host", None)
        if host is None:
            raise ValueError("cpuSphere needs a tree built from host arrays (build, not build_device)")
        kernel = kernel or Kernel()
        q = np.asarray(qStart, np.float32).reshape(3)
        idx, _ = self.knearest(q.reshape(1, 3), int(self.m_knn))
        f = np.float32
        s_pn, s_pp, s_w = f(0), f(0), f(0)
        s_p = np.zeros(3, np.float32)
        s_n = np.zeros(3, np.float32)
        for i in idx[0]:
            if i < 0:
                continue
            p = host[0][i]
            n = host[1][i]
            wi = f(kernel.w(p, q))
            s_pn = f(s_pn + f(wi * f(np.dot(p, n))))
            s_pp = f(s_pp + f(wi * f(np.dot(p, p))))
            s_p = (s_p + wi * p).astype(np.float32)
            s_n = (s_n + wi * n).astype(np.float32)
            s_w = f(s_w + wi)
        u4 = f(0.5 * (s_pn - f(np.dot(s_p, (s_n / s_w).astype(np.float32))))
               / (s_pp - f(np.dot(s_p, (s_p / s_w).astype(np.float32)))))
        u123 = ((s_n - f(2) * u4 * s_p) / s_w).astype(np.float32)
        u0 = f(-(f(np.dot(s_p, u123)) + u4 * s_pp) / s_w)
        return float(u0), u123, float(u4)

    def getKnn(self, x, k: int):
        """APSSOctree::getKnn (CPUUtils.cpp:665-672): the k nearest points of x."""
        idx, _ = self.knearest(np.asarray(x, np.float32).reshape(1, 3), k)
        return idx[0]

    def export(self) -> dict:
        """Topology and moments in breadth-first order (see mlods_tree_export)."""
        inf = self.info()
        nn, n = int(inf.n_nodes), int(inf.n_points)
        out = {
            "depth": np.empty(nn, np.int32), "parent": np.empty(nn, np.int32),
            "first_child": np.empty(nn, np.int32), "n_children": np.empty(nn, np.int32),
            "next_brother": np.empty(nn, np.int32), "leaf_off": np.empty(nn, np.int32),
            "leaf_cnt": np.empty(nn, np.int32), "perm": np.empty(n, np.int32),
            "bmin": np.empty((nn, 3), np.float32), "bmax": np.empty((nn, 3), np.float32),
            "mom": np.empty((nn, 9), np.float64), "area": np.empty(n, np.float32),
        }
        keys = ["depth", "parent", "first_child", "n_children", "next_brother", "leaf_off", "leaf_cnt", "perm",
                "bmin", "bmax", "mom", "area"]
        capi.check(self._lib.mlods_tree_export(self.handle, *[capi.ptr(out[k]) for k in keys]))
        return out


def _cuda_available() -> bool:
    try:
        import torch

        return bool(torch.cuda.is_available())
    except Exception:
        return False


class DCGrid:
    """Dual-contouring cell grid.  ``cells`` is an int32 (n, 4) array of
    (depth, x, y, z) in sorted_octree order, ``max_depth`` the deepest level
    and ``xform`` the 3x4 map from the grid's unit frame to the tree's frame
    (new2bbox, scene.cpp:1311).

    ``DCGrid(points, max_depth)`` is the grid on the input points
    (OctreeGenerator::generateFromPoints + uniformizeFromPoints,
    upsample.cpp:128-144, :253-260; the ``-b`` mode), its set work on the
    GPU when one is present (``device=None``), else on the host; points may
    be a CUDA tensor;
    ``DCGrid.adaptive(apss, max_depth)`` the projection-driven grid of the
    default mode (OctreeGenerator::generate + uniformize, upsample.cpp:228-273).
    """

    def __init__(self, points=None, max_depth: int = 0, box_min=(-1.0, -1.0, -1.0), box_max=(1.0, 1.0, 1.0),
                 _handle=None, device: bool | None = None, stream=None):
        self._lib = capi.load()
        if _handle is None:
            on_gpu = getattr(points, "is_cuda", False)
            if device is None:
                device = on_gpu or _cuda_available()
            if on_gpu:
                pts = points.detach().to(dtype=__import__("torch").float32).reshape(-1, 3).contiguous()
                if not device:
                    pts = pts.cpu().numpy()
            else:
                pts = _f32x3(points, "points")
            bmin = np.asarray(box_min, np.float32)
            bmax = np.asarray(box_max, np.float32)
            g = C.c_void_p(0)
            if device:
                capi.check(self._lib.mlods_dcgrid_from_points_device(capi.ptr(pts), len(pts), int(max_depth),
                                                                     capi.ptr(bmin), capi.ptr(bmax),
                                                                     C.c_void_p(stream or 0), C.byref(g)))
            else:
                capi.check(self._lib.mlods_dcgrid_from_points(capi.ptr(pts), len(pts), int(max_depth),
                                                              capi.ptr(bmin), capi.ptr(bmax), C.byref(g)))
        else:
            g = _handle
        self._g = g
        n = C.c_int64(0)
        d = C.c_int32(0)
        capi.check(self._lib.mlods_dcgrid_info(g, C.byref(n), C.byref(d)))
        self.cells = np.empty((n.value, 4), np.int32)
        if n.value:
            capi.check(self._lib.mlods_dcgrid_cells(g, capi.ptr(self.cells)))
        self.max_depth = int(d.value)
        self.xform = np.empty((3, 4), np.float32)
        npj = C.c_int64(0)
        capi.check(self._lib.mlods_dcgrid_xform(g, capi.ptr(self.xform), C.byref(npj)))
        self.n_projected = int(npj.value)

    @classmethod
    def adaptive(cls, apss: "APSS", max_depth: int, cut: bool = False, stream=None) -> "DCGrid":
        apss._sync_params()
        lib = capi.load()
        g = C.c_void_p(0)
        capi.check(lib.mlods_dcgrid_adaptive(apss.m_apssOctree.handle, int(max_depth), 1 if cut else 0,
                                             C.c_void_p(stream or 0), C.byref(g)))
        return cls(_handle=g)

    def __del__(self):
        try:
            if getattr(self, "_g", None):
                self._lib.mlods_dcgrid_free(self._g)
                self._g = None
        except Exception:
            pass


def _mesh_arrays(lib, m, pinned: bool = False):
    nv = C.c_int64(0)
    nt = C.c_int64(0)
    capi.check(lib.mlods_mesh_info(m, C.byref(nv), C.byref(nt)))
    if pinned:  # page-locked host memory: the device-to-host copy runs at link speed
        import torch

        v = torch.empty((nv.value, 3), dtype=torch.float32, pin_memory=True).numpy()
        n = torch.empty((nv.value, 3), dtype=torch.float32, pin_memory=True).numpy()
        t = torch.empty((nt.value, 3), dtype=torch.int32, pin_memory=True).numpy().view(np.uint32)
    else:
        v = np.empty((nv.value, 3), np.float32)
        n = np.empty((nv.value, 3), np.float32)
        t = np.empty((nt.value, 3), np.uint32)
    capi.check(lib.mlods_mesh_get(m, capi.ptr(v), capi.ptr(n), capi.ptr(t)))
    return v, n, t


class _DeviceView:
    """__cuda_array_interface__ of an array owned by the library."""

    def __init__(self, ptr: int, shape, typestr: str, owner):
        self._owner = owner  # keeps the mesh alive while the view exists
        self.__cuda_array_interface__ = {"shape": tuple(shape), "typestr": typestr, "data": (int(ptr), False),
                                         "version": 3, "strides": None, "stream": None}


class Mesh:
    """A triangle mesh held by the library (positions, normals, uint32
    triangles): dual-contouring output and the refinement steps of
    scene::computeDualContouring (scene.cpp:1396-1452)."""

    def __init__(self, handle):
        self._lib = capi.load()
        self._m = handle

    @classmethod
    def extract(cls, cells, corner_f, cell_vertex) -> "Mesh":
        """dual_contour::extract over a grid's cells from their corner values
        and per-cell vertices (host only)."""
        lib = capi.load()
        cells = np.ascontiguousarray(np.asarray(cells, np.int32).reshape(-1, 4))
        cf = np.ascontiguousarray(np.asarray(corner_f, np.float32).reshape(-1, 8))
        vx = np.ascontiguousarray(np.asarray(cell_vertex, np.float32).reshape(-1, 3))
        if len(cf) != len(cells) or len(vx) != len(cells):
            raise ValueError("corner_f and cell_vertex need one row per cell")
        m = C.c_void_p(0)
        capi.check(lib.mlods_dc_extract(len(cells), capi.ptr(cells), capi.ptr(cf), capi.ptr(vx), C.byref(m)))
        return cls(m)

    def arrays(self, pinned: bool = False):
        """(vertices (n, 3), normals (n, 3), triangles (m, 3) uint32) as host
        arrays; pinned=True copies into page-locked memory."""
        return _mesh_arrays(self._lib, self._m, pinned)

    def device_arrays(self):
        """The mesh of APSS.dc_mesh in device memory, without a copy: torch
        CUDA tensors (vertices (n, 3) float32, normals (n, 3) float32,
        triangles (m, 3) int32 holding the uint32 indices), valid while this
        mesh is alive and unchanged."""
        import torch

        nv = C.c_int64(0)
        nt = C.c_int64(0)
        capi.check(self._lib.mlods_mesh_info(self._m, C.byref(nv), C.byref(nt)))
        pv, pn, pt = C.c_void_p(0), C.c_void_p(0), C.c_void_p(0)
        capi.check(self._lib.mlods_mesh_device_arrays(self._m, C.byref(pv), C.byref(pn), C.byref(pt)))
        out = []
        for p, shape, ts in ((pv, (nv.value, 3), "<f4"), (pn, (nv.value, 3), "<f4"), (pt, (nt.value, 3), "<i4")):
            if shape[0] == 0:
                out.append(torch.empty(shape, dtype=torch.float32 if ts == "<f4" else torch.int32, device="cuda"))
            else:
                out.append(torch.as_tensor(_DeviceView(p.value, shape, ts, self), device="cuda"))
        return tuple(out)

    def stage_ms(self) -> dict:
        """Host time of the pipeline stages of APSS.dc_mesh (ms)."""
        ms = np.zeros(7, np.float64)
        capi.check(self._lib.mlods_mesh_stage_ms(self._m, capi.ptr(ms)))
        names = ("corner_field", "extract", "upload", "project", "smooth", "subdivide", "download")
        return {k: float(v) for k, v in zip(names, ms)}

    def transform(self, xform) -> None:
        x = np.ascontiguousarray(np.asarray(xform, np.float32).reshape(3, 4))
        capi.check(self._lib.mlods_mesh_transform(self._m, capi.ptr(x)))

    def smooth(self) -> None:
        capi.check(self._lib.mlods_mesh_smooth(self._m))

    def subdivide(self) -> None:
        capi.check(self._lib.mlods_mesh_subdivide(self._m))

    def project(self, apss: "APSS", n_iterations: int = 3, stream=None) -> None:
        apss._sync_params()
        capi.check(self._lib.mlods_mesh_project(apss.m_apssOctree.handle, self._m, int(n_iterations),
                                                C.c_void_p(stream or 0)))

    def __del__(self):
        try:
            if getattr(self, "_m", None):
                self._lib.mlods_mesh_free(self._m)
                self._m = None
        except Exception:
            pass


def unit2bbox(box_min=(-1.0, -1.0, -1.0), box_max=(1.0, 1.0, 1.0)) -> np.ndarray:
    """3x4 map from the unit cube to the octree zone box (scene.cpp:1257-1269)."""
    bmin = np.asarray(box_min, np.float32)
    d = (np.asarray(box_max, np.float32) - bmin).astype(np.float32)
    m = np.zeros((3, 4), np.float32)
    for a in range(3):
        m[a, a] = d[a]
        m[a, 3] = bmin[a]
    return m


class APSS:
    """Projection interface (GPUUtils.h:22-67) over a device octree."""

    mode = capi.MODE_MLOD

    def __init__(self, apssOctree: APSSOctree, kernel: Kernel | None = None, nbOfVectors: int = 0):
        self.m_apssOctree = apssOctree
        self._lib = capi.load()
        self.m_scalingProtectionSphere = 2.0  # GPUUtils.h:63
        self.m_minDepth = 0
        self.blend_rule = capi.BLEND_GPU
        self.reorder = True
        self.prune_tol = 0.0
        self.converge = capi.CONVERGE_OFF
        self.converge_tol = 0.0
        self.local_output = False  # extension: results relative to the tree's origin (non in-place calls)
        self.queries_per_warp = 1  # extension: the walk schedule (1 or 2 queries per warp)
        self._n_uploaded = 0
        q = C.c_void_p(0)
        capi.check(self._lib.mlods_queries_create(C.byref(q)))
        self._q = q  # the device query buffer this object owns (APSS::m_outPts, GPUUtils.h:56)
        if kernel is not None:
            self.copyToGPU(kernel, nbOfVectors)

    def __del__(self):
        try:
            if getattr(self, "_q", None):
                self._lib.mlods_queries_destroy(self._q)
                self._q = None
        except Exception:
            pass

    def _params(self) -> capi.mlods_params:
        p = capi.mlods_params()
        self._lib.mlods_default_params(C.byref(p))
        t = self.m_apssOctree
        p.cutoff = float(self.m_scalingProtectionSphere)
        p.min_depth = int(self.m_minDepth)
        p.mode = int(self._mode())
        p.knn = int(t.m_knn)
        p.ball_radius = float(t.m_ballRadius)
        p.blend_rule = int(self.blend_rule)
        p.reorder = 1 if self.reorder else 0
        p.prune_tol = float(self.prune_tol)
        p.converge = int(self.converge)
        p.converge_tol = float(self.converge_tol)
        p.local_output = 1 if self.local_output else 0
        p.queries_per_warp = int(self.queries_per_warp)
        return p

    def _mode(self) -> int:
        t = self.m_apssOctree
        if t.m_knnMode:
            return capi.MODE_KNN
        if t.m_ballMode:
            return capi.MODE_BALL
        return self.mode

    def _sync_params(self) -> None:
        p = self._params()
        capi.check(self._lib.mlods_set_params(self.m_apssOctree.handle, C.byref(p)))

    # -- GPUUtils.h:29-51
    def copyToGPU(self, kernel: Kernel, nbOfVectors: int = 0) -> None:
        self.updateKernel(kernel)

    def updateKernel(self, kernel: Kernel) -> None:
        k = kernel.to_c()
        capi.check(self._lib.mlods_set_kernel(self.m_apssOctree.handle, C.byref(k)))

    def eraseFromGPU(self) -> None:
        self.erasePointsFromGPU()

    def copyPointsToGPU(self, nbOfVectors: int, outputPoints) -> None:
        pts = _f32x3(outputPoints, "points")[:nbOfVectors]
        capi.check(self._lib.mlods_queries_upload(self._q, int(nbOfVectors), capi.ptr(pts), C.c_void_p(0)))
        self._n_uploaded = int(nbOfVectors)

    def erasePointsFromGPU(self) -> None:
        capi.check(self._lib.mlods_queries_free(self._q))
        self._n_uploaded = 0

    def reorganizePoints(self, invalidPts, endValid: int) -> None:
        """APSS::reorganizePoints (GPUUtils.cu:503-517)."""
        inv = np.ascontiguousarray(np.asarray(invalidPts, np.uint32))
        capi.check(self._lib.mlods_queries_reorganize(self._q, len(inv), capi.ptr(inv), int(endValid),
                                                      C.c_void_p(0)))

    def project(self, nbOfVectors: int, outputPoints, outputNormals, n_iterations: int, kernel: Kernel | None = None,
                stepMaxSize: float = -1.0) -> None:
        """Fastapss::project (Fastapss.cu:439-455): iterate in place on the device
        buffer, copy back into the given float32 (n, 3) arrays when not None.
        As in the reference, ``kernel`` is ignored: the device kernel is the
        one from copyToGPU/updateKernel."""
        self._sync_params()
        op = outputPoints if outputPoints is not None else None
        on = outputNormals if outputNormals is not None else None
        for a in (op, on):
            if a is not None and (a.dtype != np.float32 or not a.flags.c_contiguous or a.shape[0] < nbOfVectors):
                raise ValueError("output arrays must be C-contiguous float32 with at least n rows")
        capi.check(self._lib.mlods_project(self.m_apssOctree.handle, self._q, int(nbOfVectors), int(n_iterations),
                                           float(stepMaxSize), capi.ptr(op), capi.ptr(on), C.c_void_p(0)))

    def projectCPU(self, qStart, n_iterations: int, kernel: Kernel | None = None, stepMaxSize: float = -1.0):
        """APSSOctree::projectCPU semantics (CPU blend rule, CPUUtils.cpp:621-636)
        for one query or an (n, 3) array, evaluated on the device without
        touching the query buffer: (points, normals).  Re-entrant: host threads
        may call it at once on one tree."""
        self._sync_params()
        q = np.ascontiguousarray(np.asarray(qStart, np.float32).reshape(-1, 3))
        op = np.empty_like(q)
        on = np.empty_like(q)
        capi.check(self._lib.mlods_project_host(self.m_apssOctree.handle, len(q), capi.ptr(q), capi.ptr(op),
                                                capi.ptr(on), int(n_iterations), float(stepMaxSize),
                                                capi.BLEND_CPU, C.c_void_p(0)))
        if np.ndim(qStart) == 1:
            return op[0], on[0]
        return op, on

    def project_device(self, d_q, d_out_p, d_out_n, n_iterations: int, stepMaxSize: float = -1.0,
                       stream=None) -> None:
        """Device-buffer projection (torch CUDA tensors), asynchronous."""
        self._sync_params()
        capi.check(self._lib.mlods_project_device(self.m_apssOctree.handle, int(d_q.shape[0]), capi.ptr(d_q),
                                                  capi.ptr(d_out_p), capi.ptr(d_out_n), int(n_iterations),
                                                  float(stepMaxSize), C.c_void_p(stream or 0)))

    def tune_schedule(self, d_q, n_iterations: int, stream=None) -> dict:
        """mlods_tune_schedule: times the walk schedules on the device queries
        d_q (torch CUDA float32 (n, 3)) and keeps the fastest as this
        object's queries_per_warp.  Returns {"queries_per_warp": q, "ms": {1: .., 2: .., 4: ..}}."""
        self._sync_params()
        chosen = C.c_int32(0)
        ms = (C.c_float * 3)()
        capi.check(self._lib.mlods_tune_schedule(self.m_apssOctree.handle, int(d_q.shape[0]), capi.ptr(d_q),
                                                 int(n_iterations), C.c_void_p(stream or 0), C.byref(chosen), ms))
        self.queries_per_warp = int(chosen.value)
        return {"queries_per_warp": int(chosen.value), "ms": {w: float(m) for w, m in zip((1, 2, 4), ms)}}

    def dc_evaluate(self, cells, max_depth: int, xform=None, use_normals: bool = False):
        """Corner field and per-cell vertex of a DC grid (scene.cpp:1346-1394,
        dual_contouring.h:124-176): (corner_f (n, 8), vertex (n, 3) in the unit
        cube, n_cross (n,), number of unique corners projected)."""
        self._sync_params()
        cells = np.ascontiguousarray(np.asarray(cells, np.int32).reshape(-1, 4))
        xf = np.ascontiguousarray(unit2bbox() if xform is None else np.asarray(xform, np.float32).reshape(3, 4))
        n = len(cells)
        cf = np.empty((n, 8), np.float32)
        vx = np.empty((n, 3), np.float32)
        nc = np.empty(n, np.int32)
        nu = C.c_int64(0)
        capi.check(self._lib.mlods_dc_evaluate(self.m_apssOctree.handle, n, capi.ptr(cells), int(max_depth),
                                               capi.ptr(xf), 1 if use_normals else 0, capi.ptr(cf), capi.ptr(vx),
                                               capi.ptr(nc), C.byref(nu), C.c_void_p(0)))
        return cf, vx, nc, nu.value

    def dc_evaluate_device(self, d_cells, max_depth: int, xform=None, use_normals: bool = False, stream=None):
        """dc_evaluate with the cells (an (n, 4) int32 CUDA tensor) and the
        results in device memory: (corner_f (n, 8), vertex (n, 3), n_cross
        (n,) as CUDA tensors, number of unique corners projected)."""
        import torch

        self._sync_params()
        cells = d_cells.reshape(-1, 4)
        if cells.dtype != torch.int32 or not cells.is_cuda or not cells.is_contiguous():
            raise ValueError("cells must be a contiguous int32 CUDA tensor of shape (n, 4)")
        xf = np.ascontiguousarray(unit2bbox() if xform is None else np.asarray(xform, np.float32).reshape(3, 4))
        n = cells.shape[0]
        cf = torch.empty((n, 8), dtype=torch.float32, device=cells.device)
        vx = torch.empty((n, 3), dtype=torch.float32, device=cells.device)
        nc = torch.empty((n,), dtype=torch.int32, device=cells.device)
        nu = C.c_int64(0)
        s = stream if stream is not None else torch.cuda.current_stream(cells.device).cuda_stream
        capi.check(self._lib.mlods_dc_evaluate_device(self.m_apssOctree.handle, n, capi.ptr(cells), int(max_depth),
                                                      capi.ptr(xf), 1 if use_normals else 0, capi.ptr(cf),
                                                      capi.ptr(vx), capi.ptr(nc), C.byref(nu), C.c_void_p(s)))
        return cf, vx, nc, nu.value

    def dc_mesh(self, grid: DCGrid, use_normals: bool = False, refine_rounds: int = 2, stream=None) -> Mesh:
        """scene::computeDualContouring's mesh (scene.cpp:1346-1452): corner
        field, extraction, transform to the tree's frame, projection, then
        refine_rounds x (smooth, subdivide, project)."""
        self._sync_params()
        m = C.c_void_p(0)
        capi.check(self._lib.mlods_dc_mesh(self.m_apssOctree.handle, grid._g, 1 if use_normals else 0,
                                           int(refine_rounds), C.c_void_p(stream or 0), C.byref(m)))
        return Mesh(m)

    def last_stats(self):
        v = C.c_int64(0)
        r = C.c_int64(0)
        m = C.c_int32(0)
        o = C.c_int64(0)
        ms = C.c_float(0)
        capi.check(self._lib.mlods_last_stats(self.m_apssOctree.handle, C.byref(v), C.byref(r), C.byref(m),
                                              C.byref(o), C.byref(ms)))
        it = C.c_int64(0)
        capi.check(self._lib.mlods_last_iterations(self.m_apssOctree.handle, C.byref(it)))
        lv = C.c_int64(0)
        pr = C.c_int64(0)
        capi.check(self._lib.mlods_last_walk_counts(self.m_apssOctree.handle, C.byref(lv), C.byref(pr)))
        return {"node_visits": v.value, "rounds": r.value, "max_stack": m.value, "overflows": o.value,
                "kernel_ms": ms.value, "iterations": it.value, "lane_visits": lv.value, "pruned": pr.value}

    # -- options, GPUUtils.h:40-43
    def setScalingProtectionSphere(self, val: float) -> None:
        self.m_scalingProtectionSphere = float(val)
        self.m_apssOctree.setScalingProtectionSphere(val)

    def getScalingProtectionSphere(self) -> float:
        return self.m_scalingProtectionSphere

    def setMinDepth(self, val: int) -> None:
        self.m_minDepth = int(val)
        self.m_apssOctree.setMinDepth(val)

    def getMinDepth(self) -> int:
        return self.m_minDepth

    def CPU(self) -> APSSOctree:
        return self.m_apssOctree

    def cpuSphere(self, qStart, kernel: Kernel | None = None):
        """GlobalAPSS::cpuSphere (GlobalAPSS.cu:288-291): the octree's."""
        return self.m_apssOctree.cpuSphere(qStart, kernel)

    def stop(self) -> None:
        """APSS::stop (GPUUtils.cu:394-397) ends a CUDA profiler range in the
        reference; nothing to stop here."""

    def eraseAndRestart(self) -> None:
        """APSS::eraseAndRestart (GPUUtils.cu:399-404): drops the device data
        and starts over with an empty octree (build it again before use)."""
        self.eraseFromGPU()
        self.m_apssOctree = APSSOctree()


class Fastapss(APSS):
    """MLoD projection (Fastapss.h:32-51)."""

    mode = capi.MODE_MLOD


class GlobalAPSS(APSS):
    """APSS over every point, no level of detail (GlobalAPSS.h:19-43)."""

    mode = capi.MODE_GLOBAL


class FastapssBatch:
    """Many resident Fastapss objects projected in one kernel launch.

    No counterpart in the reference (one ``Fastapss::project`` launch per tree,
    Fastapss.cu:439-455).  ``projectors`` are :class:`Fastapss` objects whose
    kernel has been set; each keeps its own settings (cutoff, min depth, blend
    rule, convergence mode).  :meth:`project_device` takes one concatenated
    device query buffer (torch CUDA tensors, float32 (n, 3)) and the per-tree
    query counts, and gives results identical to one ``project_device`` call
    per tree.  The projectors must outlive the batch.
    """

    def __init__(self, projectors):
        self._lib = capi.load()
        self._projectors = list(projectors)
        if not self._projectors:
            raise ValueError("need at least one projector")
        for p in self._projectors:
            if p._mode() != capi.MODE_MLOD:
                raise ValueError("batched projection supports the MLoD mode only")
        handles = (C.c_void_p * len(self._projectors))(*[p.m_apssOctree.handle.value for p in self._projectors])
        b = C.c_void_p(0)
        capi.check(self._lib.mlods_batch_create(handles, len(self._projectors), C.byref(b)))
        self._b = b

    def __del__(self):
        try:
            if getattr(self, "_b", None):
                self._lib.mlods_batch_free(self._b)
                self._b = None
        except Exception:
            pass

    def _offsets(self, counts) -> np.ndarray:
        counts = np.asarray(counts, np.int64)
        if counts.shape != (len(self._projectors),) or (counts < 0).any():
            raise ValueError("counts must give one non-negative count per projector")
        return np.ascontiguousarray(np.concatenate([[0], np.cumsum(counts)]).astype(np.int64))

    def project_device(self, counts, d_q, d_out_p, d_out_n, n_iterations: int, use_graph: bool = False,
                       stream=None) -> None:
        for p in self._projectors:
            p._sync_params()
        off = self._offsets(counts)
        capi.check(self._lib.mlods_batch_project(self._b, capi.ptr(off), capi.ptr(d_q), capi.ptr(d_out_p),
                                                 capi.ptr(d_out_n), int(n_iterations), 1 if use_graph else 0,
                                                 C.c_void_p(stream or 0)))

    def tune(self, counts, d_q, d_out_p, d_out_n, n_iterations: int, stream=None) -> None:
        for p in self._projectors:
            p._sync_params()
        off = self._offsets(counts)
        capi.check(self._lib.mlods_batch_tune(self._b, capi.ptr(off), capi.ptr(d_q), capi.ptr(d_out_p),
                                              capi.ptr(d_out_n), int(n_iterations), C.c_void_p(stream or 0)))

    @staticmethod
    def _schedule_dict(sc) -> dict:
        return {"queries_per_warp": sc.queries_per_warp, "reorder": sc.reorder, "grid_pct": sc.grid_pct,
                "line_order": "by specialisation" if sc.line_order == 1 else "most work first",
                "solo_min_queries": sc.solo_min_queries}

    def schedule(self) -> dict:
        """The launch shape in use: walk schedule (queries per warp), Morton
        order (reorder), share of the grid, order of the trees in the launch,
        and the size from which a tree runs in a launch of its own (0: none)."""
        sc = capi.mlods_batch_schedule()
        capi.check(self._lib.mlods_batch_get_schedule(self._b, C.byref(sc)))
        return self._schedule_dict(sc)

    def last_stats(self):
        """Statistics of the last call, with the schedule it ran."""
        v = C.c_int64(0)
        r = C.c_int64(0)
        o = C.c_int64(0)
        ms = C.c_float(0)
        lv = C.c_int64(0)
        nl = C.c_int32(0)
        capi.check(self._lib.mlods_batch_stats(self._b, C.byref(v), C.byref(r), C.byref(o), C.byref(ms),
                                               C.byref(lv), C.byref(nl)))
        out = {"node_visits": v.value, "rounds": r.value, "overflows": o.value, "kernel_ms": ms.value,
               "lane_visits": lv.value, "walk_launches": nl.value}
        out.update(self.schedule())
        return out

    def set_schedule(self, queries_per_warp: int = 0, reorder: bool = True, grid_pct: int = 100,
                     by_specialisation: bool = False, solo_min_queries: int = 0) -> None:
        """Sets the launch shape without tuning (see :meth:`schedule`)."""
        sc = capi.mlods_batch_schedule(int(queries_per_warp), 1 if reorder else 0, int(grid_pct),
                                       1 if by_specialisation else 0, int(solo_min_queries))
        capi.check(self._lib.mlods_batch_set_schedule(self._b, C.byref(sc)))

    def tune_results(self):
        """The candidates of the last :meth:`tune` with their device times (ms)."""
        n = C.c_int32(0)
        capi.check(self._lib.mlods_batch_tune_results(self._b, 0, None, None, C.byref(n)))
        k = n.value
        cands = (capi.mlods_batch_schedule * max(k, 1))()
        ms = (C.c_float * max(k, 1))()
        capi.check(self._lib.mlods_batch_tune_results(self._b, k, cands, ms, C.byref(n)))
        return [dict(self._schedule_dict(cands[i]), ms=ms[i]) for i in range(k)]


class ProjectionServer:
    """Asynchronous projection requests over resident trees (no counterpart
    in the reference).  ``projectors`` are :class:`Fastapss` objects with a
    kernel set; requests name one of them by index.  :meth:`submit` queues
    float32 (n, 3) host queries and returns a ticket at once; :meth:`wait`
    returns (points, normals, latency_ms) once the request has run (results
    equal ``project`` on the same tree and kernel).  Queued requests run in
    batches, one multi-tree launch per batch, on ``n_streams`` worker streams.
    """

    def __init__(self, projectors, n_streams: int = 2, max_batch_queries: int = 1 << 18,
                 max_batch_requests: int = 4096, max_device_bytes: int = 0, max_pending_bytes: int = 0,
                 max_wait_us: int = 0):
        self._lib = capi.load()
        self._projectors = list(projectors)
        for p in self._projectors:
            if p._mode() != capi.MODE_MLOD:
                raise ValueError("the server supports the MLoD mode only")
            p._sync_params()
        cfg = capi.mlods_server_config()
        self._lib.mlods_server_default_config(C.byref(cfg))
        cfg.n_streams = int(n_streams)
        cfg.max_batch_queries = int(max_batch_queries)
        cfg.max_batch_requests = int(max_batch_requests)
        cfg.max_device_bytes = int(max_device_bytes)
        cfg.max_pending_bytes = int(max_pending_bytes)
        cfg.max_wait_us = int(max_wait_us)
        handles = (C.c_void_p * len(self._projectors))(*[p.m_apssOctree.handle.value for p in self._projectors])
        s = C.c_void_p(0)
        capi.check(self._lib.mlods_server_create(handles, len(self._projectors), C.byref(cfg), C.byref(s)))
        self._s = s
        self._pending = {}

    def submit(self, tree: int, queries, n_iterations: int = 10, kernel: Kernel | None = None) -> int:
        q = _f32x3(queries, "queries")
        out_p = np.empty_like(q)
        out_n = np.empty_like(q)
        kc = C.byref(kernel.to_c()) if kernel is not None else None
        t = C.c_uint64(0)
        capi.check(self._lib.mlods_server_submit(self._s, int(tree), len(q), capi.ptr(q), capi.ptr(out_p),
                                                 capi.ptr(out_n), int(n_iterations), kc, C.byref(t)))
        self._pending[t.value] = (q, out_p, out_n)  # keep the buffers alive until wait
        return t.value

    def wait(self, ticket: int, timeout_ms: int = 60000):
        lat = C.c_double(0)
        rc = self._lib.mlods_server_wait(self._s, C.c_uint64(ticket), int(timeout_ms), C.byref(lat))
        if rc == capi.MLODS_ERR_TIMEOUT:
            raise TimeoutError(self._lib.mlods_last_error().decode(errors="replace"))
        bufs = self._pending.pop(ticket, None)
        capi.check(rc)
        return bufs[1], bufs[2], lat.value

    def stats(self):
        c, b, q, qd = C.c_int64(0), C.c_int64(0), C.c_int64(0), C.c_int64(0)
        busy = C.c_double(0)
        capi.check(self._lib.mlods_server_stats(self._s, C.byref(c), C.byref(b), C.byref(q), C.byref(qd),
                                                C.byref(busy)))
        return {"completed": c.value, "batches": b.value, "queries": q.value, "queued": qd.value,
                "busy_ms": busy.value}

    def memory(self):
        """Device bytes in flight (now, peak), footprint of the queued work and
        the two budgets (mlods_server_memory)."""
        v = [C.c_int64(0) for _ in range(5)]
        capi.check(self._lib.mlods_server_memory(self._s, *[C.byref(x) for x in v]))
        return dict(zip(("in_flight_bytes", "peak_in_flight_bytes", "pending_bytes", "max_device_bytes",
                         "max_pending_bytes"), (x.value for x in v)))

    @staticmethod
    def batch_bytes(n_queries: int, n_requests: int = 1) -> int:
        """Device bytes a batch of n_queries from n_requests holds in flight."""
        return int(capi.load().mlods_server_batch_bytes(int(n_queries), int(n_requests)))

    def close(self) -> None:
        if getattr(self, "_s", None):
            self._lib.mlods_server_free(self._s)
            self._s = None
            self._pending.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

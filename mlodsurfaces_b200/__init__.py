"""mlodsurfaces_b200 -- B200 (sm_100a) point-set surface projection.

The Moving Level-of-Detail (MLoD) and APSS projection path of
CorentinMercier/MlodSurfaces, rebuilt around hand-written CUDA kernels in
``libmlods.so`` (C ABI: ``include/mlods.h``).  This package is the Python
mirror of the reference's C++ projection API (``Kernel``, ``APSSOctree``,
``APSS``/``Fastapss``) plus seeded synthetic inputs (``synth``).
"""
from .apss import APSS, APSSOctree, DCGrid, Fastapss, FastapssBatch, GlobalAPSS, Kernel, Mesh, ProjectionServer, unit2bbox  # noqa: F401
from . import io, shard, synth  # noqa: F401


def release_scratch() -> None:
    """Return the unused memory of the library's per-call scratch pool on the
    current device (up to 8 GiB of freed scratch is kept for later calls)."""
    from . import _capi as capi

    capi.check(capi.load().mlods_release_scratch())

__all__ = ["APSS", "APSSOctree", "DCGrid", "Fastapss", "FastapssBatch", "GlobalAPSS", "Kernel", "Mesh", "ProjectionServer",
           "io", "release_scratch", "shard", "synth", "unit2bbox"]

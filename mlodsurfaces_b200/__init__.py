"""mlodsurfaces_b200 -- B200 (sm_100a) point-set surface projection.

The Moving Level-of-Detail (MLoD) and APSS projection path of
CorentinMercier/MlodSurfaces, rebuilt around hand-written CUDA kernels in
``libmlods.so`` (C ABI: ``include/mlods.h``).  This package is the Python
mirror of the reference's C++ projection API (``Kernel``, ``APSSOctree``,
``APSS``/``Fastapss``) plus seeded synthetic inputs (``synth``).
"""
from .apss import APSS, APSSOctree, DCGrid, Fastapss, FastapssBatch, GlobalAPSS, Kernel, Mesh, ProjectionServer, unit2bbox  # noqa: F401
from . import io, synth  # noqa: F401

__all__ = ["APSS", "APSSOctree", "DCGrid", "Fastapss", "FastapssBatch", "GlobalAPSS", "Kernel", "Mesh", "ProjectionServer", "io", "synth", "unit2bbox"]

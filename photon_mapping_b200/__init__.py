"""B200-native photon-mapping hot path (sm_100a CUDA behind a C ABI).

The compute path is libpm_cuda.so (include/pm_cuda.h); this package is the
host-side mirror of the reference's interface (PhotonMap and friends) over
that library, plus the build recipe and seeded synthetic workloads.
"""
from ._native import Context, PMError, PM_MAP_CAUSTICS, PM_MAP_GLOBAL, PM_MAX_K  # noqa: F401
from .photon_map import PhotonMap, radiance_queries  # noqa: F401

__all__ = ["Context", "PMError", "PhotonMap", "radiance_queries",
           "PM_MAP_GLOBAL", "PM_MAP_CAUSTICS", "PM_MAX_K"]

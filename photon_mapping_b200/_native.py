"""ctypes binding of libpm_cuda.so (the C ABI declared in include/pm_cuda.h).

The library is the only compute path: if it is missing this module raises,
there is no fallback.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

LIB_PATH = Path(__file__).resolve().parent / "_lib" / "libpm_cuda.so"
HEADER = Path(__file__).resolve().parent.parent / "include" / "pm_cuda.h"

PM_OK = 0
PM_ERR_INVALID_ARGUMENT = 1
PM_ERR_CUDA = 2
PM_ERR_OUT_OF_MEMORY = 3
PM_ERR_NOT_BUILT = 4
PM_ERR_DEVICE_STATUS = 5

PM_MAP_GLOBAL = 0
PM_MAP_CAUSTICS = 1
PM_MAX_K = 1024
PM_NOALLOC_MAX_PHOTONS = 65536

# pm_radiance_query: {px,py,pz,rho_r, wox,woy,woz,rho_g, nsx,nsy,nsz,rho_b}
RADIANCE_QUERY_FLOATS = 12


class PMError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{status_string(status)}: {msg}")
        self.status = status


_lib: C.CDLL | None = None

_i64 = C.c_int64
_vp = C.c_void_p
_fp = C.POINTER(C.c_float)
_ip = C.POINTER(C.c_int32)

_SIGNATURES = {
    "pm_ctx_create": (C.c_int, [C.c_int, C.POINTER(_vp)]),
    "pm_ctx_destroy": (C.c_int, [_vp]),
    "pm_ctx_synchronize": (C.c_int, [_vp]),
    "pm_ctx_last_error": (C.c_char_p, [_vp]),
    "pm_status_string": (C.c_char_p, [C.c_int]),
    "pm_ctx_set_stats": (C.c_int, [_vp, C.c_int]),
    "pm_ctx_get_stats": (C.c_int, [_vp, _vp, C.c_int]),
    "pm_photonmap_build": (C.c_int, [_vp, C.c_int, _vp, _i64]),
    "pm_photonmap_build_device": (C.c_int, [_vp, C.c_int, _vp, _i64, _vp]),
    "pm_photonmap_size": (C.c_int, [_vp, C.c_int, C.POINTER(_i64)]),
    "pm_photonmap_set_emitted": (C.c_int, [_vp, C.c_int, _i64]),
    "pm_photonmap_get_photons": (C.c_int, [_vp, C.c_int, _i64, _i64, _vp]),
    "pm_photonmap_knn": (C.c_int, [_vp, C.c_int, _vp, _i64, C.c_int, _vp, _vp, _vp]),
    "pm_photonmap_radiance": (C.c_int, [_vp, C.c_int, _vp, _i64, C.c_int, _i64, _vp]),
    "pm_photonmap_radiance_device": (C.c_int, [_vp, C.c_int, _vp, _i64, C.c_int, _i64, _vp, _vp]),
    "pm_scene_upload": (C.c_int, [_vp, _vp, _vp, _vp, _i64]),
    "pm_scene_intersect": (C.c_int, [_vp, _vp, _i64, _vp]),
    "pm_photons_trace": (C.c_int, [_vp, C.c_int, C.c_uint64, _i64, C.c_int, _vp]),
    "pm_render": (C.c_int, [_vp, _vp, _vp, _vp, _vp]),
    "pm_integrate": (C.c_int, [_vp, _vp, _i64, _vp, _vp, _vp]),
    "pm_path_trace_rays": (C.c_int, [_vp, _vp, _i64, _vp, C.c_int32, _vp]),
    "pm_render_path_tracing": (C.c_int, [_vp, _vp, C.c_int32, C.c_int32, C.c_int32, C.c_int32,
                                         _vp, _vp]),
    "pm_photonmap_radiance_noalloc": (C.c_int, [_vp, _i64, _vp, _i64, C.c_int, _i64, _vp, _vp]),
    "pm_diff_set_parameters": (C.c_int, [_vp, _vp, _i64, C.c_int32]),
    "pm_diff_forward": (C.c_int, [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "pm_diff_backward": (C.c_int, [_vp, _vp, _vp, _vp]),
    "pm_batch_create": (C.c_int, [C.c_int, _vp, C.c_int32, C.POINTER(_vp)]),
    "pm_batch_destroy": (C.c_int, [_vp]),
    "pm_batch_last_error": (C.c_char_p, [_vp]),
    "pm_batch_set_tuning": (C.c_int, [_vp, _vp]),
    "pm_batch_get_tuning": (C.c_int, [_vp, _vp]),
    "pm_batch_autotune": (C.c_int, [_vp, _vp, _vp]),
    "pm_batch_render": (C.c_int, [_vp, C.c_int32, _vp]),
    "pm_batch_image": (C.c_int, [_vp, C.c_int32, _vp]),
    "pm_batch_counts": (C.c_int, [_vp, _vp, _vp]),
    "pm_batch_photons": (C.c_int, [_vp, C.c_int32, _vp]),
    "pm_batch_stage_times": (C.c_int, [_vp, _vp, C.c_int32]),
}


def load(path: Path | str | None = None) -> C.CDLL:
    """Loads libpm_cuda.so (raises if it has not been built)."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = Path(path) if path else LIB_PATH
    if not p.exists():
        raise RuntimeError(
            f"{p} is missing: build it with `python -m photon_mapping_b200.build` "
            "(there is no CPU fallback)")
    lib = C.CDLL(str(p))
    for name, (res, args) in _SIGNATURES.items():
        fn = getattr(lib, name, None)
        if fn is None:
            continue
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _lib = lib
    return lib


def status_string(status: int) -> str:
    try:
        return load().pm_status_string(status).decode()
    except Exception:  # library not loadable: still give a readable name
        return f"status {status}"


def ptr(a: np.ndarray | None) -> int | None:
    if a is None:
        return None
    assert a.flags["C_CONTIGUOUS"], "arrays passed to libpm_cuda must be C-contiguous"
    return a.ctypes.data


class Context:
    """A pm_ctx: device buffers, a stream and the two photon maps."""

    def __init__(self, device: int = 0):
        self.lib = load()
        h = _vp()
        st = self.lib.pm_ctx_create(int(device), C.byref(h))
        if st != PM_OK:
            raise PMError(st, f"pm_ctx_create(device={device})")
        self.handle = h
        self.device = device

    def check(self, st: int, what: str) -> None:
        if st != PM_OK:
            msg = self.lib.pm_ctx_last_error(self.handle).decode()
            raise PMError(st, f"{what}: {msg}")

    def close(self) -> None:
        if getattr(self, "handle", None):
            self.lib.pm_ctx_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def synchronize(self) -> None:
        self.check(self.lib.pm_ctx_synchronize(self.handle), "synchronize")

    STAT_FIELDS = ("queries", "cold_starts", "candidates", "leaves", "nodes", "selects", "walks")

    def set_stats(self, enable: bool) -> None:
        self.check(self.lib.pm_ctx_set_stats(self.handle, int(bool(enable))), "pm_ctx_set_stats")

    def get_stats(self, reset: bool = False) -> dict:
        buf = (C.c_uint64 * len(self.STAT_FIELDS))()
        self.check(self.lib.pm_ctx_get_stats(self.handle, C.addressof(buf), int(reset)),
                   "pm_ctx_get_stats")
        return dict(zip(self.STAT_FIELDS, (int(v) for v in buf)))

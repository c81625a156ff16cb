"""ORACLE — test infrastructure only.

ctypes access to the CPU restatement (``_build/liboracle.so``) and to the
reference's own code compiled unchanged (``_ref/*.so``). Only tests/,
``__graft_entry__.smoke()`` and the CPU-baseline leg of bench.py use this
module; the product never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ORACLE_SO = HERE / "_build" / "liboracle.so"
REF_PM_SO = HERE / "_ref" / "libpmref_photonmap.so"
REF_INT_SO = HERE / "_ref" / "libpmref_integrator.so"

_i64, _vp = C.c_int64, C.c_void_p


def build() -> None:
    r = subprocess.run(["make", "-s", "-C", str(HERE)], capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"oracle build failed:\n{r.stdout}\n{r.stderr}")


def _load(path: Path, sigs: dict) -> C.CDLL:
    if not path.exists():
        build()
    lib = C.CDLL(str(path))
    for name, (res, args) in sigs.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


_oracle = None
_refpm = None
_refint = None


def oracle_lib() -> C.CDLL:
    global _oracle
    if _oracle is None:
        _oracle = _load(ORACLE_SO, {
            "orc_knn": (None, [_vp, _i64, _vp, _i64, C.c_int, _vp, _vp, _vp]),
            "orc_radiance_fp64": (None, [_vp, _vp, _vp, _vp, C.c_int, _vp, _i64, _i64, _vp]),
            "orc_radiance_fp32": (None, [_vp, _vp, _vp, _vp, C.c_int, _vp, _i64, _i64, _vp]),
            "orc_scene_new": (_vp, [_vp, _vp, _vp, _i64]),
            "orc_scene_free": (None, [_vp]),
            "orc_intersect": (None, [_vp, _vp, _i64, _vp]),
            "orc_trace": (_i64, [_vp, C.c_int, C.c_uint64, _i64, _i64, C.c_int, _vp, _i64, _vp]),
            "orc_sincos": (None, [_vp, _i64, _vp, _vp]),
            "orc_render": (None, [_vp, _vp, _i64, _i64, _vp, _i64, _i64, _vp, _vp, _vp, _vp]),
            "orc_render_pt": (None, [_vp, _vp, C.c_int, C.c_int, C.c_int, C.c_int, _vp, _vp]),
            "orc_integrate": (None, [_vp, _vp, _i64, _i64, _vp, _i64, _i64, _vp, _i64, _vp, _vp,
                                     _vp]),
            "orc_grad": (None, [_vp, _vp, C.c_int, C.c_uint64, _i64, _i64, _vp, _vp, _vp, _vp,
                                _vp]),
        })
    return _oracle


def ref_available() -> bool:
    return REF_PM_SO.exists()


def ref_pm_lib() -> C.CDLL:
    global _refpm
    if _refpm is None:
        _refpm = _load(REF_PM_SO, {
            "ref_pm_build": (_vp, [_vp, _i64]),
            "ref_pm_free": (None, [_vp]),
            "ref_max_threads": (C.c_int, []),
            "ref_pm_knn": (None, [_vp, _vp, _i64, C.c_int, _vp, _vp, _vp]),
            "ref_pm_radiance": (None, [_vp, _vp, _i64, C.c_int, C.c_int, _vp]),
        })
    return _refpm


def ref_integrator_available() -> bool:
    return REF_INT_SO.exists()


def ref_int_lib() -> C.CDLL:
    global _refint
    if _refint is None:
        _refint = _load(REF_INT_SO, {
            "ref_int_max_threads": (C.c_int, []),
            "ref_int_new": (_vp, [C.c_char_p, C.c_char_p]),
            "ref_int_free": (None, [_vp]),
            "ref_int_build": (C.c_double, [_vp, C.c_int, C.c_int, C.c_float, C.c_int, C.c_int,
                                           C.c_int]),
            "ref_int_n_photons": (_i64, [_vp]),
            "ref_int_set_maps": (None, [_vp, _vp, _i64, _vp, _i64, C.c_int, C.c_int, C.c_float,
                                        C.c_int, C.c_int, C.c_int]),
            "ref_int_render": (C.c_double, [_vp, _vp, C.c_int, C.c_int, C.c_int, C.c_int,
                                            C.c_int, _vp]),
            "ref_int_render_pt": (C.c_double, [_vp, _vp, C.c_int, C.c_int, C.c_int, C.c_int,
                                               C.c_int, C.c_int, _vp]),
        })
    return _refint


class RefIntegrator:
    """The reference's own Scene + PhotonMapping/PathTracing on the CPU
    (include/scene.h, include/integrator.h compiled unchanged), over an
    OBJ/MTL pair on disk. Rendering covers rows [row0, row1) and returns the
    raw per-pixel mean (no gamma) and the seconds taken."""

    def __init__(self, obj_path):
        obj_path = Path(obj_path).resolve()
        self.lib = ref_int_lib()
        self.h = self.lib.ref_int_new(str(obj_path.parent).encode(), obj_path.name.encode())
        if not self.h:
            raise RuntimeError(f"reference Scene could not load {obj_path}")

    @staticmethod
    def threads() -> int:
        return int(ref_int_lib().ref_int_max_threads())

    def build(self, n_photons, n_est_global, caustics_multiplier, n_est_caustics, fg_depth,
              max_depth) -> float:
        """PhotonMapping(...) + build; returns seconds."""
        return float(self.lib.ref_int_build(self.h, n_photons, n_est_global,
                                            float(caustics_multiplier), n_est_caustics,
                                            fg_depth, max_depth))

    def set_maps(self, global_photons, caustic_photons, n_photons, n_est_global,
                 caustics_multiplier, n_est_caustics, fg_depth, max_depth) -> None:
        """A PhotonMapping whose two maps hold the given photons (no tracing)."""
        g = _c(global_photons, np.float32).reshape(-1, 9)
        cph = _c(caustic_photons, np.float32).reshape(-1, 9)
        self.lib.ref_int_set_maps(self.h, g.ctypes.data, g.shape[0], cph.ctypes.data,
                                  cph.shape[0], n_photons, n_est_global,
                                  float(caustics_multiplier), n_est_caustics, fg_depth, max_depth)

    def n_photons(self) -> int:
        return int(self.lib.ref_int_n_photons(self.h))

    def render(self, position, forward, fov, width, height, spp, row0=0, row1=None):
        row1 = height if row1 is None else row1
        cam = np.array([*position, *forward, fov], np.float32)
        out = np.zeros((row1 - row0, width, 3), np.float32)
        sec = self.lib.ref_int_render(self.h, cam.ctypes.data, width, height, spp, row0, row1,
                                      out.ctypes.data)
        return out, float(sec)

    def render_pt(self, position, forward, fov, width, height, spp, max_depth, row0=0,
                  row1=None):
        row1 = height if row1 is None else row1
        cam = np.array([*position, *forward, fov], np.float32)
        out = np.zeros((row1 - row0, width, 3), np.float32)
        sec = self.lib.ref_int_render_pt(self.h, cam.ctypes.data, width, height, spp, max_depth,
                                         row0, row1, out.ctypes.data)
        return out, float(sec)

    def close(self):
        if self.h:
            self.lib.ref_int_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _c(a, dtype):
    return np.ascontiguousarray(np.asarray(a, dtype=dtype))


def knn(photons, queries, k: int):
    """Exact kNN by brute force: (idx (nq,k) in heap-pop order, count, maxdist2)."""
    ph = _c(photons, np.float32).reshape(-1, 9)
    q = _c(queries, np.float32).reshape(-1, 3)
    nq = q.shape[0]
    idx = np.empty((nq, k), np.int32)
    cnt = np.empty(nq, np.int32)
    md2 = np.empty(nq, np.float32)
    oracle_lib().orc_knn(ph.ctypes.data, ph.shape[0], q.ctypes.data, nq, k,
                         idx.ctypes.data, cnt.ctypes.data, md2.ctypes.data)
    return idx, cnt, md2


def radiance_fp64(photons, idx, cnt, md2, queries, n_emitted: int) -> np.ndarray:
    ph = _c(photons, np.float32).reshape(-1, 9)
    idx, cnt, md2 = _c(idx, np.int32), _c(cnt, np.int32), _c(md2, np.float32)
    q = _c(queries, np.float32).reshape(-1, 12)
    out = np.empty((q.shape[0], 3), np.float64)
    oracle_lib().orc_radiance_fp64(ph.ctypes.data, idx.ctypes.data, cnt.ctypes.data,
                                   md2.ctypes.data, idx.shape[1], q.ctypes.data,
                                   q.shape[0], int(n_emitted), out.ctypes.data)
    return out


def radiance_fp32(photons, idx, cnt, md2, queries, n_emitted: int) -> np.ndarray:
    ph = _c(photons, np.float32).reshape(-1, 9)
    idx, cnt, md2 = _c(idx, np.int32), _c(cnt, np.int32), _c(md2, np.float32)
    q = _c(queries, np.float32).reshape(-1, 12)
    out = np.empty((q.shape[0], 3), np.float32)
    oracle_lib().orc_radiance_fp32(ph.ctypes.data, idx.ctypes.data, cnt.ctypes.data,
                                   md2.ctypes.data, idx.shape[1], q.ctypes.data,
                                   q.shape[0], int(n_emitted), out.ctypes.data)
    return out


class RefPhotonMap:
    """The reference's PhotonMap (photon_map.h), compiled unchanged."""

    def __init__(self, photons):
        self.lib = ref_pm_lib()
        self.ph = _c(photons, np.float32).reshape(-1, 9)
        self.h = self.lib.ref_pm_build(self.ph.ctypes.data, self.ph.shape[0])

    def knn(self, queries, k: int):
        q = _c(queries, np.float32).reshape(-1, 3)
        nq = q.shape[0]
        idx = np.empty((nq, k), np.int32)
        cnt = np.empty(nq, np.int32)
        md2 = np.empty(nq, np.float32)
        self.lib.ref_pm_knn(self.h, q.ctypes.data, nq, k, idx.ctypes.data,
                            cnt.ctypes.data, md2.ctypes.data)
        return idx, cnt, md2

    def radiance(self, queries, k: int, n_emitted: int) -> np.ndarray:
        q = _c(queries, np.float32).reshape(-1, 12)
        out = np.empty((q.shape[0], 3), np.float32)
        self.lib.ref_pm_radiance(self.h, q.ctypes.data, q.shape[0], k, int(n_emitted),
                                 out.ctypes.data)
        return out

    def close(self):
        if self.h:
            self.lib.ref_pm_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def ref_threads() -> int:
    return int(ref_pm_lib().ref_max_threads())


class OracleScene:
    """CPU restatement of the scene: brute-force closest hit and the
    reference's photon tracing loops (oracle/pm_oracle_trace.cpp)."""

    def __init__(self, mesh):
        self.lib = oracle_lib()
        self.v = _c(mesh.vertices, np.float32)
        self.n = _c(mesh.normals, np.float32)
        self.m = np.ascontiguousarray(mesh.materials)
        self.h = self.lib.orc_scene_new(self.v.ctypes.data, self.n.ctypes.data,
                                        self.m.ctypes.data, self.v.shape[0])

    def intersect(self, rays8):
        r = _c(rays8, np.float32).reshape(-1, 8)
        out = np.empty((r.shape[0], 4), np.float32)
        self.lib.orc_intersect(self.h, r.ctypes.data, r.shape[0], out.ctypes.data)
        return out

    def trace(self, map_id: int, seed: int, first: int, count: int, max_depth: int,
              cap: int | None = None):
        cap = cap if cap is not None else max(16, count * 8)
        out = np.empty((cap, 9), np.float32)
        st = np.zeros(2, np.uint32)
        n = self.lib.orc_trace(self.h, map_id, seed, first, count, max_depth, out.ctypes.data,
                               cap, st.ctypes.data)
        if n > cap:
            return self.trace(map_id, seed, first, count, max_depth, cap=n)
        return out[:n], st

    def render(self, global_photons, g_emitted, caustic_photons, c_emitted, camera_arr,
               width, height, spp, k_global, k_caustics, fg_depth, max_depth, n_gather=1):
        """Restated render loop (examples/main.cpp:33-70 + integrate)."""
        g = _c(global_photons, np.float32).reshape(-1, 9)
        cph = _c(caustic_photons, np.float32).reshape(-1, 9)
        cam = _c(camera_arr, np.float32)
        prm = np.array([width, height, spp, k_global, k_caustics, fg_depth, max_depth, n_gather],
                       np.int32)
        out = np.empty((height, width, 3), np.float32)
        dropped = np.zeros(2, np.int64)
        self.lib.orc_render(self.h, g.ctypes.data, g.shape[0], int(g_emitted), cph.ctypes.data,
                            cph.shape[0], int(c_emitted), cam.ctypes.data, prm.ctypes.data,
                            out.ctypes.data, dropped.ctypes.data)
        return out, dropped

    def integrate(self, global_photons, g_emitted, caustic_photons, c_emitted, rays6, states,
                  k_global, k_caustics, fg_depth, max_depth, n_gather=1):
        """PhotonMapping::integrate per ray; returns (radiance (n,3), advanced states)."""
        g = _c(global_photons, np.float32).reshape(-1, 9)
        cph = _c(caustic_photons, np.float32).reshape(-1, 9)
        r = _c(rays6, np.float32).reshape(-1, 6)
        st = np.array(states, dtype=np.uint64, copy=True)
        prm = np.array([k_global, k_caustics, fg_depth, max_depth, n_gather], np.int32)
        out = np.empty((r.shape[0], 3), np.float32)
        self.lib.orc_integrate(self.h, g.ctypes.data, g.shape[0], int(g_emitted), cph.ctypes.data,
                               cph.shape[0], int(c_emitted), r.ctypes.data, r.shape[0],
                               st.ctypes.data, prm.ctypes.data, out.ctypes.data)
        return out, st

    def grad(self, face_param, n_params, seed, n_global, n_caustic, camera_arr, width, height,
             spp, k, fg_depth, max_depth, n_gather, grad_img):
        """FP64 forward-mode derivative of the traced-and-rendered image
        (photon maps traced here: global with `seed`, caustics with seed + 1)
        contracted with grad_img = d loss / d image. Returns (d loss / d
        albedo (n_params, 3), d loss / d emission (3,), image)."""
        pid = _c(face_param, np.int32)
        cam = _c(camera_arr, np.float32)
        prm = np.array([width, height, spp, k, fg_depth, max_depth, n_gather], np.int32)
        gi = _c(grad_img, np.float32).reshape(height, width, 3)
        out = np.zeros((n_params + 1) * 3, np.float64)
        img = np.empty((height, width, 3), np.float32)
        self.lib.orc_grad(self.h, pid.ctypes.data, int(n_params), C.c_uint64(seed), int(n_global),
                          int(n_caustic), cam.ctypes.data, prm.ctypes.data, gi.ctypes.data,
                          out.ctypes.data, img.ctypes.data)
        return out[: 3 * n_params].reshape(n_params, 3), out[3 * n_params:], img

    def render_pt(self, camera_arr, width, height, spp, max_depth):
        cam = _c(camera_arr, np.float32)
        out = np.empty((height, width, 3), np.float32)
        dropped = np.zeros(1, np.int64)
        self.lib.orc_render_pt(self.h, cam.ctypes.data, width, height, spp, max_depth,
                               out.ctypes.data, dropped.ctypes.data)
        return out, int(dropped[0])

    def close(self):
        if self.h:
            self.lib.orc_scene_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def sincos(x):
    x = _c(x, np.float32).ravel()
    s = np.empty_like(x)
    c = np.empty_like(x)
    oracle_lib().orc_sincos(x.ctypes.data, x.shape[0], s.ctypes.data, c.ctypes.data)
    return s, c

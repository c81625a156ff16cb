"""PhotonMapping: the reference integrator's interface over the device.

Mirrors ``PhotonMapping`` of integrator.h:109-570: the constructor takes the
same six parameters, ``build`` traces the global (and, with final gathering,
the caustics) photon map on the device, ``getPhotonMapPtr`` exposes the
global map.
"""
from __future__ import annotations

import ctypes as C

from . import _native as N
from ._native import Context
from .photon_map import PhotonMap


class RenderParams(C.Structure):
    _fields_ = [("width", C.c_int32), ("height", C.c_int32), ("spp", C.c_int32),
                ("k_global", C.c_int32), ("k_caustics", C.c_int32),
                ("final_gathering_depth", C.c_int32), ("max_depth", C.c_int32),
                ("n_gather", C.c_int32), ("spp_batch", C.c_int32), ("flags", C.c_int32)]

PM_RENDER_FP64_CHECK = 1


class RenderStats(C.Structure):
    _fields_ = [("samples", C.c_int64), ("dropped_nan", C.c_int64),
                ("dropped_negative", C.c_int64), ("queries_global", C.c_int64),
                ("queries_caustics", C.c_int64), ("passes", C.c_int32), ("reserved", C.c_int32),
                ("accum_rel_err", C.c_double), ("rays", C.c_int64), ("camera_ms", C.c_float),
                ("estimate_ms", C.c_float)]

    def as_dict(self) -> dict:
        d = {k: int(getattr(self, k)) for k, t in self._fields_
             if k != "reserved" and t not in (C.c_float, C.c_double)}
        for k in ("accum_rel_err", "camera_ms", "estimate_ms"):
            d[k] = float(getattr(self, k))
        return d


class IntegrateParams(C.Structure):
    _fields_ = [("k_global", C.c_int32), ("k_caustics", C.c_int32),
                ("final_gathering_depth", C.c_int32), ("max_depth", C.c_int32),
                ("n_gather", C.c_int32), ("reserved", C.c_int32)]


class TraceStats(C.Structure):
    _fields_ = [("emitted", C.c_int64), ("stored", C.c_int64),
                ("nan_throughput", C.c_uint32), ("negative_throughput", C.c_uint32),
                ("rays", C.c_int64), ("trace_ms", C.c_float), ("build_ms", C.c_float)]

    def as_dict(self) -> dict:
        return {k: (float if t is C.c_float else int)(getattr(self, k)) for k, t in self._fields_}


def trace_photons(ctx: Context, map_id: int, seed: int, n_emit: int, max_depth: int) -> dict:
    """pm_photons_trace: trace n_emit photons into map `map_id`."""
    st = TraceStats()
    ctx.check(ctx.lib.pm_photons_trace(ctx.handle, int(map_id), C.c_uint64(seed), int(n_emit),
                                       int(max_depth), C.addressof(st)),
              "pm_photons_trace")
    return st.as_dict()


class PhotonMapping:
    """integrator.h:380-390 constructor arguments, in order."""

    def __init__(self, nPhotonsGlobal: int, nEstimationGlobal: int,
                 nPhotonsCausticsMultiplier: float, nEstimationCaustics: int,
                 strictCalcDepth: int, maxDepth: int, ctx: Context | None = None):
        self.ctx = ctx if ctx is not None else Context(0)
        self.nPhotonsGlobal = int(nPhotonsGlobal)
        self.nEstimationGlobal = int(nEstimationGlobal)
        # int * float, stored into an int member (integrator.h:385)
        self.nPhotonsCaustics = int(C.c_float(nPhotonsGlobal * C.c_float(nPhotonsCausticsMultiplier).value).value)
        self.nEstimationCaustics = int(nEstimationCaustics)
        self.finalGatheringDepth = int(strictCalcDepth)
        self.maxDepth = int(maxDepth)
        self.global_map = PhotonMap(self.ctx, N.PM_MAP_GLOBAL)
        self.caustics_map = PhotonMap(self.ctx, N.PM_MAP_CAUSTICS)
        self.stats: dict = {}

    def getPhotonMapPtr(self) -> PhotonMap:  # integrator.h:390
        return self.global_map

    def build(self, scene, seed: int = 1) -> dict:  # integrator.h:393
        """Traces the photon maps for `scene` (already built on this
        context). The caustics map is traced only with final gathering
        (integrator.h:477)."""
        self.stats = {"global": trace_photons(self.ctx, N.PM_MAP_GLOBAL, seed, self.nPhotonsGlobal,
                                              self.maxDepth)}
        if self.finalGatheringDepth > 0:
            self.stats["caustics"] = trace_photons(self.ctx, N.PM_MAP_CAUSTICS, seed + 1,
                                                   self.nPhotonsCaustics, self.maxDepth)
        else:
            self.ctx.check(self.ctx.lib.pm_photonmap_build(self.ctx.handle, N.PM_MAP_CAUSTICS,
                                                           None, 0), "pm_photonmap_build")
        return self.stats

    def integrate_batch(self, origins, directions, rng_states, n_gather: int = 1):
        """PhotonMapping::integrate (integrator.h:566-569) for many rays, each
        with its sampler's PCG32 state: returns (radiance (n, 3), states
        advanced by the draws integrate made)."""
        import numpy as np
        o = np.asarray(origins, np.float32).reshape(-1, 3)
        d = np.asarray(directions, np.float32).reshape(-1, 3)
        rays = np.ascontiguousarray(np.concatenate([o, d], axis=1))
        st = np.array(rng_states, dtype=np.uint64, copy=True).reshape(-1)
        out = np.empty((rays.shape[0], 3), np.float32)
        p = IntegrateParams(self.nEstimationGlobal, self.nEstimationGlobal,
                            self.finalGatheringDepth, self.maxDepth, int(n_gather), 0)
        self.ctx.check(self.ctx.lib.pm_integrate(self.ctx.handle, rays.ctypes.data, rays.shape[0],
                                                 st.ctypes.data, C.addressof(p), out.ctypes.data),
                       "pm_integrate")
        return out, st

    def integrate(self, ray, scene, sampler):
        """integrator.h:566: radiance along one ray; `sampler` (a state
        holder with a `state` attribute) advances like the reference's."""
        out, st = self.integrate_batch([ray[0]], [ray[1]], [sampler.state])
        sampler.state = int(st[0])
        return out[0]

    def render(self, camera, width: int, height: int, n_samples: int, n_gather: int = 1,
               spp_batch: int = 0, fp64_check: bool = False):
        """The render loop of examples/main.cpp:33-70 on the device: returns
        (image (height, width, 3) float32 averaged over n_samples, stats).
        The caustics estimate uses k = nEstimationGlobal like the reference
        (integrator.h:161). fp64_check: also sum the samples in FP64 and
        report the image's largest relative difference from those sums
        (stats["accum_rel_err"])."""
        import numpy as np
        p = RenderParams(int(width), int(height), int(n_samples), self.nEstimationGlobal,
                         self.nEstimationGlobal, self.finalGatheringDepth, self.maxDepth,
                         int(n_gather), int(spp_batch),
                         PM_RENDER_FP64_CHECK if fp64_check else 0)
        out = np.empty((height, width, 3), np.float32)
        st = RenderStats()
        cam = camera.as_struct()
        self.ctx.check(self.ctx.lib.pm_render(self.ctx.handle, C.addressof(cam), C.addressof(p),
                                              out.ctypes.data, C.addressof(st)), "pm_render")
        return out, st.as_dict()


class PathTracing:
    """PathTracing (integrator.h:51-106): the unidirectional reference
    integrator, rendered on the device."""

    def __init__(self, maxDepth: int = 100, ctx: Context | None = None):
        self.ctx = ctx if ctx is not None else Context(0)
        self.maxDepth = int(maxDepth)

    def build(self, scene, seed: int = 1) -> None:  # integrator.h:58: nothing to do
        pass

    def render(self, camera, width: int, height: int, n_samples: int):
        """tests/test_path_tracing.cpp:25-52 on the device: (image, NaN drops)."""
        import numpy as np
        out = np.empty((height, width, 3), np.float32)
        dropped = C.c_int64(0)
        cam = camera.as_struct()
        self.ctx.check(self.ctx.lib.pm_render_path_tracing(
            self.ctx.handle, C.addressof(cam), int(width), int(height), int(n_samples),
            self.maxDepth, out.ctypes.data, C.byref(dropped)), "pm_render_path_tracing")
        return out, int(dropped.value)

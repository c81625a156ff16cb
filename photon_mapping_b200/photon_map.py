"""PhotonMap: the reference's photon-map interface over the device map.

Mirrors ``PhotonMap`` of photon_map.h:186-212 (setPhotons, addPhoton, build,
queryKNearestPhotons, getIthPhoton, getNPhotons) and adds the batched calls
a GPU wants (``query_knn``, ``radiance``). A photon is 9 floats
{throughput.rgb, position.xyz, wi.xyz} (photon_map.h:10-22).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _native as N
from ._native import Context, PMError, ptr


def as_photons(photons) -> np.ndarray:
    a = np.ascontiguousarray(np.asarray(photons, dtype=np.float32))
    if a.size == 0:
        return a.reshape(0, 9)
    if a.ndim != 2 or a.shape[1] != 9:
        raise ValueError(f"photons must be (n, 9) float32, got {a.shape}")
    return a


def radiance_queries(pos, wo, ns, rho) -> np.ndarray:
    """Packs pm_radiance_query records (n, 12) float32 from (n, 3) arrays."""
    pos, wo, ns, rho = (np.asarray(x, dtype=np.float32).reshape(-1, 3) for x in (pos, wo, ns, rho))
    q = np.empty((pos.shape[0], 12), dtype=np.float32)
    q[:, 0:3], q[:, 3] = pos, rho[:, 0]
    q[:, 4:7], q[:, 7] = wo, rho[:, 1]
    q[:, 8:11], q[:, 11] = ns, rho[:, 2]
    return q


class PhotonMap:
    """A photon map living on the device (one of the context's two maps)."""

    def __init__(self, ctx: Context | None = None, map_id: int = N.PM_MAP_GLOBAL):
        self.ctx = ctx if ctx is not None else Context(0)
        self.map_id = map_id
        self._pending: list[np.ndarray] = []
        self._photons = np.zeros((0, 9), dtype=np.float32)
        self._built = False

    # photon_map.h:197-200
    def addPhoton(self, photon) -> None:
        self._pending.append(np.asarray(photon, dtype=np.float32).reshape(1, 9))
        self._built = False

    def setPhotons(self, photons) -> None:
        self._photons = as_photons(photons).copy()
        self._pending = []
        self._built = False

    # photon_map.h:202-206
    def build(self) -> None:
        if self._pending:
            self._photons = np.concatenate([self._photons, *self._pending], axis=0)
            self._pending = []
        a = self._photons
        self.ctx.check(self.ctx.lib.pm_photonmap_build(self.ctx.handle, self.map_id,
                                                       ptr(a), a.shape[0]),
                       "pm_photonmap_build")
        self._built = True

    # photon_map.h:194
    def getNPhotons(self) -> int:
        n = C.c_int64()
        self.ctx.check(self.ctx.lib.pm_photonmap_size(self.ctx.handle, self.map_id, C.byref(n)),
                       "pm_photonmap_size")
        return int(n.value)

    # photon_map.h:195
    def getIthPhoton(self, i: int) -> np.ndarray:
        out = np.empty(9, dtype=np.float32)
        self.ctx.check(self.ctx.lib.pm_photonmap_get_photons(self.ctx.handle, self.map_id,
                                                             int(i), 1, ptr(out)),
                       "pm_photonmap_get_photons")
        return out

    def photons(self) -> np.ndarray:
        n = self.getNPhotons()
        out = np.empty((n, 9), dtype=np.float32)
        if n:
            self.ctx.check(self.ctx.lib.pm_photonmap_get_photons(self.ctx.handle, self.map_id,
                                                                 0, n, ptr(out)),
                           "pm_photonmap_get_photons")
        return out

    # photon_map.h:208-211
    def queryKNearestPhotons(self, p, k: int) -> tuple[list[int], float]:
        idx, cnt, md2 = self.query_knn(np.asarray(p, dtype=np.float32).reshape(1, 3), k)
        return [int(x) for x in idx[0, : cnt[0]]], float(md2[0])

    def query_knn(self, queries, k: int):
        """Batched queryKNearestPhotons: (idx (nq,k) int32, count (nq,), maxdist2 (nq,))."""
        q = np.ascontiguousarray(np.asarray(queries, dtype=np.float32).reshape(-1, 3))
        nq = q.shape[0]
        idx = np.empty((nq, max(k, 1)), dtype=np.int32)
        cnt = np.empty(nq, dtype=np.int32)
        md2 = np.empty(nq, dtype=np.float32)
        self.ctx.check(self.ctx.lib.pm_photonmap_knn(self.ctx.handle, self.map_id, ptr(q), nq,
                                                     int(k), ptr(idx), ptr(cnt), ptr(md2)),
                       "pm_photonmap_knn")
        return idx, cnt, md2

    def radiance(self, queries: np.ndarray, k: int, n_emitted: int) -> np.ndarray:
        """Batched computeRadianceWithPhotonMap (integrator.h:133-152): (nq, 3)."""
        q = np.ascontiguousarray(np.asarray(queries, dtype=np.float32).reshape(-1, 12))
        out = np.empty((q.shape[0], 3), dtype=np.float32)
        self.ctx.check(self.ctx.lib.pm_photonmap_radiance(self.ctx.handle, self.map_id, ptr(q),
                                                          q.shape[0], int(k), int(n_emitted),
                                                          ptr(out)),
                       "pm_photonmap_radiance")
        return out


__all__ = ["PhotonMap", "PMError", "radiance_queries", "as_photons"]

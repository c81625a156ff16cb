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


# Binary photon file: 16-byte header {magic "PMPH", version 1 (u32), photon
# count (u64)}, the number of photons emitted (u64), then count records of 9
# little-endian float32 {throughput, position, wi} (photon_map.h:10-22).
PHOTON_FILE_MAGIC = b"PMPH"


def save_photons(path, photons, n_emitted: int) -> None:
    """Writes a photon set and the number of photons emitted to make it
    (the estimate's normalisation, integrator.h:149)."""
    a = np.ascontiguousarray(as_photons(photons), dtype="<f4")
    with open(path, "wb") as f:
        f.write(PHOTON_FILE_MAGIC + np.array([1], "<u4").tobytes() +
                np.array([a.shape[0], int(n_emitted)], "<u8").tobytes())
        f.write(a.tobytes())


def load_photons(path) -> tuple[np.ndarray, int]:
    """Reads a file of save_photons: (photons (n, 9) float32, n_emitted)."""
    with open(path, "rb") as f:
        head = f.read(24)
        if len(head) != 24 or head[:4] != PHOTON_FILE_MAGIC:
            raise ValueError(f"{path}: not a photon file")
        version = int(np.frombuffer(head, "<u4", 1, 4)[0])
        if version != 1:
            raise ValueError(f"{path}: photon file version {version}")
        n, emitted = (int(x) for x in np.frombuffer(head, "<u8", 2, 8))
        body = f.read()
    if len(body) != n * 36:
        raise ValueError(f"{path}: {len(body)} bytes for {n} photons")
    return np.frombuffer(body, "<f4").reshape(n, 9).astype(np.float32), emitted


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

    def save(self, path, n_emitted: int) -> None:
        """Writes the map's photons (index order) to a photon file."""
        save_photons(path, self.photons(), n_emitted)

    def load(self, path) -> int:
        """Replaces the photons with a photon file's and builds the map;
        returns the number of photons emitted recorded in the file."""
        photons, emitted = load_photons(path)
        self.setPhotons(photons)
        self.build()
        self.ctx.check(self.ctx.lib.pm_photonmap_set_emitted(self.ctx.handle, self.map_id,
                                                             int(emitted)),
                       "pm_photonmap_set_emitted")
        return emitted

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


__all__ = ["PhotonMap", "PMError", "radiance_queries", "as_photons", "save_photons",
           "load_photons"]

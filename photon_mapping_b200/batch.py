"""Batched rendering of many scenes in one step (pm_batch_* of the C ABI).

The reference renders one scene per run (examples/main.cpp:7-71). A batch
renders many scenes, views and query sets of uneven size together: one
launch traces every scene's photons, the maps are built per scene on 8
streams, one launch runs every camera pass, one persistent launch answers
every photon-map query, one launch resolves every image; the step is
captured in a CUDA graph and replayed. `autotune` picks the launch shapes
(kNN warps per block, queries per work item, candidate buffer size, BVH
traversal stack depth, block size) by timing them on the batch itself.

`random_scene` draws the scenes of the batched benchmark: Cornell rooms with
1 to 40 random boxes and a displaced heightfield floor, the triangle count
log-uniform in [1k, 500k]; per scene the photon count is log-uniform in
[100k, 4M], k is 50 or 100 and the image side log-uniform in [128, 1024].
`sequential` renders the same scenes one after another through the
per-scene API (PhotonMapping.build + render on one context per scene).
"""
from __future__ import annotations

import ctypes as C
import math
import time

import numpy as np

from . import _native as N
from . import scene as S
from .camera import Camera, PMCamera


class BatchSceneDesc(C.Structure):
    _fields_ = [("vertices", C.c_void_p), ("normals", C.c_void_p), ("materials", C.c_void_p),
                ("n_faces", C.c_int64), ("camera", PMCamera), ("width", C.c_int32),
                ("height", C.c_int32), ("spp", C.c_int32), ("k", C.c_int32),
                ("max_depth", C.c_int32), ("reserved", C.c_int32), ("n_photons", C.c_int64),
                ("seed", C.c_uint64)]


class BatchTuning(C.Structure):
    _fields_ = [("knn_warps", C.c_int32), ("knn_chunk", C.c_int32), ("knn_buffer", C.c_int32),
                ("bvh_stack", C.c_int32), ("block", C.c_int32), ("reserved", C.c_int32)]

    def as_dict(self) -> dict:
        return {k: int(getattr(self, k)) for k, _ in self._fields_ if k != "reserved"}


def random_scene(seed: int, tri_range=(1_000, 500_000), photon_range=(100_000, 4_000_000),
                 side_range=(128, 1024), ks=(50, 100), spp: int = 2, max_depth: int = 100):
    """One scene of the batched benchmark and its render settings (a dict
    with mesh, camera, width, height, spp, k, photons, seed, max_depth)."""
    rng = np.random.default_rng(seed)
    target = math.exp(rng.uniform(math.log(tri_range[0]), math.log(tri_range[1])))
    n_boxes = int(rng.integers(1, 41))
    room = S.cornell_box(0, boxes=False)
    keep = [i for i, nm in enumerate(room.names) if nm != "floor"]
    mesh = S.Mesh(room.vertices[keep], room.normals[keep], room.materials[keep],
                  [room.names[i] for i in keep])
    # the displaced floor: (g - 1)^2 cells of 2 triangles
    cells = max(target - mesh.n_faces - 12 * n_boxes, 2 * 15 * 15) / 2.0
    g = int(round(math.sqrt(cells))) + 1
    mesh = mesh + S.heightfield(g, 0.02, int(rng.integers(1 << 30)), S.material(rho=S.WHITE),
                                "floor", n_sines=8, amp_max=0.015, wl=(0.08, 0.4))
    for b in range(n_boxes):
        size = rng.uniform(0.05, 0.22, 3)
        size[1] = rng.uniform(0.05, 0.45)
        center = (rng.uniform(0.15, 0.85), 0.04 + size[1] / 2.0, rng.uniform(0.15, 0.85))
        alb = tuple(rng.uniform(0.1, 0.85, 3))
        mesh = mesh + S.box_mesh(center, tuple(size), rng.uniform(0, math.pi / 2),
                                 S.material(rho=alb), f"box{b}")
    photons = int(math.exp(rng.uniform(math.log(photon_range[0]), math.log(photon_range[1]))))
    side = int(round(math.exp(rng.uniform(math.log(side_range[0]), math.log(side_range[1])))))
    cam = Camera(S.CAMERA["position"], S.CAMERA["forward"], S.CAMERA["fov"])
    return dict(mesh=mesh, camera=cam, width=side, height=side, spp=spp, k=int(rng.choice(ks)),
                photons=photons, seed=int(seed) + 1, max_depth=max_depth)


class BatchRenderer:
    """A pm_batch over `scenes` (dicts as random_scene returns)."""

    def __init__(self, scenes, device: int = 0):
        self.lib = N.load()
        self.scenes = scenes
        self._keep = []
        arr = (BatchSceneDesc * len(scenes))()
        for i, sc in enumerate(scenes):
            m = sc["mesh"]
            v = np.ascontiguousarray(m.vertices, np.float32)
            n = np.ascontiguousarray(m.normals, np.float32)
            mt = np.ascontiguousarray(m.materials, S.MATERIAL_DTYPE)
            self._keep += [v, n, mt]
            d = arr[i]
            d.vertices, d.normals, d.materials = v.ctypes.data, n.ctypes.data, mt.ctypes.data
            d.n_faces = m.n_faces
            d.camera = sc["camera"].as_struct()
            d.width, d.height, d.spp, d.k = sc["width"], sc["height"], sc["spp"], sc["k"]
            d.max_depth, d.n_photons, d.seed = sc["max_depth"], sc["photons"], sc["seed"]
        h = C.c_void_p()
        st = self.lib.pm_batch_create(int(device), C.addressof(arr), len(scenes), C.byref(h))
        self.handle = h
        self._keep = []
        if st != N.PM_OK:
            msg = self.lib.pm_batch_last_error(h).decode() if h.value else ""
            self.close()
            raise N.PMError(st, f"pm_batch_create: {msg}")

    def check(self, st: int, what: str) -> None:
        if st != N.PM_OK:
            raise N.PMError(st, f"{what}: {self.lib.pm_batch_last_error(self.handle).decode()}")

    def close(self) -> None:
        if getattr(self, "handle", None) and self.handle.value:
            self.lib.pm_batch_destroy(self.handle)
        self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def tuning(self) -> dict:
        t = BatchTuning()
        self.check(self.lib.pm_batch_get_tuning(self.handle, C.addressof(t)),
                   "pm_batch_get_tuning")
        return t.as_dict()

    def set_tuning(self, **kw) -> None:
        t = BatchTuning(**{**self.tuning(), **kw})
        self.check(self.lib.pm_batch_set_tuning(self.handle, C.addressof(t)),
                   "pm_batch_set_tuning")

    def autotune(self) -> tuple[dict, list]:
        t = BatchTuning()
        ms = (C.c_float * 3)()
        self.check(self.lib.pm_batch_autotune(self.handle, C.addressof(t), C.addressof(ms)),
                   "pm_batch_autotune")
        return t.as_dict(), [float(x) for x in ms]

    def render(self, use_graph: bool = True) -> float:
        """One step over every scene; returns its device time in ms."""
        ms = C.c_float(0.0)
        self.check(self.lib.pm_batch_render(self.handle, int(bool(use_graph)),
                                            C.addressof(ms)), "pm_batch_render")
        return float(ms.value)

    STAGES = ("trace", "maps", "camera", "sort", "knn", "resolve")

    def stage_times(self) -> dict:
        """One step without a graph, each stage timed on the device (ms)."""
        ms = (C.c_float * len(self.STAGES))()
        self.check(self.lib.pm_batch_stage_times(self.handle, C.addressof(ms), len(ms)),
                   "pm_batch_stage_times")
        return {k: float(v) for k, v in zip(self.STAGES, ms)}

    def image(self, i: int) -> np.ndarray:
        sc = self.scenes[i]
        out = np.empty((sc["height"], sc["width"], 3), np.float32)
        self.check(self.lib.pm_batch_image(self.handle, int(i), out.ctypes.data), "pm_batch_image")
        return out

    def photons(self, i: int) -> np.ndarray:
        """Scene i's stored photons (n, 9) in index order, after the last step."""
        stored, _ = self.counts()
        out = np.empty((int(stored[i]), 9), np.float32)
        self.check(self.lib.pm_batch_photons(self.handle, int(i), out.ctypes.data),
                   "pm_batch_photons")
        return out

    def counts(self) -> tuple[np.ndarray, np.ndarray]:
        n = len(self.scenes)
        st, q = np.zeros(n, np.int64), np.zeros(n, np.int64)
        self.check(self.lib.pm_batch_counts(self.handle, st.ctypes.data, q.ctypes.data),
                   "pm_batch_counts")
        return st, q


class Sequential:
    """The per-scene loop the batch replaces: one context per scene (scene
    uploaded once), then per step and scene PhotonMapping.build +
    PhotonMapping.render, one after another."""

    def __init__(self, scenes, device: int = 0):
        from .integrator import PhotonMapping
        self.scenes = scenes
        self.ctxs, self.pmis = [], []
        for sc in scenes:
            ctx = N.Context(device)
            s = S.Scene(ctx)
            s.setMesh(sc["mesh"])
            s.build()
            self.ctxs.append((ctx, s))
            self.pmis.append(PhotonMapping(sc["photons"], sc["k"], 1.0, sc["k"], 0,
                                           sc["max_depth"], ctx=ctx))

    def render(self) -> tuple[list, float]:
        """(images, wall seconds) of one pass over every scene."""
        imgs = []
        t0 = time.perf_counter()
        for sc, (ctx, s), pmi in zip(self.scenes, self.ctxs, self.pmis):
            pmi.build(s, seed=sc["seed"])
            img, _ = pmi.render(sc["camera"], sc["width"], sc["height"], sc["spp"])
            imgs.append(img)
        return imgs, time.perf_counter() - t0

    def close(self) -> None:
        for ctx, _ in self.ctxs:
            ctx.close()
        self.ctxs = []

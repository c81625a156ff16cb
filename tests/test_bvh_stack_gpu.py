"""The BVH traversal-stack guard (pm_scene.cuh, intersect_t): a ray that
needs more stack entries than the traversal has drops the deepest pending
subtrees, sets bit 0 of the device error word and carries on, so the call
reports PM_ERR_DEVICE_STATUS instead of reading or writing out of bounds
(the guard-log-continue style of integrator.h:418-426).

The scenes are built so that every node box is the same: every triangle has
the vertices (0,0,0) and (1,1,1) and its third vertex inside that cube. The
clustering build (pm_scene.cu) then pairs the clusters (2k, 2k + 1) pass
after pass, a balanced tree with ceil(log2(faces)) levels, and a ray from
inside the cube enters every box at the same distance: the traversal goes
left and pushes the right child on every level whose children are both
inner nodes. 160,016 faces give 18 levels, 17 pushes: more than a 16-entry
stack holds, within 32 and 64.
"""
from __future__ import annotations

import numpy as np
import pytest

from oracle import oracle as O
from photon_mapping_b200 import _native as N
from photon_mapping_b200 import batch as B
from photon_mapping_b200 import scene as S
from photon_mapping_b200.camera import Camera

pytestmark = pytest.mark.gpu

N_CHAIN_BITS = 24     # Morton code bits 0..23: cells 512 + 2^j stay inside [342, 681]
N_REST = 4096         # triangles with the base code
N_LIGHTS = 16         # emitting triangles, also with the base code
N_DEEP = 160000       # white faces of the overflow scene: 18 tree levels


def _tri(cell, frac):
    """Vertices (0,0,0), (1,1,1), C with centroid (cell + frac) / 1024 per axis."""
    c = (np.asarray(cell, np.float64) + np.asarray(frac, np.float64)) / 1024.0
    return np.concatenate([[0.0, 0.0, 0.0], [1.0, 1.0, 1.0], 3.0 * c - 1.0])


def deep_chain_mesh(n_rest: int = N_REST) -> S.Mesh:
    """Faces whose boxes are all the unit cube (centroids spread over the
    Morton cells 512 + 2^j along the axes, then n_rest more on one cell)."""
    base = np.array([512, 512, 512])
    frac = (0.2, 0.5, 0.8)            # centroid off the diagonal: no degenerate triangle
    tris = []
    for b in range(N_CHAIN_BITS):
        axis = 2 - (b % 3)            # Morton bit 3j+2 is x bit j, 3j+1 is y, 3j is z
        cell = base.copy()
        cell[axis] += 1 << (b // 3)
        tris += [_tri(cell, frac)] * 2
    white = S.mesh_from_triangles(np.array(tris + [_tri(base, frac)] * n_rest),
                                  S.material(rho=S.WHITE), "white")
    light = S.mesh_from_triangles(np.array([_tri(base, frac)] * N_LIGHTS),
                                  S.material(rho=(0.0, 0.0, 0.0), le=(1.0, 1.0, 1.0)), "light")
    return white + light


def test_deep_tree_intersections_exact_with_the_default_stack(ctx):
    """The context's intersector (64 entries) holds the 12 pushes the tree
    needs; every ray that enters the cube visits every node."""
    mesh = deep_chain_mesh()
    sc = S.Scene(ctx)
    sc.setMesh(mesh)
    sc.build()
    rng = np.random.default_rng(3)
    o = rng.uniform(-0.5, 1.5, (2000, 3)).astype(np.float32)
    d = rng.normal(size=(2000, 3))
    d = (d / np.linalg.norm(d, axis=1, keepdims=True)).astype(np.float32)
    got = sc.intersect(o, d)
    r = np.empty((o.shape[0], 8), np.float32)
    r[:, 0:3], r[:, 3], r[:, 4:7], r[:, 7] = o, 1e-5, d, np.finfo(np.float32).max
    want = O.OracleScene(mesh).intersect(r)
    np.testing.assert_array_equal(got["prim"], want[:, 3].view(np.int32))
    hit = got["prim"] >= 0
    assert hit.sum() > 20          # thin triangles: few rays hit one
    np.testing.assert_array_equal(got["t"][hit], want[hit, 0])


def test_stack_overflow_is_reported_and_rejected_by_the_autotuner():
    cam = Camera(S.CAMERA["position"], S.CAMERA["forward"], S.CAMERA["fov"])
    mesh = deep_chain_mesh(N_DEEP - 2 * N_CHAIN_BITS)
    assert mesh.n_faces == N_DEEP + N_LIGHTS
    scene = dict(mesh=mesh, camera=cam, width=8, height=8, spp=1, k=10,
                 photons=200, seed=5, max_depth=4)
    br = B.BatchRenderer([scene])
    try:
        br.set_tuning(bvh_stack=64)
        br.render(use_graph=False)
        img = br.image(0)
        # 16 entries: every photon ray overflows; the step reports it
        br.set_tuning(bvh_stack=16)
        for use_graph in (False, True):
            with pytest.raises(N.PMError) as e:
                br.render(use_graph=use_graph)
            assert e.value.status == N.PM_ERR_DEVICE_STATUS
            assert "device error bits 0x1" in str(e.value)
        # the batch stays usable, and the tuner never picks the failing depth
        br.set_tuning(bvh_stack=64)
        br.render(use_graph=False)
        np.testing.assert_array_equal(br.image(0), img)
        br.set_tuning(bvh_stack=32)
        br.render(use_graph=False)
        np.testing.assert_array_equal(br.image(0), img)
        best, _ = br.autotune()
        assert best["bvh_stack"] in (32, 64)
        br.render(use_graph=True)
        np.testing.assert_array_equal(br.image(0), img)
    finally:
        br.close()

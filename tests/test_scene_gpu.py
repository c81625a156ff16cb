"""Parity of the device scene (BVH closest hit) and of the photon tracer
with the CPU oracle.

Bar: closest hits identical (t, u, v and face index, bit for bit) to a
brute-force test of every triangle with the same arithmetic; traced photon
sets identical, photon by photon, to the oracle's restatement of the
reference's tracing loops fed the same per-photon random streams.
"""
from __future__ import annotations

import numpy as np
import pytest

from oracle import oracle as O
from photon_mapping_b200 import Context, PMError
from photon_mapping_b200 import scene as S
from photon_mapping_b200.integrator import PhotonMapping, trace_photons
from photon_mapping_b200.photon_map import PhotonMap

pytestmark = pytest.mark.gpu


def random_rays(rng, n, lo=-0.2, hi=1.2):
    o = rng.uniform(lo, hi, (n, 3)).astype(np.float32)
    d = rng.normal(size=(n, 3))
    d = (d / np.linalg.norm(d, axis=1, keepdims=True)).astype(np.float32)
    return o, d


def rays8(o, d, tmin=1e-5, tmax=np.finfo(np.float32).max):
    r = np.empty((o.shape[0], 8), np.float32)
    r[:, 0:3], r[:, 3], r[:, 4:7], r[:, 7] = o, tmin, d, tmax
    return r


def check_hits(gpu, orc):
    prim = gpu["prim"]
    oprim = orc[:, 3].view(np.int32)
    np.testing.assert_array_equal(prim, oprim)
    hit = prim >= 0
    np.testing.assert_array_equal(gpu["t"][hit], orc[hit, 0])
    np.testing.assert_array_equal(gpu["u"][hit], orc[hit, 1])
    np.testing.assert_array_equal(gpu["v"][hit], orc[hit, 2])


@pytest.fixture(scope="module")
def small_caustics():
    return S.caustics_scene(0, grid=48, subdiv=3)


def test_cornell_intersections_exact(ctx):
    mesh = S.cornell_box(3)
    sc = S.Scene(ctx)
    sc.setMesh(mesh)
    sc.build()
    rng = np.random.default_rng(0)
    o, d = random_rays(rng, 50000)
    # axis-aligned rays and rays along the walls' planes
    o2 = rng.uniform(0, 1, (4000, 3)).astype(np.float32)
    d2 = np.zeros((4000, 3), np.float32)
    d2[np.arange(4000), rng.integers(0, 3, 4000)] = rng.choice([-1.0, 1.0], 4000)
    o = np.concatenate([o, o2])
    d = np.concatenate([d, d2])
    got = sc.intersect(o, d)
    want = O.OracleScene(mesh).intersect(rays8(o, d))
    check_hits(got, want)
    assert (got["prim"] >= 0).mean() > 0.5


def _edge_case_mesh(kind: str) -> S.Mesh:
    """Small or tie-heavy scenes for the clustering build (pm_scene.cu):
    the fewest faces with an inner node, duplicates (equal boxes and equal
    hit distances), zero-area faces, one face far larger than the rest, and
    faces whose boxes are all the same cube."""
    seeds = {"two": 1, "three": 2, "duplicates": 3, "zero_area": 4, "huge_and_tiny": 5,
             "equal_boxes": 6}
    rng = np.random.default_rng(seeds[kind])

    def tris(n, lo=0.0, hi=1.0, size=0.2):
        c = rng.uniform(lo, hi, (n, 1, 3))
        return (c + rng.uniform(-size, size, (n, 3, 3))).reshape(n, 9)

    if kind == "two":
        t = tris(2)
    elif kind == "three":
        t = tris(3)
    elif kind == "duplicates":
        t = np.concatenate([np.repeat(tris(1), 300, axis=0), tris(5)])
    elif kind == "zero_area":
        a = rng.uniform(0, 1, (200, 3))
        b = rng.uniform(0, 1, (200, 3))
        line = np.concatenate([a, b, 0.5 * (a + b)], axis=1)  # collinear vertices
        t = np.concatenate([line, tris(200)])[rng.permutation(400)]
    elif kind == "huge_and_tiny":
        big = np.array([[-10.0, -10.0, 0.5, 10.0, -10.0, 0.5, 0.0, 10.0, 0.5]])
        t = np.concatenate([tris(5000, size=0.01), big])
    elif kind == "equal_boxes":
        third = rng.uniform(0.05, 0.95, (1000, 3))
        t = np.concatenate([np.zeros((1000, 3)), np.ones((1000, 3)), third], axis=1)
    else:
        raise ValueError(kind)
    up = np.tile(np.array([0.0, 0.0, 1.0]), (t.shape[0], 3))  # zero-area faces have no normal
    return S.mesh_from_triangles(t.astype(np.float64), S.material(rho=S.WHITE), "white",
                                 normals=up)


@pytest.mark.parametrize("kind", ["two", "three", "duplicates", "zero_area", "huge_and_tiny",
                                  "equal_boxes"])
def test_bvh_edge_case_scenes_exact(ctx, kind):
    mesh = _edge_case_mesh(kind)
    sc = S.Scene(ctx)
    sc.setMesh(mesh)
    sc.build()
    rng = np.random.default_rng(7)
    o, d = random_rays(rng, 20000)
    o2 = rng.uniform(0, 1, (2000, 3)).astype(np.float32)
    d2 = np.zeros((2000, 3), np.float32)
    d2[np.arange(2000), rng.integers(0, 3, 2000)] = rng.choice([-1.0, 1.0], 2000)
    o = np.concatenate([o, o2])
    d = np.concatenate([d, d2])
    got = sc.intersect(o, d)
    want = O.OracleScene(mesh).intersect(rays8(o, d))
    check_hits(got, want)
    assert (got["prim"] >= 0).sum() > 0


def test_shadow_ray_tmax_and_misses(ctx):
    mesh = S.cornell_box(1)
    sc = S.Scene(ctx)
    sc.setMesh(mesh)
    sc.build()
    o = np.array([[0.5, 0.5, 0.5], [0.5, 0.5, 0.5], [0.5, 0.5, 5.0]], np.float32)
    d = np.array([[0, -1, 0], [0, -1, 0], [0, 0, 1]], np.float32)
    r = rays8(o, d)
    r[1, 7] = 0.1  # the floor is 0.5 away: no hit before tmax
    got = O.OracleScene(mesh).intersect(r)
    gpu = np.empty(3, S.HIT_DTYPE)
    ctx.check(ctx.lib.pm_scene_intersect(ctx.handle, r.ctypes.data, 3, gpu.ctypes.data), "isect")
    check_hits(gpu, got)
    assert gpu["prim"][1] == -1 and gpu["prim"][2] == -1


def test_caustics_scene_intersections_exact(ctx, small_caustics):
    sc = S.Scene(ctx)
    sc.setMesh(small_caustics)
    sc.build()
    rng = np.random.default_rng(1)
    o, d = random_rays(rng, 20000, 0.0, 1.0)
    got = sc.intersect(o, d)
    want = O.OracleScene(small_caustics).intersect(rays8(o, d))
    check_hits(got, want)


def test_full_size_caustics_scene_sample(ctx):
    mesh = S.caustics_scene(0)  # 563,238 triangles
    sc = S.Scene(ctx)
    sc.setMesh(mesh)
    sc.build()
    rng = np.random.default_rng(2)
    o, d = random_rays(rng, 200000, 0.0, 1.0)
    got = sc.intersect(o, d)
    sample = rng.choice(o.shape[0], 600, replace=False)
    want = O.OracleScene(mesh).intersect(rays8(o[sample], d[sample]))
    check_hits(got[sample], want)


def test_scene_errors(ctx):
    c2 = Context(0)
    try:
        sc = S.Scene(c2)
        with pytest.raises(PMError) as e:
            c2.check(c2.lib.pm_scene_intersect(c2.handle, np.zeros(8, np.float32).ctypes.data, 1,
                                               np.zeros(4, np.float32).ctypes.data), "isect")
        assert e.value.status == 4
        bad = S.cornell_box(0)
        bad.materials["type"][0] = 7
        sc.setMesh(bad)
        with pytest.raises(PMError):
            sc.build()
        # a scene without lights cannot emit photons
        dark = S.cornell_box(0, light_le=(0.0, 0.0, 0.0))
        sc.setMesh(dark)
        sc.build()
        with pytest.raises(PMError):
            trace_photons(c2, 0, 1, 100, 10)
    finally:
        c2.close()


@pytest.mark.parametrize("map_id", [0, 1])
def test_trace_matches_oracle(ctx, small_caustics, map_id):
    sc = S.Scene(ctx)
    sc.setMesh(small_caustics)
    sc.build()
    n_emit, seed, depth = 20000, 77, 100
    st = trace_photons(ctx, map_id, seed, n_emit, depth)
    pm = PhotonMap(ctx, map_id)
    got = pm.photons()
    want, ost = O.OracleScene(small_caustics).trace(map_id, seed, 0, n_emit, depth)
    assert st["stored"] == want.shape[0]
    assert st["nan_throughput"] == ost[0] and st["negative_throughput"] == ost[1]
    np.testing.assert_array_equal(got, want)
    assert want.shape[0] > (n_emit if map_id == 0 else 100)


def test_trace_large_matches_oracle(ctx):
    """More than 1M stored photons: the photon-order sort spans more than 256
    tiles."""
    mesh = S.cornell_box(2)
    sc = S.Scene(ctx)
    sc.setMesh(mesh)
    sc.build()
    st = trace_photons(ctx, 0, 11, 400000, 100)
    got = PhotonMap(ctx, 0).photons()
    want, _ = O.OracleScene(mesh).trace(0, 11, 0, 400000, 100)
    assert want.shape[0] > 1_100_000
    assert st["stored"] == want.shape[0]
    np.testing.assert_array_equal(got, want)


def test_photon_mapping_build_cornell(ctx):
    mesh = S.cornell_box(0)
    sc = S.Scene(ctx)
    sc.setMesh(mesh)
    sc.build()
    pmi = PhotonMapping(30000, 100, 1.0, 100, 0, 100, ctx=ctx)
    stats = pmi.build(sc, seed=5)
    got = pmi.getPhotonMapPtr().photons()
    want, _ = O.OracleScene(mesh).trace(0, 5, 0, 30000, 100)
    np.testing.assert_array_equal(got, want)
    assert stats["global"]["stored"] == want.shape[0]
    # photons lie on the room's surfaces, inside [0,1]^3
    assert np.all(got[:, 3:6] >= -1e-6) and np.all(got[:, 3:6] <= 1 + 1e-6)
    # with final gathering off the caustics map is empty
    assert pmi.caustics_map.getNPhotons() == 0

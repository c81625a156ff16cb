"""Scene generators and the OBJ/MTL reader (no GPU)."""
from __future__ import annotations

import numpy as np

from oracle import oracle as O
from photon_mapping_b200 import scene as S


def test_cornell_box_layout():
    m = S.cornell_box(0)
    assert m.n_faces == 36  # 10 wall + 24 box + 2 light triangles
    lights = np.nonzero(m.materials["le"].sum(1) > 0)[0]
    assert len(lights) == 2
    np.testing.assert_allclose(m.materials["le"][lights[0]], S.LIGHT_LE)
    # every wall faces into the room
    g = S.loader_geometric_normals(m.vertices)[:, :3]
    c = m.vertices.reshape(-1, 3, 3).mean(1)
    walls = [i for i, n in enumerate(m.names) if n.endswith("Wall") or n in ("floor", "ceiling")]
    assert np.all(np.sum(g[walls] * (0.5 - c[walls]), axis=1) > 0)
    # the seed moves the boxes
    assert not np.array_equal(S.cornell_box(1).vertices, m.vertices)


def test_caustics_scene_size():
    m = S.caustics_scene(0, grid=512, subdiv=5)
    assert m.n_faces == 36 + 2 * 20480 + 2 * 511 * 511
    kinds = set(m.materials["type"].tolist())
    assert kinds == {S.PM_LAMBERT, S.PM_MIRROR, S.PM_GLASS}
    water = np.array(m.names) == "water"
    np.testing.assert_allclose(m.materials["ior"][water], 1.33, rtol=1e-6)
    y = m.vertices[water][:, 1::3]
    assert y.max() - 0.22 <= 8 * 0.01 + 1e-6


def test_obj_round_trip(tmp_path):
    m = S.caustics_scene(0, grid=16, subdiv=1)
    S.write_obj(m, tmp_path / "scene.obj")
    m2 = S.load_obj(tmp_path / "scene.obj")
    np.testing.assert_array_equal(m.vertices, m2.vertices)
    np.testing.assert_array_equal(m.normals, m2.normals)
    np.testing.assert_array_equal(m.materials, m2.materials)
    assert m.names == m2.names


def test_obj_loader_rules(tmp_path):
    """scene.h:15-51 and :182-196: default material, geometric normals,
    illum 5/7, emission, polygon triangulation."""
    (tmp_path / "t.mtl").write_text(
        "newmtl m5\nKd 0.1 0.2 0.3\nillum 5\n\nnewmtl m7\nKd 0.5 0.5 0.5\nNi 1.5\nillum 7\n\n"
        "newmtl lamp\nKd 0.4 0.4 0.4\nKe 1 2 3\nillum 2\n")
    (tmp_path / "t.obj").write_text(
        "mtllib t.mtl\nv 0 0 0\nv 1 0 0\nv 1 1 0\nv 0 1 0\n"
        "f 1 2 3\nusemtl m5\nf 1 2 3\nusemtl m7\nf 1 2 3 4\nusemtl lamp\nf 1 2 3\n")
    m = S.load_obj(tmp_path / "t.obj")
    assert m.n_faces == 5
    assert m.materials["type"].tolist() == [S.PM_LAMBERT, S.PM_MIRROR, S.PM_GLASS, S.PM_GLASS,
                                            S.PM_LAMBERT]
    np.testing.assert_allclose(m.materials["rho"][0], 0.9)
    np.testing.assert_allclose(m.materials["rho"][1], 1.0)
    np.testing.assert_allclose(m.materials["ior"][2], 1.5)
    np.testing.assert_allclose(m.materials["le"][4], [1, 2, 3])
    np.testing.assert_array_equal(m.normals[0], [0, 0, 1] * 3)
    np.testing.assert_array_equal(m.vertices[3], [0, 0, 0, 1, 1, 0, 0, 1, 0])


def test_oracle_sincos_accuracy():
    x = np.random.default_rng(0).uniform(0.0, 6.2832, 200000).astype(np.float32)
    s, c = O.sincos(x)
    xd = x.astype(np.float64)
    # within one float ulp of the exact value
    assert np.all(np.abs(s - np.sin(xd)) <= np.spacing(np.abs(np.sin(xd)).astype(np.float32)) + 1e-45)
    assert np.all(np.abs(c - np.cos(xd)) <= np.spacing(np.abs(np.cos(xd)).astype(np.float32)) + 1e-45)


def test_oracle_intersect_basic():
    m = S.cornell_box(0, boxes=False)
    sc = O.OracleScene(m)
    r = np.array([[0.5, 0.5, 0.5, 1e-5, 0, -1, 0, 1e30]], np.float32)
    h = sc.intersect(r)
    assert abs(h[0, 0] - 0.5) < 1e-6 and m.names[h[0, 3].view(np.int32)] == "floor"


def test_batch_scene_generator():
    """Scenes of the batched benchmark: triangle count in range (the floor
    grid plus 1-40 boxes), settings in range, reproducible from the seed."""
    from photon_mapping_b200 import batch as B
    for seed in range(4):
        sc = B.random_scene(seed)
        assert 450 <= sc["mesh"].n_faces <= 520_000
        assert 100_000 <= sc["photons"] <= 4_000_000
        assert 128 <= sc["width"] == sc["height"] <= 1024
        assert sc["k"] in (50, 100)
        again = B.random_scene(seed)
        assert np.array_equal(again["mesh"].vertices, sc["mesh"].vertices)
        assert sum(1 for nm in sc["mesh"].names if nm == "light") == 2

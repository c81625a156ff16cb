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
    """The float sin/cos of the cosine-hemisphere draw (the oracle's copy of
    the device's sincos_f32): within 2 float ulps of the exact value over
    [-8, 8], and near the multiples of pi/2, where the reduction cancels."""
    rng = np.random.default_rng(0)
    near = (np.arange(-5, 6)[:, None] * (np.pi / 2) + np.linspace(-1e-5, 1e-5, 401)[None, :])
    x = np.concatenate([rng.uniform(0.0, 6.2832, 200000), rng.uniform(-8, 8, 100000),
                        near.ravel()]).astype(np.float32)
    s, c = O.sincos(x)
    xd = x.astype(np.float64)
    for got, want in ((s, np.sin(xd)), (c, np.cos(xd))):
        ulp = np.spacing(np.abs(want).astype(np.float32)).astype(np.float64)
        assert np.all(np.abs(got - want) <= 2 * ulp + 1e-45)
    # the same formulas in numpy float32 (one rounding per operation) agree bit for bit
    f = np.float32
    q = np.rint(x * f(float.fromhex("0x1.45f306p-1")))
    r = x - q * f(float.fromhex("0x1.921fbp+0"))
    r = r - q * f(float.fromhex("0x1.5110bp-22"))
    r = r - q * f(float.fromhex("0x1.184698p-44"))
    r2 = r * r
    ps = f(1 / 362880) * r2 + f(-1 / 5040)
    ps = (ps * r2 + f(1 / 120)) * r2 + f(-1 / 6)
    sr = r + (r * r2) * ps
    pc = f(-1 / 3628800) * r2 + f(1 / 40320)
    pc = ((pc * r2 + f(-1 / 720)) * r2 + f(1 / 24)) * r2 + f(-0.5)
    cr = f(1) + r2 * pc
    quad = q.astype(np.int32) & 3
    np.testing.assert_array_equal(s, np.select([quad == 0, quad == 1, quad == 2], [sr, cr, -sr], -cr))
    np.testing.assert_array_equal(c, np.select([quad == 0, quad == 1, quad == 2], [cr, -sr, -cr], sr))


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

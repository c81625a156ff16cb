"""The oracle's camera pass and path tracer against the reference's own
Scene / PhotonMapping / PathTracing (include/scene.h, include/integrator.h,
compiled unchanged into oracle/_ref/libpmref_integrator.so over the
project's Embree-3 and tinyobjloader stand-ins).

Given the same photon maps, both camera passes draw the same per-pixel
random streams (UniformSampler(j + width*i), examples/main.cpp:37), so the
images agree per pixel: exactly where no direction is sampled from a sine
or cosine (no final gathering), and to float rounding of sin/cos where one
is. Photon tracing itself is compared statistically: the reference seeds
one sampler per OpenMP thread (integrator.h:397-401), so its photon set
depends on the thread count.
"""
from __future__ import annotations

import numpy as np
import pytest

from oracle import oracle as O
from photon_mapping_b200 import scene as S
from photon_mapping_b200.camera import Camera

pytestmark = pytest.mark.skipif(not O.ref_integrator_available(),
                                reason="reference integrator not built")

W = H = 32
K = 50


def _scenes(tmp_path, which):
    mesh = S.caustics_scene(0, grid=12, subdiv=2) if which == "caustics" else S.cornell_box(0)
    path = tmp_path / f"{which}.obj"
    S.write_obj(mesh, path)
    return mesh, O.RefIntegrator(path)


def _cam():
    c = S.CAMERA
    return c["position"], c["forward"], c["fov"]


@pytest.mark.parametrize("which,fg,rtol", [
    ("cornell", 0, 0.0),        # no sampled directions: bit-exact
    ("caustics", 0, 0.0),
    ("cornell", 4, 1e-4),       # final gathering samples cos-weighted directions
    ("caustics", 1, 1e-3),
])
def test_camera_pass_matches_reference_per_pixel(tmp_path, which, fg, rtol):
    mesh, ref = _scenes(tmp_path, which)
    osc = O.OracleScene(mesh)
    n = 20000
    g, _ = osc.trace(0, 3, 0, n, 100)
    c, _ = osc.trace(1, 4, 0, n, 100) if fg else (np.zeros((0, 9), np.float32), None)
    ref.set_maps(g, c, n, K, 1.0, K, fg, 100)
    pos, fwd, fov = _cam()
    want, _ = ref.render(pos, fwd, fov, W, H, 4)
    got, dropped = osc.render(g, n, c, n, Camera(pos, fwd, fov).as_array(), W, H, 4, K, K, fg, 100)
    assert np.isfinite(got).all()
    if rtol == 0.0:
        np.testing.assert_array_equal(got, want)
    else:
        np.testing.assert_allclose(got, want, rtol=rtol, atol=1e-6)
        rel = np.abs(got - want) / np.maximum(np.abs(want), 1e-6)
        assert np.quantile(rel, 0.99) < 2e-5
    np.testing.assert_allclose(got.mean(axis=(0, 1)), want.mean(axis=(0, 1)), rtol=1e-5)


def test_path_tracing_matches_reference_per_pixel(tmp_path):
    mesh, ref = _scenes(tmp_path, "caustics")
    pos, fwd, fov = _cam()
    want, _ = ref.render_pt(pos, fwd, fov, W, H, 32, 100)
    got, dropped = O.OracleScene(mesh).render_pt(Camera(pos, fwd, fov).as_array(), W, H, 32, 100)
    assert dropped == 0
    np.testing.assert_allclose(got, want, rtol=1e-3, atol=1e-6)
    rel = np.abs(got - want) / np.maximum(np.abs(want), 1e-6)
    assert (rel > 1e-5).mean() < 5e-3


@pytest.mark.parametrize("which,fg", [("cornell", 0), ("caustics", 1)])
def test_traced_photon_maps_agree_statistically(tmp_path, which, fg):
    """The reference's own photon tracing + camera pass vs the oracle's
    tracing + camera pass: image means per channel within 2 %, 8x8-pixel
    block means within 10 % of the image mean, and stored photons per
    emitted photon within 2 %."""
    mesh, ref = _scenes(tmp_path, which)
    n = 50000
    ref.build(n, K, 1.0, K, fg, 100)
    pos, fwd, fov = _cam()
    want, _ = ref.render(pos, fwd, fov, W, H, 16)
    osc = O.OracleScene(mesh)
    g, _ = osc.trace(0, 3, 0, n, 100)
    c, _ = osc.trace(1, 4, 0, n, 100) if fg else (np.zeros((0, 9), np.float32), None)
    got, _ = osc.render(g, n, c, n, Camera(pos, fwd, fov).as_array(), W, H, 16, K, K, fg, 100)
    assert abs(len(g) / ref.n_photons() - 1.0) < 0.02
    m_got, m_want = got.mean(axis=(0, 1)), want.mean(axis=(0, 1))
    np.testing.assert_allclose(m_got, m_want, rtol=0.02)
    b = 8
    bg = got.reshape(H // b, b, W // b, b, 3).mean(axis=(1, 3))
    bw = want.reshape(H // b, b, W // b, b, 3).mean(axis=(1, 3))
    assert (np.abs(bg - bw) / m_want).max() < 0.10

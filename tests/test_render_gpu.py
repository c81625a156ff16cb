"""Parity of the device camera pass (pm_render) with the oracle's
restatement of the reference's render loop and integrator.

Both take the same traced photon maps and the same per-pixel random
streams, so the control flow is identical; images agree per pixel up to
the order of float sums (tolerance below).
"""
from __future__ import annotations

import numpy as np
import pytest

from oracle import oracle as O
from photon_mapping_b200 import scene as S
from photon_mapping_b200.camera import Camera
from photon_mapping_b200.integrator import PhotonMapping

pytestmark = pytest.mark.gpu

RTOL = 2e-5   # per pixel and channel, relative (float sum order only)
ATOL = 1e-6


def setup(ctx, mesh, n_photons, k, fg_depth, max_depth, mult=1.0, seed=3):
    sc = S.Scene(ctx)
    sc.setMesh(mesh)
    sc.build()
    pmi = PhotonMapping(n_photons, k, mult, k, fg_depth, max_depth, ctx=ctx)
    pmi.build(sc, seed=seed)
    return pmi


def oracle_render(mesh, pmi, cam, w, h, spp, n_gather=1):
    g = pmi.global_map.photons()
    c = pmi.caustics_map.photons()
    return O.OracleScene(mesh).render(g, pmi.nPhotonsGlobal, c, pmi.nPhotonsCaustics,
                                      cam.as_array(), w, h, spp, pmi.nEstimationGlobal,
                                      pmi.nEstimationGlobal, pmi.finalGatheringDepth,
                                      pmi.maxDepth, n_gather)


def assert_images_close(got, want):
    np.testing.assert_array_equal(np.isfinite(got), np.isfinite(want))
    np.testing.assert_allclose(got, want, rtol=RTOL, atol=ATOL)


def test_cornell_no_final_gathering(ctx):
    mesh = S.cornell_box(0)
    pmi = setup(ctx, mesh, 20000, 50, 0, 100)
    cam = Camera(S.CAMERA["position"], S.CAMERA["forward"], S.CAMERA["fov"])
    img, st = pmi.render(cam, 40, 32, 3)
    want, dropped = oracle_render(mesh, pmi, cam, 40, 32, 3)
    assert_images_close(img, want)
    assert st["dropped_nan"] == dropped[0] and st["dropped_negative"] == dropped[1]
    assert st["queries_caustics"] == 0 and st["queries_global"] > 0
    assert img.mean() > 0


def test_cornell_final_gathering(ctx):
    mesh = S.cornell_box(1)
    pmi = setup(ctx, mesh, 20000, 40, 1, 20)
    cam = Camera(S.CAMERA["position"], S.CAMERA["forward"], S.CAMERA["fov"])
    img, st = pmi.render(cam, 24, 24, 2, spp_batch=1)
    want, dropped = oracle_render(mesh, pmi, cam, 24, 24, 2)
    assert_images_close(img, want)
    assert st["passes"] == 2


def test_caustics_scene_specular_branches(ctx):
    mesh = S.caustics_scene(0, grid=24, subdiv=2)
    pmi = setup(ctx, mesh, 20000, 30, 1, 12, mult=2.0)
    assert pmi.caustics_map.getNPhotons() > 0
    cam = Camera(S.CAMERA["position"], S.CAMERA["forward"], S.CAMERA["fov"])
    img, st = pmi.render(cam, 24, 20, 2)
    want, dropped = oracle_render(mesh, pmi, cam, 24, 20, 2)
    assert_images_close(img, want)
    assert st["queries_caustics"] > 0


def test_multiple_gather_rays(ctx):
    mesh = S.cornell_box(2)
    pmi = setup(ctx, mesh, 10000, 20, 1, 10)
    cam = Camera(S.CAMERA["position"], S.CAMERA["forward"], S.CAMERA["fov"])
    img, st = pmi.render(cam, 16, 16, 2, n_gather=4)
    want, _ = oracle_render(mesh, pmi, cam, 16, 16, 2, n_gather=4)
    np.testing.assert_allclose(img, want, rtol=1e-4, atol=1e-6)


def test_path_tracing_matches_oracle(ctx):
    from photon_mapping_b200.integrator import PathTracing
    for mesh in (S.cornell_box(4), S.caustics_scene(0, grid=16, subdiv=2)):
        sc = S.Scene(ctx)
        sc.setMesh(mesh)
        sc.build()
        cam = Camera(S.CAMERA["position"], S.CAMERA["forward"], S.CAMERA["fov"])
        pt = PathTracing(30, ctx=ctx)
        img, dropped = pt.render(cam, 32, 24, 8)
        want, wd = O.OracleScene(mesh).render_pt(cam.as_array(), 32, 24, 8, 30)
        # same per-sample arithmetic and the same per-pixel sum order
        np.testing.assert_array_equal(img, want)
        assert dropped == wd


def test_photon_mapping_converges_to_path_tracing(ctx):
    """Image-level check (oracle part iii): the photon-map render and the
    path-traced image of the same scene agree in the mean (photon mapping's
    only bias is the kNN blur) and per pixel up to noise. Pixels seeing the
    light (Le = 17) are left out of the per-pixel figure: their value is
    the fraction of samples landing on the light, noisy at low spp."""
    from photon_mapping_b200.integrator import PathTracing
    mesh = S.cornell_box(0)
    sc = S.Scene(ctx)
    sc.setMesh(mesh)
    sc.build()
    cam = Camera(S.CAMERA["position"], S.CAMERA["forward"], S.CAMERA["fov"])
    ref, _ = PathTracing(100, ctx=ctx).render(cam, 64, 64, 8192)
    mask = ref.max(axis=2) < 1.0
    for fg, spp in ((1, 64), (0, 16)):
        pmi = PhotonMapping(1000000, 100, 1.0, 100, fg, 100, ctx=ctx)
        pmi.build(sc, seed=9)
        img, _ = pmi.render(cam, 64, 64, spp, n_gather=16)
        err = (img - ref)[mask]
        bias = float(err.mean()) / float(ref[mask].mean())
        rel = float(np.sqrt(np.mean(err ** 2))) / float(ref[mask].mean())
        print(f"final gathering {fg}: mean bias {bias:+.4f}, relative RMSE {rel:.3f}")
        assert abs(bias) < 0.02
        assert rel < 0.3


@pytest.mark.parametrize("fg", [0, 1])
def test_integrate_rays_match_oracle(ctx, fg):
    """pm_integrate: arbitrary rays with their samplers' states; the radiance
    matches the oracle and the states advance by the same draws."""
    mesh = S.caustics_scene(0, grid=24, subdiv=2)
    pmi = setup(ctx, mesh, 20000, 30, fg, 12, mult=2.0)
    rng = np.random.default_rng(5)
    n = 3000
    o = rng.uniform(0.05, 0.95, (n, 3)).astype(np.float32)
    d = rng.normal(size=(n, 3))
    d = (d / np.linalg.norm(d, axis=1, keepdims=True)).astype(np.float32)
    states = rng.integers(0, 2**63, n, dtype=np.uint64)
    got, gst = pmi.integrate_batch(o, d, states)
    want, wst = O.OracleScene(mesh).integrate(
        pmi.global_map.photons(), pmi.nPhotonsGlobal, pmi.caustics_map.photons(),
        pmi.nPhotonsCaustics, np.concatenate([o, d], axis=1), states, pmi.nEstimationGlobal,
        pmi.nEstimationGlobal, pmi.finalGatheringDepth, pmi.maxDepth)
    np.testing.assert_array_equal(gst, wst)
    np.testing.assert_allclose(got, want, rtol=RTOL, atol=ATOL)


needs_ref = pytest.mark.skipif(not O.ref_integrator_available(),
                               reason="reference integrator not built")


@needs_ref
@pytest.mark.parametrize("fg", [0, 1])
def test_render_matches_reference_integrator(ctx, tmp_path, fg):
    """pm_render against the reference's own PhotonMapping::integrate in the
    loop of examples/main.cpp (compiled unchanged on the host), both over
    the photon maps traced on the device: per pixel to float rounding (the
    reference's sin/cos in sampled directions), bit-exact without final
    gathering up to the device's sum order."""
    mesh = S.caustics_scene(0, grid=32, subdiv=3)
    pmi = setup(ctx, mesh, 100000, 100, fg, 100)
    path = tmp_path / "scene.obj"
    S.write_obj(mesh, path)
    ref = O.RefIntegrator(path)
    ref.set_maps(pmi.global_map.photons(), pmi.caustics_map.photons(), pmi.nPhotonsGlobal,
                 100, 1.0, 100, fg, 100)
    c = S.CAMERA
    want, _ = ref.render(c["position"], c["forward"], c["fov"], 64, 64, 4)
    got, _ = pmi.render(Camera(c["position"], c["forward"], c["fov"]), 64, 64, 4)
    if fg == 0:
        np.testing.assert_allclose(got, want, rtol=2e-5, atol=1e-6)
    # a rounding change in a sampled direction can move a gather ray's hit
    # point and with it one sample's neighbour set: a few pixels differ by
    # up to about 1e-3 relative
    np.testing.assert_allclose(got, want, rtol=2e-2, atol=1e-6)
    rel = np.abs(got - want) / np.maximum(np.abs(want), 1e-6)
    assert np.quantile(rel, 0.99) < 5e-5
    np.testing.assert_allclose(got.mean(axis=(0, 1)), want.mean(axis=(0, 1)), rtol=2e-5)


@needs_ref
def test_path_tracing_matches_reference_integrator(ctx, tmp_path):
    from photon_mapping_b200.integrator import PathTracing
    mesh = S.caustics_scene(0, grid=32, subdiv=3)
    sc = S.Scene(ctx)
    sc.setMesh(mesh)
    sc.build()
    path = tmp_path / "scene.obj"
    S.write_obj(mesh, path)
    c = S.CAMERA
    want, _ = O.RefIntegrator(path).render_pt(c["position"], c["forward"], c["fov"], 48, 48, 16,
                                              100)
    got, _ = PathTracing(100, ctx=ctx).render(Camera(c["position"], c["forward"], c["fov"]),
                                               48, 48, 16)
    # the reference samples directions with std::sin/cos, the device with
    # its own sincos: paths agree, contributions differ by float rounding
    np.testing.assert_allclose(got, want, rtol=1e-3, atol=1e-6)
    rel = np.abs(got - want) / np.maximum(np.abs(want), 1e-6)
    assert (rel > 1e-5).mean() < 5e-3


def test_fp64_accumulation_check(ctx):
    """PM_RENDER_FP64_CHECK: the same image, and the FP32 per-pixel sums
    within float rounding of FP64 sums of the same samples."""
    mesh = S.cornell_box(0)
    pmi = setup(ctx, mesh, 30000, 40, 1, 100)
    cam = Camera(S.CAMERA["position"], S.CAMERA["forward"], S.CAMERA["fov"])
    plain, st0 = pmi.render(cam, 48, 40, 16)
    img, st = pmi.render(cam, 48, 40, 16, fp64_check=True)
    np.testing.assert_array_equal(img, plain)
    assert st0["accum_rel_err"] == 0.0
    assert 0.0 < st["accum_rel_err"] < 1e-5
    # several passes accumulate into the same sums
    img2, st2 = pmi.render(cam, 48, 40, 16, spp_batch=3, fp64_check=True)
    np.testing.assert_array_equal(img2, plain)
    assert st2["passes"] == 6 and st2["accum_rel_err"] < 1e-5

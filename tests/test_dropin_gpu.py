"""The drop-in C++ API on the GPU: a C++ program written against the
reference's interface (tests/cpp/dropin_render.cpp) renders ray by ray and
in one call; both agree with each other and with the Python front end."""
from __future__ import annotations

import subprocess

import numpy as np
import pytest

from photon_mapping_b200 import scene as S
from photon_mapping_b200.camera import Camera
from photon_mapping_b200.integrator import PhotonMapping
from tests.dropin_build import ROOT, compile_dropin

pytestmark = pytest.mark.gpu


def test_dropin_program_matches_python(ctx, tmp_path):
    exe = tmp_path / "dropin_render"
    compile_dropin(ROOT / "tests" / "cpp" / "dropin_render.cpp", exe)
    mesh = S.caustics_scene(0, grid=12, subdiv=1)
    S.write_obj(mesh, tmp_path / "scene.obj")
    w, h, spp = 20, 16, 2
    r = subprocess.run([str(exe), "scene.obj", str(w), str(h), str(spp), "out"], cwd=tmp_path,
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr

    def load(name, dtype=np.float32, shape=(h, w, 3)):
        return np.fromfile(tmp_path / name, dtype=dtype).reshape(shape)

    perray, batched = load("out_perray.f32"), load("out_batched.f32")
    # the same samples, summed per pixel in the same order
    np.testing.assert_allclose(perray, batched, rtol=2e-5, atol=1e-6)
    np.testing.assert_allclose(load("out_pt_perray.f32"), load("out_pt_batched.f32"), rtol=1e-6,
                               atol=0)
    # the Python front end on the same OBJ, camera and parameters
    sc = S.Scene(ctx)
    sc.loadModel(tmp_path / "scene.obj")
    sc.build()
    pmi = PhotonMapping(20000, 30, 1.0, 30, 1, 12, ctx=ctx)
    pmi.build(sc, seed=1)
    cam = Camera((0.5, 0.5, 4.7), (0, 0, -1), 0.25 * 3.14159265359)
    img, _ = pmi.render(cam, w, h, spp)
    np.testing.assert_array_equal(img, batched)
    # k = 1 lookups return real photons with throughput copied into the image
    idx = load("out_nearest_idx.i32", np.int32, (h, w))
    ph = pmi.global_map.photons()
    near = load("out_nearest.f32")
    hit = idx >= 0
    assert hit.mean() > 0.5
    np.testing.assert_array_equal(near[hit], ph[idx[hit], 0:3])

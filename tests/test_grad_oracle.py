"""The oracle's FP64 gradient of the photon-mapping image loss (forward
differentiation through photon tracing and the camera pass) against
central finite differences of the oracle's own render.

With max_depth = 2 every photon is stored before Russian roulette can stop
it (integrator.h:431-449: the store at bounce 1 precedes the roulette), so
the plain render is a smooth function of the albedos and the finite
differences need no frozen decisions. CPU only.
"""
from __future__ import annotations

import numpy as np

from oracle import oracle as O
from photon_mapping_b200 import differentiable as D
from photon_mapping_b200 import scene as S
from photon_mapping_b200.camera import Camera

W, H, SPP, K, FG, MD, NG = 24, 20, 2, 20, 1, 2, 2
N_PHOTONS, SEED = 4000, 5
H_STEP = 1e-3


def oracle_image(mesh0, fp, albedo, emission, cam):
    mesh = D.apply_parameters(mesh0, fp, albedo, emission)
    osc = O.OracleScene(mesh)
    g, _ = osc.trace(0, SEED, 0, N_PHOTONS, MD)
    c, _ = osc.trace(1, SEED + 1, 0, N_PHOTONS, MD)
    img, _ = osc.render(g, N_PHOTONS, c, N_PHOTONS, cam.as_array(), W, H, SPP, K, K, FG, MD, NG)
    osc.close()
    return img


def test_oracle_gradient_matches_finite_differences():
    mesh0 = S.cornell_box(0)
    fp = D.face_parameters(mesh0)
    a0, e0 = D.base_parameters(mesh0, fp, len(D.CORNELL_MATERIALS))
    cam = Camera(S.CAMERA["position"], S.CAMERA["forward"], S.CAMERA["fov"])
    ta, te = D.perturbed_parameters(a0, e0, seed=11)
    target = oracle_image(mesh0, fp, ta, te, cam).astype(np.float64)
    img0 = oracle_image(mesh0, fp, a0, e0, cam)
    gimg = (2.0 / img0.size) * (img0.astype(np.float64) - target)
    osc = O.OracleScene(D.apply_parameters(mesh0, fp, a0, e0))
    ga, ge, img = osc.grad(fp, len(a0), SEED, N_PHOTONS, N_PHOTONS, cam.as_array(), W, H, SPP,
                           K, FG, MD, NG, gimg)
    np.testing.assert_array_equal(img, img0)   # the same render
    grad = np.concatenate([ga, ge[None]], axis=0)
    theta = np.concatenate([a0, e0[None]], axis=0).astype(np.float64)
    fd = np.zeros_like(grad)
    for p in range(grad.shape[0]):
        for c in range(3):
            vals = []
            for sgn in (1.0, -1.0):
                th = theta.copy()
                th[p, c] += sgn * H_STEP
                th32 = th.astype(np.float32)
                im = oracle_image(mesh0, fp, th32[:-1], th32[-1], cam).astype(np.float64)
                vals.append(np.mean((im - target) ** 2))
            hp = float(np.float32(theta[p, c] + H_STEP)) - float(np.float32(theta[p, c] - H_STEP))
            fd[p, c] = (vals[0] - vals[1]) / hp
    scale = np.abs(grad).max()
    assert scale > 0
    np.testing.assert_allclose(grad, fd, rtol=2e-3, atol=2e-3 * scale)

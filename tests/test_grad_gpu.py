"""The device adjoint of the differentiable render (pm_diff_forward /
pm_diff_backward) against the oracle's FP64 forward-mode gradient, against
central finite differences on the device (decisions frozen at the base
point), and through the torch.autograd.Function.

Tolerances: the device sums the adjoint in float per block and in double
across blocks; the oracle sums in double. 1e-3 relative per component, with
an absolute floor of 1e-4 of the largest component (components near zero).
The finite differences (step 1e-3, float32 images, the loss in double) are
held to 5e-3 relative with a floor of 5e-3 of the largest component.
"""
from __future__ import annotations

import numpy as np
import pytest

from oracle import oracle as O
from photon_mapping_b200 import differentiable as D
from photon_mapping_b200 import scene as S
from photon_mapping_b200._native import PMError
from photon_mapping_b200.camera import Camera
from photon_mapping_b200.integrator import PhotonMapping

pytestmark = pytest.mark.gpu

NP = len(D.CORNELL_MATERIALS)


def camera():
    return Camera(S.CAMERA["position"], S.CAMERA["forward"], S.CAMERA["fov"])


def stack(ga, ge):
    return np.concatenate([np.asarray(ga, np.float64), np.asarray(ge, np.float64)[None]])


def test_forward_is_the_plain_render(ctx):
    """With decisions equal to the parameters, pm_diff_forward renders what
    PhotonMapping.build + render give (same seeds, same streams)."""
    mesh = S.cornell_box(0)
    cam = camera()
    r = D.DiffRenderer(ctx, mesh, cam, 32, 24, 3, 20000, 30, final_gathering_depth=1,
                       max_depth=100, n_gather=2, seed=7)
    a0, e0 = r.base()
    img = r.forward(a0, e0)
    pmi = PhotonMapping(20000, 30, 1.0, 30, 1, 100, ctx=ctx)
    pmi.build(r.scene, seed=7)
    want, _ = pmi.render(cam, 32, 24, 3, n_gather=2)
    np.testing.assert_array_equal(img, want)


@pytest.mark.parametrize("fg,n_gather,md", [(1, 2, 100), (0, 1, 100), (1, 1, 6)])
def test_gradient_matches_oracle_fp64(ctx, fg, n_gather, md):
    mesh0 = S.cornell_box(3)
    fp = D.face_parameters(mesh0)
    cam = camera()
    W, H, SPP, K, NPH, SEED = 24, 20, 2, 20, 6000, 5
    r = D.DiffRenderer(ctx, mesh0, cam, W, H, SPP, NPH, K, final_gathering_depth=fg,
                       max_depth=md, n_gather=n_gather, seed=SEED)
    a0, e0 = r.base()
    a1, e1 = D.perturbed_parameters(a0, e0, seed=3, amount=0.1)
    ta, te = D.perturbed_parameters(a0, e0, seed=4)
    target = r.forward(ta, te).astype(np.float64)
    img = r.forward(a1, e1)
    gimg = (2.0 / img.size) * (img.astype(np.float64) - target)
    ga, ge = r.backward(gimg)
    osc = O.OracleScene(D.apply_parameters(mesh0, fp, a1, e1))
    oa, oe, oimg = osc.grad(fp, NP, SEED, NPH, NPH, cam.as_array(), W, H, SPP, K, fg, md,
                            n_gather, gimg.astype(np.float32))
    np.testing.assert_allclose(img, oimg, rtol=2e-5, atol=1e-6)
    got, want = stack(ga, ge), stack(oa, oe)
    scale = np.abs(want).max()
    assert scale > 0
    np.testing.assert_allclose(got, want, rtol=1e-3, atol=1e-4 * scale)


def test_gradient_matches_finite_differences(ctx):
    """The gradient benchmark's shape at reduced size: Cornell box, final gathering, k = 50,
    full path depth (Russian roulette active, decisions frozen)."""
    mesh0 = S.cornell_box(0)
    r = D.DiffRenderer(ctx, mesh0, camera(), 48, 48, 4, 100000, 50, final_gathering_depth=1,
                       max_depth=100, n_gather=1, seed=2)
    a0, e0 = r.base()
    ta, te = D.perturbed_parameters(a0, e0, seed=8)
    target = r.forward(ta, te).astype(np.float64)
    loss, ga, ge, _ = r.loss_and_grad(a0, e0, target)
    assert loss > 0
    fd = r.finite_differences(a0, e0, target, h=1e-3)
    got = stack(ga, ge)
    scale = np.abs(got).max()
    np.testing.assert_allclose(got, fd, rtol=5e-3, atol=5e-3 * scale)


def test_two_backwards_agree_and_autograd(ctx):
    import torch
    mesh0 = S.cornell_box(1)
    r = D.DiffRenderer(ctx, mesh0, camera(), 32, 32, 2, 30000, 40, final_gathering_depth=1,
                       max_depth=100, seed=4)
    a0, e0 = r.base()
    ta, te = D.perturbed_parameters(a0, e0, seed=9)
    target = r.forward(ta, te).astype(np.float64)
    loss, ga, ge, img = r.loss_and_grad(a0, e0, target)
    gimg = (2.0 / img.size) * (img.astype(np.float64) - target)
    ga2, ge2 = r.backward(gimg)      # the same forward, differentiated again
    # float atomics sum in a different order each time
    scale = max(np.abs(ga).max(), np.abs(ge).max())
    np.testing.assert_allclose(ga, ga2, rtol=1e-5, atol=1e-6 * scale)
    np.testing.assert_allclose(ge, ge2, rtol=1e-5, atol=1e-6 * scale)
    alb = torch.tensor(a0, requires_grad=True)
    em = torch.tensor(e0, requires_grad=True)
    out = D.render(alb, em, r)
    tl = ((out.double() - torch.from_numpy(target)) ** 2).mean()
    tl.backward()
    np.testing.assert_allclose(float(tl), loss, rtol=1e-12)
    np.testing.assert_allclose(alb.grad.numpy(), ga, rtol=1e-5, atol=1e-6 * scale)
    np.testing.assert_allclose(em.grad.numpy(), ge, rtol=1e-5, atol=1e-6 * scale)


def test_errors(ctx):
    mesh0 = S.cornell_box(0)
    r = D.DiffRenderer(ctx, mesh0, camera(), 8, 8, 1, 1000, 10, seed=1)
    a0, e0 = r.base()
    with pytest.raises(PMError):           # no forward yet on this scene
        r.backward(np.zeros((8, 8, 3), np.float32))
    bad = a0.copy()
    bad[2, 1] = 0.0
    with pytest.raises(PMError):           # parameters must be positive
        r.forward(bad, e0)
    r.forward(a0, e0)
    r.backward(np.ones((8, 8, 3), np.float32))
    pmi = PhotonMapping(1000, 10, 1.0, 10, 0, 10, ctx=ctx)
    pmi.build(r.scene, seed=1)             # the maps change: the pass is gone
    with pytest.raises(PMError):
        r.backward(np.ones((8, 8, 3), np.float32))
    fp = D.face_parameters(mesh0)
    lib = ctx.lib
    assert lib.pm_diff_set_parameters(ctx.handle, fp.ctypes.data, fp.shape[0] - 1, NP) != 0
    fp2 = fp.copy()
    fp2[0] = NP
    assert lib.pm_diff_set_parameters(ctx.handle, fp2.ctypes.data, fp2.shape[0], NP) != 0
    # a specular face cannot carry an albedo parameter
    cs = S.caustics_scene(0, grid=8, subdiv=1)
    sc = S.Scene(ctx)
    sc.setMesh(cs)
    sc.build()
    fp3 = np.zeros(cs.n_faces, np.int32)
    assert lib.pm_diff_set_parameters(ctx.handle, fp3.ctypes.data, fp3.shape[0], 1) != 0

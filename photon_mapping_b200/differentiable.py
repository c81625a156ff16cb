"""Differentiable photon mapping: d(image loss) / d(per-material Lambert
albedo, light emission) through the photon-map density estimate
(integrator.h:133-175) and final gathering (integrator.h:178-262).

The reference computes no gradients. `DiffRenderer` drives the C ABI's
pm_diff_forward / pm_diff_backward (include/pm_cuda.h): the forward pass
traces both photon maps and renders one image; the backward pass is a
hand-written adjoint on the device that runs the camera pass in reverse,
scatters each estimate's adjoint onto its k nearest photons and replays the
photon paths from their per-photon seeds (never stored).

Russian roulette in the photon trace (integrator.h:441-449) decides on the
throughput, which depends on the albedos; the forward pass takes those
decisions with separate "decision" parameters (by default the parameters
themselves), so that the image is a smooth function of the parameters with
the decisions held. The gradient is that of the estimator with frozen
decisions, and central finite differences taken with the decisions held at
the base point (`finite_differences`) measure the same function.

`RenderFunction` is the torch.autograd.Function over a DiffRenderer.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import scene as S
from ._native import Context
from .integrator import RenderStats

# the material names of the procedural Cornell box, in parameter order
CORNELL_MATERIALS = ("backWall", "ceiling", "floor", "leftWall", "light", "rightWall",
                     "shortBox", "tallBox")


class DiffParams(C.Structure):
    _fields_ = [("width", C.c_int32), ("height", C.c_int32), ("spp", C.c_int32),
                ("k", C.c_int32), ("final_gathering_depth", C.c_int32),
                ("max_depth", C.c_int32), ("n_gather", C.c_int32), ("reserved", C.c_int32),
                ("n_photons", C.c_int64), ("n_photons_caustics", C.c_int64),
                ("seed", C.c_uint64)]


def face_parameters(mesh: S.Mesh, names=CORNELL_MATERIALS) -> np.ndarray:
    """Albedo parameter of each face: the index of its material name in
    `names`, -1 for faces of other materials."""
    idx = {nm: i for i, nm in enumerate(names)}
    return np.array([idx.get(nm, -1) for nm in mesh.names], np.int32)


def base_parameters(mesh: S.Mesh, face_param: np.ndarray, n_params: int):
    """The mesh's own albedos per parameter and its emission."""
    albedo = np.zeros((n_params, 3), np.float32)
    for p in range(n_params):
        faces = np.nonzero(face_param == p)[0]
        if faces.size:
            albedo[p] = mesh.materials["rho"][faces[0]]
    le = mesh.materials["le"]
    lit = np.nonzero(le.max(axis=1) > 0)[0]
    emission = le[lit[0]].astype(np.float32) if lit.size else np.zeros(3, np.float32)
    return albedo, emission


def apply_parameters(mesh: S.Mesh, face_param: np.ndarray, albedo, emission) -> S.Mesh:
    """A copy of `mesh` with the parameters written into its materials (the
    host-side statement of what pm_diff_forward does on the device)."""
    mats = mesh.materials.copy()
    albedo = np.asarray(albedo, np.float32).reshape(-1, 3)
    sel = face_param >= 0
    mats["rho"][sel] = albedo[face_param[sel]]
    lit = mats["le"].max(axis=1) > 0
    mats["le"][lit] = np.asarray(emission, np.float32)
    return S.Mesh(mesh.vertices, mesh.normals, mats, list(mesh.names))


class DiffRenderer:
    """One scene, camera and render setting on a context, differentiable in
    the albedo parameters (face_param) and the emission.

    forward(albedo (P,3), emission (3,)) -> image (H, W, 3)
    backward(grad_image (H, W, 3)) -> (d/d albedo (P,3), d/d emission (3,))

    backward differentiates the most recent forward on this renderer; the
    context's camera buffers hold that pass, so any other render or photon
    map call on the context in between makes backward fail."""

    def __init__(self, ctx: Context, mesh: S.Mesh, camera, width: int, height: int, spp: int,
                 n_photons: int, k: int, final_gathering_depth: int = 1, max_depth: int = 100,
                 n_gather: int = 1, caustics_multiplier: float = 1.0, seed: int = 1,
                 face_param: np.ndarray | None = None, n_params: int | None = None):
        self.ctx = ctx
        self.mesh = mesh
        self.camera = camera
        self.face_param = (face_parameters(mesh) if face_param is None
                           else np.ascontiguousarray(face_param, np.int32))
        self.n_params = int(n_params if n_params is not None
                            else (self.face_param.max() + 1 if self.face_param.size else 0))
        self.scene = S.Scene(ctx)
        self.scene.setMesh(mesh)
        self.scene.build()
        ctx.check(ctx.lib.pm_diff_set_parameters(ctx.handle, self.face_param.ctypes.data,
                                                 self.face_param.shape[0], self.n_params),
                  "pm_diff_set_parameters")
        n_caustic = int(C.c_float(n_photons * C.c_float(caustics_multiplier).value).value)
        self.params = DiffParams(int(width), int(height), int(spp), int(k),
                                 int(final_gathering_depth), int(max_depth), int(n_gather), 0,
                                 int(n_photons), n_caustic, int(seed))
        self.shape = (int(height), int(width), 3)
        self.stats: dict = {}
        self._cam = camera.as_struct()
        self._forwards = 0
        self._grad_of = -1

    def base(self):
        return base_parameters(self.mesh, self.face_param, self.n_params)

    def forward(self, albedo, emission, decision_albedo=None, decision_emission=None):
        a = np.ascontiguousarray(albedo, np.float32).reshape(self.n_params, 3)
        e = np.ascontiguousarray(emission, np.float32).reshape(3)
        da = None if decision_albedo is None else np.ascontiguousarray(decision_albedo,
                                                                       np.float32)
        de = None if decision_emission is None else np.ascontiguousarray(decision_emission,
                                                                         np.float32)
        out = np.empty(self.shape, np.float32)
        st = RenderStats()
        lib = self.ctx.lib
        self.ctx.check(lib.pm_diff_forward(self.ctx.handle, C.addressof(self._cam),
                                           C.addressof(self.params), a.ctypes.data, e.ctypes.data,
                                           None if da is None else da.ctypes.data,
                                           None if de is None else de.ctypes.data,
                                           out.ctypes.data, C.addressof(st)),
                       "pm_diff_forward")
        self.stats = st.as_dict()
        self._forwards += 1
        return out

    def backward(self, grad_image):
        g = np.ascontiguousarray(grad_image, np.float32).reshape(self.shape)
        ga = np.empty((self.n_params, 3), np.float32)
        ge = np.empty(3, np.float32)
        self.ctx.check(self.ctx.lib.pm_diff_backward(self.ctx.handle, g.ctypes.data,
                                                     ga.ctypes.data, ge.ctypes.data),
                       "pm_diff_backward")
        return ga, ge

    def loss_and_grad(self, albedo, emission, target):
        """MSE over pixels and channels against `target`, and its gradient."""
        img = self.forward(albedo, emission)
        diff = img.astype(np.float64) - target
        loss = float(np.mean(diff * diff))
        ga, ge = self.backward((2.0 / diff.size) * diff)
        return loss, ga, ge, img

    def finite_differences(self, albedo, emission, target, h: float = 1e-3, which=None):
        """Central differences of the MSE loss with step h per parameter
        channel, every render with the Russian-roulette decisions held at
        (albedo, emission). which: list of (param, channel) with param ==
        n_params meaning the emission; default all. Returns (P+1, 3)."""
        a0 = np.asarray(albedo, np.float32).reshape(self.n_params, 3)
        e0 = np.asarray(emission, np.float32).reshape(3)
        theta0 = np.concatenate([a0, e0[None]], axis=0).astype(np.float64)
        out = np.full((self.n_params + 1, 3), np.nan)
        which = which or [(p, c) for p in range(self.n_params + 1) for c in range(3)]
        for p, c in which:
            vals = []
            for sgn in (1.0, -1.0):
                th = theta0.copy()
                th[p, c] += sgn * h
                th32 = th.astype(np.float32)
                img = self.forward(th32[:-1], th32[-1], a0, e0)
                d = img.astype(np.float64) - target
                vals.append(np.mean(d * d))
            # the step actually taken in float32
            hp = float(np.float32(theta0[p, c] + h)) - float(np.float32(theta0[p, c] - h))
            out[p, c] = (vals[0] - vals[1]) / hp
        return out


def _torch_function():
    import torch

    class RenderFunction(torch.autograd.Function):
        """image = render(albedo (P,3), emission (3,)) on a DiffRenderer;
        backward calls the device adjoint."""

        @staticmethod
        def forward(ctx, albedo, emission, renderer):
            img = renderer.forward(albedo.detach().cpu().numpy(), emission.detach().cpu().numpy())
            ctx.renderer = renderer
            ctx.generation = renderer._forwards
            ctx.device = albedo.device
            return torch.from_numpy(img).to(albedo.device)

        @staticmethod
        def backward(ctx, grad_img):
            r = ctx.renderer
            if r._forwards != ctx.generation:
                raise RuntimeError("RenderFunction: another forward ran on this renderer "
                                   "before backward")
            ga, ge = r.backward(grad_img.detach().float().cpu().numpy())
            return (torch.from_numpy(ga).to(ctx.device), torch.from_numpy(ge).to(ctx.device),
                    None)

    return RenderFunction


_RF = None


def render(albedo, emission, renderer: DiffRenderer):
    """Differentiable render of torch tensors albedo (P,3) and emission (3,)."""
    global _RF
    if _RF is None:
        _RF = _torch_function()
    return _RF.apply(albedo, emission, renderer)


def perturbed_parameters(albedo, emission, seed: int, amount: float = 0.2,
                         lo: float = 0.02, hi: float = 0.98):
    """Seed-drawn target parameters: every albedo channel moved by up to
    +-amount (kept in [lo, hi]) and the emission scaled by up to +-amount."""
    rng = np.random.default_rng(seed)
    a = np.clip(np.asarray(albedo, np.float64) + rng.uniform(-amount, amount, np.shape(albedo)),
                lo, hi)
    e = np.asarray(emission, np.float64) * (1.0 + rng.uniform(-amount, amount, 3))
    return a.astype(np.float32), e.astype(np.float32)

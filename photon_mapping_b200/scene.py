"""Scenes: procedural generators, OBJ/MTL files, and the device scene.

A scene is a `Mesh`: per-face unshared vertices (n, 9), per-face vertex
normals (n, 9) and per-face materials, the layout Scene::loadModel builds
(scene.h:107-270). `load_obj` reads OBJ/MTL with the reference loader's
rules (scene.h:15-51, :107-270); `write_obj` writes a mesh so that
`load_obj` returns it unchanged. `Scene` uploads a mesh to the device
(Scene::build, scene.h:275-304) and answers closest-hit queries
(Scene::intersect, scene.h:307-348).
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

from . import _native as N
from ._native import Context, ptr

PM_LAMBERT, PM_MIRROR, PM_GLASS = 0, 1, 2

MATERIAL_DTYPE = np.dtype([("type", np.int32), ("rho", np.float32, 3), ("ior", np.float32),
                           ("le", np.float32, 3)])
HIT_DTYPE = np.dtype([("t", np.float32), ("u", np.float32), ("v", np.float32),
                      ("prim", np.int32)])


def material(kind: int = PM_LAMBERT, rho=(0.9, 0.9, 0.9), ior: float = 1.0, le=(0.0, 0.0, 0.0)):
    m = np.zeros((), MATERIAL_DTYPE)
    m["type"], m["rho"], m["ior"], m["le"] = kind, rho, ior, le
    return m


@dataclass
class Mesh:
    vertices: np.ndarray                      # (n, 9) float32
    normals: np.ndarray                       # (n, 9) float32
    materials: np.ndarray                     # (n,) MATERIAL_DTYPE
    names: list = field(default_factory=list)  # material name per face ("" if none)

    @property
    def n_faces(self) -> int:
        return int(self.vertices.shape[0])

    def __add__(self, other: "Mesh") -> "Mesh":
        return Mesh(np.concatenate([self.vertices, other.vertices]),
                    np.concatenate([self.normals, other.normals]),
                    np.concatenate([self.materials, other.materials]),
                    list(self.names) + list(other.names))


def _f32(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.float32))


def loader_geometric_normals(v: np.ndarray) -> np.ndarray:
    """The normal Scene::loadModel gives a face without normals
    (scene.h:182-189): normalize(cross(normalize(v1-v0), normalize(v2-v0))),
    in float32, operation by operation."""
    v = _f32(v).reshape(-1, 3, 3)

    def normalize(a):
        ln = np.sqrt((a[:, 0] * a[:, 0] + a[:, 1] * a[:, 1]) + a[:, 2] * a[:, 2])
        return a / ln[:, None]

    e1 = normalize(v[:, 1] - v[:, 0])
    e2 = normalize(v[:, 2] - v[:, 0])
    c = np.stack([e1[:, 1] * e2[:, 2] - e1[:, 2] * e2[:, 1],
                  e1[:, 2] * e2[:, 0] - e1[:, 0] * e2[:, 2],
                  e1[:, 0] * e2[:, 1] - e1[:, 1] * e2[:, 0]], axis=1)
    n = normalize(c)
    return np.repeat(n, 3, axis=0).reshape(-1, 9)


def mesh_from_triangles(tris, mat, name: str = "", normals=None) -> Mesh:
    tris = _f32(tris).reshape(-1, 9)
    nrm = loader_geometric_normals(tris) if normals is None else _f32(normals).reshape(-1, 9)
    mats = np.repeat(np.asarray(mat, MATERIAL_DTYPE).reshape(1), tris.shape[0])
    return Mesh(tris, nrm, mats, [name] * tris.shape[0])


def quad(p0, p1, p2, p3, inward=None):
    """Two triangles of the quad p0 p1 p2 p3, wound so that the face normal
    points along `inward` when given."""
    p = np.asarray([p0, p1, p2, p3], np.float64)
    if inward is not None:
        n = np.cross(p[1] - p[0], p[2] - p[0])
        if np.dot(n, inward) < 0:
            p = p[[0, 3, 2, 1]]
    return [np.concatenate([p[0], p[1], p[2]]), np.concatenate([p[0], p[2], p[3]])]


# ------------------------------------------------------------- Cornell room

WHITE = (0.73, 0.73, 0.73)
RED = (0.63, 0.065, 0.05)
GREEN = (0.14, 0.45, 0.09)
LIGHT_LE = (17.0, 12.0, 4.0)
LIGHT_HALF = 0.125          # the light quad is 0.25 x 0.25
LIGHT_Y = 1.0 - 1e-3
CAMERA = dict(position=(0.5, 0.5, 4.7), forward=(0.0, 0.0, -1.0), fov=0.25 * math.pi)


def box_mesh(center, size, angle, mat, name) -> Mesh:
    """Axis-aligned box of `size` rotated about y by `angle`, resting at
    center (center[1] is its mid-height); 12 triangles, normals outward."""
    sx, sy, sz = (s * 0.5 for s in size)
    c, s = math.cos(angle), math.sin(angle)

    def P(x, y, z):
        return (center[0] + c * x + s * z, center[1] + y, center[2] - s * x + c * z)

    def R(v):
        x, y, z = v
        return (c * x + s * z, y, -s * x + c * z)

    faces = []
    corners = {(i, j, k): P(i * sx, j * sy, k * sz) for i in (-1, 1) for j in (-1, 1) for k in (-1, 1)}
    for axis in range(3):
        for sgn in (-1, 1):
            pts = [key for key in corners if key[axis] == sgn]
            # order the 4 corners around the face
            others = [a for a in range(3) if a != axis]
            ring = sorted(pts, key=lambda k: math.atan2(k[others[1]], k[others[0]]))
            n = [0.0, 0.0, 0.0]
            n[axis] = float(sgn)
            faces += quad(*[corners[k] for k in ring], inward=R(n))
    return mesh_from_triangles(np.array(faces), mat, name)


def cornell_box(seed: int = 0, boxes: bool = True, albedos: dict | None = None,
                light_le=LIGHT_LE) -> Mesh:
    """The procedural Cornell room: [0,1]^3 with an open front (z = 1), five
    walls of two triangles, two white boxes (0.3x0.6x0.3 and 0.3x0.3x0.3)
    rotated about y by seed-drawn angles, and a 0.25x0.25 ceiling light."""
    alb = {"floor": WHITE, "ceiling": WHITE, "backWall": WHITE, "leftWall": RED,
           "rightWall": GREEN, "tallBox": WHITE, "shortBox": WHITE, "light": (0.78, 0.78, 0.78)}
    if albedos:
        alb.update(albedos)
    walls = [
        ("floor", [(0, 0, 0), (1, 0, 0), (1, 0, 1), (0, 0, 1)], (0, 1, 0)),
        ("ceiling", [(0, 1, 0), (1, 1, 0), (1, 1, 1), (0, 1, 1)], (0, -1, 0)),
        ("backWall", [(0, 0, 0), (1, 0, 0), (1, 1, 0), (0, 1, 0)], (0, 0, 1)),
        ("leftWall", [(0, 0, 0), (0, 1, 0), (0, 1, 1), (0, 0, 1)], (1, 0, 0)),
        ("rightWall", [(1, 0, 0), (1, 1, 0), (1, 1, 1), (1, 0, 1)], (-1, 0, 0)),
    ]
    mesh = None
    for name, pts, inward in walls:
        m = mesh_from_triangles(np.array(quad(*pts, inward=inward)), material(rho=alb[name]), name)
        mesh = m if mesh is None else mesh + m
    if boxes:
        rng = np.random.default_rng(seed)
        a_tall, a_short = rng.uniform(0.0, 0.5 * math.pi, size=2)
        mesh = mesh + box_mesh((0.3, 0.3, 0.32), (0.3, 0.6, 0.3), a_tall,
                               material(rho=alb["tallBox"]), "tallBox")
        mesh = mesh + box_mesh((0.7, 0.15, 0.66), (0.3, 0.3, 0.3), a_short,
                               material(rho=alb["shortBox"]), "shortBox")
    h = LIGHT_HALF
    lq = quad((0.5 - h, LIGHT_Y, 0.5 - h), (0.5 + h, LIGHT_Y, 0.5 - h),
              (0.5 + h, LIGHT_Y, 0.5 + h), (0.5 - h, LIGHT_Y, 0.5 + h), inward=(0, -1, 0))
    mesh = mesh + mesh_from_triangles(np.array(lq), material(rho=alb["light"], le=light_le), "light")
    return mesh


def icosphere(center, radius: float, subdiv: int, mat, name: str) -> Mesh:
    """Icosphere of 20 * 4^subdiv triangles with smooth vertex normals."""
    t = (1.0 + 5 ** 0.5) / 2.0
    verts = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t), (0, -1, -t),
             (0, 1, -t), (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    verts = [np.array(v, float) / np.linalg.norm(v) for v in verts]
    faces = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4),
             (11, 10, 2), (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8),
             (3, 8, 9), (4, 9, 5), (2, 4, 11), (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    for _ in range(subdiv):
        cache = {}

        def mid(a, b):
            key = (min(a, b), max(a, b))
            if key not in cache:
                m = verts[a] + verts[b]
                verts.append(m / np.linalg.norm(m))
                cache[key] = len(verts) - 1
            return cache[key]

        nf = []
        for a, b, c in faces:
            ab, bc, ca = mid(a, b), mid(b, c), mid(c, a)
            nf += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
        faces = nf
    V = np.array(verts)
    F = np.array(faces)
    tri = (V[F] * radius + np.asarray(center)).reshape(-1, 9)
    nrm = V[F].reshape(-1, 9)
    return mesh_from_triangles(tri, mat, name, normals=nrm)


def heightfield(n: int, y0: float, seed: int, mat, name: str, n_sines: int = 8,
                amp_max: float = 0.01, wl=(0.05, 0.3)) -> Mesh:
    """n x n vertex grid over the room's floor area at height y0 + sum of
    n_sines sines (seed-drawn amplitude <= amp_max, wavelength in wl,
    direction and phase); per-vertex normals from the analytic gradient."""
    rng = np.random.default_rng(seed)
    amp = rng.uniform(0.0, amp_max, n_sines)
    lam = rng.uniform(wl[0], wl[1], n_sines)
    ang = rng.uniform(0.0, 2 * math.pi, n_sines)
    ph = rng.uniform(0.0, 2 * math.pi, n_sines)
    x = np.linspace(0.0, 1.0, n)
    X, Z = np.meshgrid(x, x, indexing="ij")
    H = np.full_like(X, y0)
    dX = np.zeros_like(X)
    dZ = np.zeros_like(X)
    for a, l, t, p in zip(amp, lam, ang, ph):
        kx, kz = 2 * math.pi / l * math.cos(t), 2 * math.pi / l * math.sin(t)
        arg = kx * X + kz * Z + p
        H += a * np.sin(arg)
        dX += a * kx * np.cos(arg)
        dZ += a * kz * np.cos(arg)
    P = np.stack([X, H, Z], -1)
    Nn = np.stack([-dX, np.ones_like(X), -dZ], -1)
    Nn /= np.linalg.norm(Nn, axis=-1, keepdims=True)
    i, j = np.meshgrid(np.arange(n - 1), np.arange(n - 1), indexing="ij")
    i, j = i.ravel(), j.ravel()
    a, b, c, d = (i, j), (i + 1, j), (i + 1, j + 1), (i, j + 1)
    # wound so the face normal points up (+y): (a, d, c) and (a, c, b)
    t1 = [a, d, c]
    t2 = [a, c, b]
    tris, nrms = [], []
    for t in (t1, t2):
        tris.append(np.concatenate([P[v] for v in t], axis=1))
        nrms.append(np.concatenate([Nn[v] for v in t], axis=1))
    order = np.stack([np.arange(len(i)), np.arange(len(i))], 1).ravel()
    tri = np.empty((2 * len(i), 9))
    nrm = np.empty((2 * len(i), 9))
    tri[0::2], tri[1::2] = tris[0], tris[1]
    nrm[0::2], nrm[1::2] = nrms[0], nrms[1]
    del order
    return mesh_from_triangles(tri, mat, name, normals=nrm)


def caustics_scene(seed: int = 0, grid: int = 512, subdiv: int = 5) -> Mesh:
    """The Cornell room plus a mirror and a glass (IOR 1.5) icosphere and a
    water surface (IOR 1.33): a grid x grid heightfield of 8 sines."""
    m = cornell_box(seed)
    m = m + icosphere((0.74, 0.55, 0.3), 0.13, subdiv, material(PM_MIRROR, rho=(1, 1, 1)), "mirror")
    m = m + icosphere((0.3, 0.72, 0.68), 0.12, subdiv, material(PM_GLASS, rho=(1, 1, 1), ior=1.5),
                      "glass")
    m = m + heightfield(grid, 0.22, seed + 1, material(PM_GLASS, rho=(1, 1, 1), ior=1.33), "water")
    return m


# ------------------------------------------------------------------ OBJ / MTL

def write_obj(mesh: Mesh, path: str | Path) -> None:
    """Writes mesh as OBJ + MTL (one material per distinct name; v/vn per
    face corner, so load_obj gives back the same per-face arrays)."""
    path = Path(path)
    mtl = path.with_suffix(".mtl")
    names = list(dict.fromkeys(mesh.names))
    first = {nm: mesh.names.index(nm) for nm in names}
    with open(mtl, "w") as f:
        for nm in names:
            m = mesh.materials[first[nm]]
            illum = {PM_LAMBERT: 1, PM_MIRROR: 5, PM_GLASS: 7}[int(m["type"])]
            kd = " ".join(f"{float(x):.9g}" for x in m["rho"])
            ke = " ".join(f"{float(x):.9g}" for x in m["le"])
            f.write(f"newmtl {nm}\nKd {kd}\nKe {ke}\nNi {float(m['ior']):.9g}\nillum {illum}\n\n")
    with open(path, "w") as f:
        f.write(f"mtllib {mtl.name}\n")
        v = mesh.vertices.reshape(-1, 3)
        nv = mesh.normals.reshape(-1, 3)
        # 9 significant digits give back the same float32
        f.write("".join(f"v {x:.9g} {y:.9g} {z:.9g}\n" for x, y, z in v.tolist()))
        f.write("".join(f"vn {x:.9g} {y:.9g} {z:.9g}\n" for x, y, z in nv.tolist()))
        cur = None
        for fi in range(mesh.n_faces):
            if mesh.names[fi] != cur:
                cur = mesh.names[fi]
                f.write(f"usemtl {cur}\n")
            a = 3 * fi + 1
            f.write(f"f {a}//{a} {a + 1}//{a + 1} {a + 2}//{a + 2}\n")


def _parse_mtl(path: Path) -> dict:
    mats, cur = {}, None
    for line in path.read_text().splitlines():
        tok = line.split()
        if not tok or tok[0].startswith("#"):
            continue
        if tok[0] == "newmtl":
            cur = tok[1]
            mats[cur] = {"Kd": (0.0, 0.0, 0.0), "Ke": (0.0, 0.0, 0.0), "Ni": 1.0, "illum": 0}
        elif cur is not None and tok[0] in ("Kd", "Ke"):
            mats[cur][tok[0]] = tuple(float(x) for x in tok[1:4])
        elif cur is not None and tok[0] == "Ni":
            mats[cur]["Ni"] = float(tok[1])
        elif cur is not None and tok[0] == "illum":
            mats[cur]["illum"] = int(tok[1])
    return mats


def load_obj(path: str | Path, mtl_search_path: str | Path | None = None) -> Mesh:
    """Reads an OBJ file with Scene::loadModel's rules (scene.h:107-270):
    polygons are fan-triangulated; a face without normals gets the loader's
    geometric normal three times (:182-189); materials map illum 5 -> Mirror,
    illum 7 -> Glass(Ni), else Lambert(Kd), Ke > 0 -> area light (:21-51); a
    face without material is Lambert(0.9) (:16-18)."""
    path = Path(path)
    base = Path(mtl_search_path) if mtl_search_path else path.parent
    V, VN = [], []
    mats, mat_names = {}, []
    cur = None
    faces = []  # (vertex ids, normal ids or None, material name)
    for line in path.read_text().splitlines():
        tok = line.split()
        if not tok or tok[0].startswith("#"):
            continue
        if tok[0] == "v":
            V.append([float(x) for x in tok[1:4]])
        elif tok[0] == "vn":
            VN.append([float(x) for x in tok[1:4]])
        elif tok[0] == "mtllib":
            p = base / tok[1]
            if p.exists():
                mats.update(_parse_mtl(p))
        elif tok[0] == "usemtl":
            cur = tok[1]
        elif tok[0] == "f":
            vi, ni = [], []
            for c in tok[1:]:
                parts = c.split("/")
                iv = int(parts[0])
                vi.append(iv - 1 if iv > 0 else len(V) + iv)
                if len(parts) >= 3 and parts[2]:
                    inn = int(parts[2])
                    ni.append(inn - 1 if inn > 0 else len(VN) + inn)
            for k in range(1, len(vi) - 1):
                tv = [vi[0], vi[k], vi[k + 1]]
                tn = [ni[0], ni[k], ni[k + 1]] if len(ni) == len(vi) else None
                faces.append((tv, tn, cur))
    Va = np.asarray(V, np.float32).reshape(-1, 3)
    VNa = np.asarray(VN, np.float32).reshape(-1, 3)
    nf = len(faces)
    verts = np.empty((nf, 9), np.float32)
    nrms = np.empty((nf, 9), np.float32)
    has_n = np.zeros(nf, bool)
    mat_arr = np.zeros(nf, MATERIAL_DTYPE)
    names = []
    for fi, (tv, tn, mn) in enumerate(faces):
        verts[fi] = Va[tv].ravel()
        if tn is not None:
            nrms[fi] = VNa[tn].ravel()
            has_n[fi] = True
        md = mats.get(mn) if mn is not None else None
        if md is None:
            mat_arr[fi] = material(PM_LAMBERT, rho=(0.9, 0.9, 0.9))
        else:
            kind = {5: PM_MIRROR, 7: PM_GLASS}.get(md["illum"], PM_LAMBERT)
            rho = md["Kd"] if kind == PM_LAMBERT else (1.0, 1.0, 1.0)
            mat_arr[fi] = material(kind, rho=rho, ior=md["Ni"], le=md["Ke"])
        names.append(mn or "")
    if (~has_n).any():
        nrms[~has_n] = loader_geometric_normals(verts[~has_n])
    return Mesh(verts, nrms, mat_arr, names)


# ----------------------------------------------------------- device scene

class Scene:
    """The reference's Scene (scene.h:53-356) over the device scene."""

    def __init__(self, ctx: Context | None = None):
        self.ctx = ctx if ctx is not None else Context(0)
        self.mesh: Mesh | None = None

    def loadModel(self, path) -> None:  # scene.h:109
        self.mesh = load_obj(path)

    def setMesh(self, mesh: Mesh) -> None:
        self.mesh = mesh

    def nVertices(self) -> int:
        return 0 if self.mesh is None else 3 * self.mesh.n_faces

    def nFaces(self) -> int:
        return 0 if self.mesh is None else self.mesh.n_faces

    def build(self) -> None:  # scene.h:275
        m = self.mesh
        v, n = _f32(m.vertices), _f32(m.normals)
        mats = np.ascontiguousarray(m.materials, MATERIAL_DTYPE)
        self.ctx.check(self.ctx.lib.pm_scene_upload(self.ctx.handle, ptr(v), ptr(n),
                                                    mats.ctypes.data, m.n_faces),
                       "pm_scene_upload")

    def intersect(self, origins, directions, tmin: float = 1e-5, tmax=None) -> np.ndarray:
        """Batched closest hit: HIT_DTYPE records (prim = -1 on a miss)."""
        o = _f32(origins).reshape(-1, 3)
        d = _f32(directions).reshape(-1, 3)
        r = np.empty((o.shape[0], 8), np.float32)
        r[:, 0:3], r[:, 3] = o, tmin
        r[:, 4:7] = d
        r[:, 7] = np.finfo(np.float32).max if tmax is None else tmax
        out = np.empty(o.shape[0], HIT_DTYPE)
        self.ctx.check(self.ctx.lib.pm_scene_intersect(self.ctx.handle, ptr(r), r.shape[0],
                                                       out.ctypes.data),
                       "pm_scene_intersect")
        return out

"""Seeded synthetic photon sets and query sets.

These stand in for photon maps and hit points when a test or benchmark
needs one without tracing a scene: uniform photons in the unit cube,
photons lying on the five walls of the [0,1]^3 Cornell room (the layout a
traced photon map has: points on surfaces, directions in the hemisphere
above each surface), and lattice photons that make many distances tie.
"""
from __future__ import annotations

import numpy as np

# The five walls of the unit Cornell room: (axis, value, inward normal, albedo)
WALLS = (
    (1, 0.0, (0.0, 1.0, 0.0), (0.73, 0.73, 0.73)),      # floor
    (1, 1.0, (0.0, -1.0, 0.0), (0.73, 0.73, 0.73)),     # ceiling
    (2, 0.0, (0.0, 0.0, 1.0), (0.73, 0.73, 0.73)),      # back wall
    (0, 0.0, (1.0, 0.0, 0.0), (0.63, 0.065, 0.05)),     # left wall (red)
    (0, 1.0, (-1.0, 0.0, 0.0), (0.14, 0.45, 0.09)),     # right wall (green)
)


def _unit(v: np.ndarray) -> np.ndarray:
    return v / np.linalg.norm(v, axis=-1, keepdims=True)


def hemisphere(rng: np.random.Generator, normals: np.ndarray) -> np.ndarray:
    """Uniform unit directions with dot(d, n) > 0 for each row of normals."""
    d = _unit(rng.normal(size=normals.shape))
    flip = np.sum(d * normals, axis=1) < 0
    d[flip] = -d[flip]
    return d


def uniform_photons(n: int, seed: int = 0) -> np.ndarray:
    rng = np.random.default_rng(seed)
    ph = np.empty((n, 9), np.float32)
    ph[:, 0:3] = rng.uniform(0.0, 2.0, size=(n, 3))
    ph[:, 3:6] = rng.uniform(0.0, 1.0, size=(n, 3))
    ph[:, 6:9] = _unit(rng.normal(size=(n, 3)))
    return ph


def wall_points(rng: np.random.Generator, n: int):
    """n points on the Cornell walls: (positions, inward normals, albedos)."""
    w = rng.integers(0, len(WALLS), size=n)
    pos = rng.uniform(0.0, 1.0, size=(n, 3))
    nrm = np.empty((n, 3))
    rho = np.empty((n, 3))
    for i, (axis, val, nn, alb) in enumerate(WALLS):
        m = w == i
        pos[m, axis] = val
        nrm[m] = nn
        rho[m] = alb
    return pos, nrm, rho


def wall_photons(n: int, seed: int = 0) -> np.ndarray:
    """Photons on the walls with wi in the hemisphere above the wall."""
    rng = np.random.default_rng(seed)
    pos, nrm, rho = wall_points(rng, n)
    ph = np.empty((n, 9), np.float32)
    ph[:, 0:3] = rng.uniform(0.0, 1.5, size=(n, 3)) * rho
    ph[:, 3:6] = pos
    ph[:, 6:9] = hemisphere(rng, nrm)
    # a few photons arriving from below the surface (grazing leaks) so the
    # Lambert cosine test has both outcomes
    leak = rng.random(n) < 0.05
    ph[leak, 6:9] = -ph[leak, 6:9]
    return ph


def lattice_photons(m: int = 12, spacing: float = 0.125, seed: int = 0) -> np.ndarray:
    """Photons on an m^3 lattice: many exactly equal distances."""
    rng = np.random.default_rng(seed)
    g = np.arange(m, dtype=np.float32) * np.float32(spacing)
    x, y, z = np.meshgrid(g, g, g, indexing="ij")
    n = m ** 3
    ph = np.empty((n, 9), np.float32)
    ph[:, 0:3] = rng.uniform(0.1, 1.0, size=(n, 3))
    ph[:, 3] = x.ravel()
    ph[:, 4] = y.ravel()
    ph[:, 5] = z.ravel()
    ph[:, 6:9] = _unit(rng.normal(size=(n, 3)))
    return ph


def wall_queries(n: int, seed: int = 1) -> np.ndarray:
    """pm_radiance_query records (n, 12) for points on the walls: wo in the
    hemisphere above the wall, ns = the wall normal, rho = its albedo."""
    rng = np.random.default_rng(seed)
    pos, nrm, rho = wall_points(rng, n)
    wo = hemisphere(rng, nrm)
    q = np.empty((n, 12), np.float32)
    q[:, 0:3], q[:, 3] = pos, rho[:, 0]
    q[:, 4:7], q[:, 7] = wo, rho[:, 1]
    q[:, 8:11], q[:, 11] = nrm, rho[:, 2]
    return q


# --------------------------------------------------------------- camera rays

_PCG_MULT = np.uint64(6364136223846793005)


def pcg32_next(state: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    """One PCG32 XSH-RR step for many generators with inc = 1, as the
    reference's RNG (sampler.h:11-47): returns (uint32 output, new state)."""
    old = state
    with np.errstate(over="ignore"):
        new = old * _PCG_MULT + np.uint64(1)
    xs = (((old >> np.uint64(18)) ^ old) >> np.uint64(27)).astype(np.uint32)
    rot = (old >> np.uint64(59)).astype(np.uint32)
    out = (xs >> rot) | (xs << ((np.uint32(32) - rot) & np.uint32(31)))
    return out.astype(np.uint32), new


def pcg32_float(u: np.ndarray) -> np.ndarray:
    """RNG::getNext: float(u32) * (1.0f / UINT32_MAX) in float32 (1.0 reachable)."""
    return u.astype(np.float32) * np.float32(1.0 / 4294967295.0)


ROOM_CAMERA = dict(position=(0.5, 0.5, 4.7), forward=(0.0, 0.0, -1.0), fov=0.25 * 3.14159265359)
LIGHT_MIN, LIGHT_MAX, LIGHT_Y = 0.375, 0.625, 0.999


def room_primary_hit_queries(width: int = 512, height: int = 512, spp: int = 4) -> np.ndarray:
    """pm_radiance_query records for the primary hits of a width x height x spp
    frame of the empty unit Cornell room (five walls, ceiling light quad).

    Camera samples follow the reference's render loop (examples/main.cpp:33-47
    with camera.h:41-47): pixel (i, j) owns a sampler seeded j + width*i and
    each sample draws the u then the v jitter; with no final gathering a
    diffuse hit draws nothing else, so sample s uses draws 2s and 2s+1.
    Queries come in pixel-major, sample-minor order; rays that hit the light
    (which returns Le, no photon-map query) are left out.
    """
    f32 = np.float32
    pos = np.array(ROOM_CAMERA["position"], f32)
    fwd = np.array(ROOM_CAMERA["forward"], f32)
    right = np.cross(fwd, np.array([0, 1, 0], f32)).astype(f32)
    right = right / np.sqrt(f32(np.dot(right, right)))
    up = np.cross(right, fwd).astype(f32)
    up = up / np.sqrt(f32(np.dot(up, up)))
    focal = f32(1.0) / f32(np.tan(f32(0.5) * f32(ROOM_CAMERA["fov"])))
    ii, jj = np.meshgrid(np.arange(height), np.arange(width), indexing="ij")
    state = (jj + width * ii).astype(np.uint64).ravel()
    jf = jj.ravel().astype(f32)
    if_ = ii.ravel().astype(f32)
    rays_o, rays_d = [], []
    for _ in range(spp):
        a, state = pcg32_next(state)
        b, state = pcg32_next(state)
        u = (f32(2.0) * (jf + pcg32_float(a)) - f32(width)) / f32(height)
        v = (f32(2.0) * (if_ + pcg32_float(b)) - f32(height)) / f32(height)
        pin = pos + focal * fwd
        sensor = pos[None, :] + u[:, None] * right[None, :] + v[:, None] * up[None, :]
        d = (pin[None, :] - sensor).astype(f32)
        d = d / np.sqrt((d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1]) + d[:, 2] * d[:, 2])[:, None]
        rays_o.append(sensor)
        rays_d.append(d)
    o = np.stack(rays_o, axis=1).reshape(-1, 3).astype(np.float64)
    d = np.stack(rays_d, axis=1).reshape(-1, 3).astype(np.float64)
    best_t = np.full(o.shape[0], np.inf)
    best_w = np.full(o.shape[0], -1)
    for wi, (axis, val, nn, alb) in enumerate(WALLS):
        with np.errstate(divide="ignore", invalid="ignore"):
            t = (val - o[:, axis]) / d[:, axis]
        p = o + t[:, None] * d
        inside = np.ones(o.shape[0], bool)
        for ax in range(3):
            if ax != axis:
                inside &= (p[:, ax] >= 0.0) & (p[:, ax] <= 1.0)
        ok = inside & (t > 1e-5) & (t < best_t)
        best_t[ok] = t[ok]
        best_w[ok] = wi
    with np.errstate(divide="ignore", invalid="ignore"):
        tl = (LIGHT_Y - o[:, 1]) / d[:, 1]
    pl = o + tl[:, None] * d
    light = ((tl > 1e-5) & (tl < best_t) & (pl[:, 0] >= LIGHT_MIN) & (pl[:, 0] <= LIGHT_MAX)
             & (pl[:, 2] >= LIGHT_MIN) & (pl[:, 2] <= LIGHT_MAX))
    keep = (best_w >= 0) & ~light
    hit = o[keep] + best_t[keep, None] * d[keep]
    w = best_w[keep]
    nrm = np.array([WALLS[i][2] for i in range(len(WALLS))])[w]
    rho = np.array([WALLS[i][3] for i in range(len(WALLS))])[w]
    q = np.empty((hit.shape[0], 12), np.float32)
    q[:, 0:3], q[:, 3] = hit, rho[:, 0]
    q[:, 4:7], q[:, 7] = -d[keep], rho[:, 1]
    q[:, 8:11], q[:, 11] = nrm, rho[:, 2]
    return q


# ------------------------------------------------- traced-scene workloads

def camera_rays(camera, width: int, height: int, spp: int):
    """Camera rays of a width x height x spp frame, pixel-major and
    sample-minor, drawn as the reference's render loop draws them
    (examples/main.cpp:37-46, camera.h:41-47) when a sample consumes no
    random number besides its u, v jitter (a render without final gathering
    of a Lambert-only scene): sample s of pixel (i, j) uses draws 2s, 2s+1
    of the sampler seeded j + width*i. Returns (origins, directions) float32."""
    f32 = np.float32
    ii, jj = np.meshgrid(np.arange(height), np.arange(width), indexing="ij")
    state = (jj + width * ii).astype(np.uint64).ravel()
    jf, if_ = jj.ravel().astype(f32), ii.ravel().astype(f32)
    pin = (camera.position + camera.focal_length * camera.forward).astype(f32)
    os_, ds = [], []
    for _ in range(spp):
        a, state = pcg32_next(state)
        b, state = pcg32_next(state)
        u = (f32(2.0) * (jf + pcg32_float(a)) - f32(width)) / f32(height)
        v = (f32(2.0) * (if_ + pcg32_float(b)) - f32(height)) / f32(height)
        sensor = ((camera.position[None, :] + u[:, None] * camera.right[None, :])
                  + v[:, None] * camera.up[None, :]).astype(f32)
        d = (pin[None, :] - sensor).astype(f32)
        ln = np.sqrt((d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1]) + d[:, 2] * d[:, 2])
        os_.append(sensor)
        ds.append((d / ln[:, None]).astype(f32))
    o = np.stack(os_, axis=1).reshape(-1, 3)
    d = np.stack(ds, axis=1).reshape(-1, 3)
    return o, d


def hit_queries(mesh, o, d, hits) -> np.ndarray:
    """pm_radiance_query records for the rays whose closest hit is a
    non-emitting Lambert face: position = o + t*d (Ray::operator()), wo =
    -d, shading normal interpolated as triangle.h:64-71, rho of the face.
    `hits` is (n, 4) {t, u, v, face bits} or the HIT_DTYPE records."""
    f32 = np.float32
    if hits.dtype.names:
        t, u, v, prim = hits["t"], hits["u"], hits["v"], hits["prim"]
    else:
        t, u, v, prim = hits[:, 0], hits[:, 1], hits[:, 2], hits[:, 3].view(np.int32)
    ok = prim >= 0
    m = mesh.materials[np.where(ok, prim, 0)]
    ok &= (m["type"] == 0) & ~(m["le"] > 0).any(axis=1)
    t, u, v, prim = t[ok], u[ok], v[ok], prim[ok]
    o, d = o[ok], d[ok]
    pos = (o + t[:, None] * d).astype(f32)
    n = mesh.normals[prim].reshape(-1, 3, 3)
    w0 = (f32(1.0) - u) - v
    ns = ((n[:, 0] * w0[:, None] + n[:, 1] * u[:, None]) + n[:, 2] * v[:, None]).astype(f32)
    rho = mesh.materials["rho"][prim]
    q = np.empty((pos.shape[0], 12), f32)
    q[:, 0:3], q[:, 3] = pos, rho[:, 0]
    q[:, 4:7], q[:, 7] = -d, rho[:, 1]
    q[:, 8:11], q[:, 11] = ns, rho[:, 2]
    return q


def rays8(o, d, tmin: float = 1e-5):
    r = np.empty((o.shape[0], 8), np.float32)
    r[:, 0:3], r[:, 3], r[:, 4:7] = o, tmin, d
    r[:, 7] = np.finfo(np.float32).max
    return r


def traced_cornell_knn_workload(ctx, n_emit: int = 1_000_000, seed: int = 1, width: int = 512,
                                height: int = 512, spp: int = 4, max_depth: int = 100):
    """The kNN radiance workload of the benchmark: the global photon map
    traced on the device from `n_emit` photons emitted in the procedural
    Cornell box (seed 0 scene, trace seed `seed`; PhotonMapping::build,
    integrator.h:393-474, without final gathering), and one
    pm_radiance_query per primary hit of a width x height x spp frame on a
    non-emitting Lambert face, in pixel order (sample-minor).

    Leaves the scene and the traced map on `ctx` (map PM_MAP_GLOBAL).
    Returns (scene, mesh, camera, photons (n, 9), queries (nq, 12), trace
    statistics)."""
    from . import scene as S
    from .camera import Camera
    from .integrator import PhotonMapping
    mesh = S.cornell_box(0)
    camera = Camera(S.CAMERA["position"], S.CAMERA["forward"], S.CAMERA["fov"])
    sc = S.Scene(ctx)
    sc.setMesh(mesh)
    sc.build()
    pmi = PhotonMapping(n_emit, 100, 1.0, 100, 0, max_depth, ctx=ctx)
    stats = pmi.build(sc, seed=seed)["global"]
    photons = pmi.global_map.photons()
    o, d = camera_rays(camera, width, height, spp)
    queries = hit_queries(mesh, o, d, sc.intersect(o, d))
    return sc, mesh, camera, photons, queries, stats


def parity_sample(nq: int, seed: int = 0, runs: int = 40, run_len: int = 64, starts: int = 512,
                  singles: int = 1024) -> np.ndarray:
    """Indices of a sample of a query stream of length nq for exactness
    checks against brute force: `runs` runs of `run_len` consecutive
    queries beginning at multiples of 16 (the first query of a run of the
    kNN kernel's work items, then its warm successors), the last run_len
    queries (the short work items at the end of a launch), the first query
    of `starts` work items, and `singles` queries drawn at random. Sorted,
    without repeats."""
    rng = np.random.default_rng(seed)
    parts = []
    if nq > 0:
        hi = max(nq - run_len, 0)
        for b in np.linspace(0, hi, runs).astype(np.int64):
            b = (b // 16) * 16
            parts.append(np.arange(b, min(b + run_len, nq)))
        parts.append(np.arange(max(nq - run_len, 0), nq))
        parts.append((rng.integers(0, max(nq // 16, 1), starts) * 16).clip(0, nq - 1))
        parts.append(rng.integers(0, nq, singles))
    if not parts:
        return np.zeros(0, np.int64)
    return np.unique(np.concatenate(parts)).astype(np.int64)

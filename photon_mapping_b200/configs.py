"""The benchmark scenes and render settings of the photon mapper, and the
image-convergence measurement: a photon-mapping render of each against a
path-traced render of the same scene at high sample count.

    python -m photon_mapping_b200.configs [--config NAME ...] [--pt-spp 4096]

(NAME: cornell-256, cornell-512-final-gathering, caustics-512; all three by
default) prints one JSON line per setting: render and photon-trace times, samples/s,
and the RMSE of the photon-mapping image against the path tracer
(integrator.h:51-106 on the device) at 2 x pt-spp, on raw linear radiance
over all pixels and channels. Also given: the same without pixels that see
the light directly (their value is the fraction of samples landing on the
emitter, noisy for both), on 8x8-pixel block means (noise averaged out,
bias kept), and corrected for the path tracer's own noise.
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

from . import scene as S
from .camera import Camera

MAX_DEPTH = 100

CONFIGS = {
    "cornell-256": dict(scene="cornell", width=256, height=256, spp=16, photons=100_000,
                        caustics_multiplier=1.0, k=100, fg=0, n_gather=1),
    "cornell-512-final-gathering": dict(scene="cornell", width=512, height=512, spp=100,
                                        photons=1_000_000, caustics_multiplier=1.0, k=100,
                                        fg=1, n_gather=16),
    "caustics-512": dict(scene="caustics", width=512, height=512, spp=64, photons=1_000_000,
                         caustics_multiplier=10.0, k=100, fg=1, n_gather=1),
}
NAMES = list(CONFIGS)


def make_scene(kind: str) -> S.Mesh:
    """cornell: the procedural Cornell box (36 triangles); caustics: the room
    plus a mirror and a glass icosphere (subdivision 5) and a 512 x 512
    water heightfield (563,238 triangles)."""
    return S.cornell_box(0) if kind == "cornell" else S.caustics_scene(0)


def camera() -> Camera:
    return Camera(S.CAMERA["position"], S.CAMERA["forward"], S.CAMERA["fov"])


def image_error(img: np.ndarray, ref: np.ndarray, ref_noise: float | None = None) -> dict:
    """Errors of img against ref over the pixels finite in both. ref_noise
    (the RMSE of ref's own Monte Carlo noise) gives the noise-corrected
    figure sqrt(rmse^2 - ref_noise^2)."""
    ok = np.isfinite(img).all(axis=2) & np.isfinite(ref).all(axis=2)
    err = img.astype(np.float64) - ref.astype(np.float64)
    mean_ref = float(ref[ok].mean())
    mask = ok & (ref.max(axis=2) < 1.0)
    e, em = err[ok], err[mask]
    rmse = float(np.sqrt(np.mean(e ** 2)))
    h, w = img.shape[:2]
    b = 8
    en = np.where(ok[..., None], err, np.nan)[: h // b * b, : w // b * b]
    blk = np.nanmean(en.reshape(h // b, b, w // b, b, 3), axis=(1, 3))
    out = {
        "rmse": rmse,
        "rel_rmse": rmse / mean_ref,
        "bias": float(e.mean()) / mean_ref,
        "rel_rmse_without_light_pixels": float(np.sqrt(np.mean(em ** 2))) / float(ref[mask].mean()),
        "rel_rmse_8x8_blocks": float(np.sqrt(np.nanmean(blk ** 2))) / mean_ref,
        "light_pixels": int((ok & ~mask).sum()),
        "nonfinite_pixels": {"image": int((~np.isfinite(img).all(axis=2)).sum()),
                             "reference": int((~np.isfinite(ref).all(axis=2)).sum()),
                             "image_first": np.argwhere(~np.isfinite(img).all(axis=2))[:4].tolist(),
                             "reference_first":
                                 np.argwhere(~np.isfinite(ref).all(axis=2))[:4].tolist()},
    }
    if ref_noise is not None:
        out["reference_noise_rmse"] = ref_noise
        out["rel_rmse_noise_corrected"] = float(np.sqrt(max(rmse ** 2 - ref_noise ** 2, 0.0))) / mean_ref
    return out


def path_traced_reference(ctx, cam, width: int, height: int, spp: int):
    """Path-traced image at 2*spp and the RMSE of its own noise. The
    per-pixel sampler streams make the 2*spp render the mean of the spp
    render and an independent second half, so the half-difference gives the
    noise: rmse(first - second) / 2 for the mean of both."""
    from .integrator import PathTracing
    pt = PathTracing(MAX_DEPTH, ctx=ctx)
    first, _ = pt.render(cam, width, height, spp)
    t0 = time.perf_counter()
    both, _ = pt.render(cam, width, height, 2 * spp)
    secs = time.perf_counter() - t0
    second = 2.0 * both.astype(np.float64) - first
    ok = np.isfinite(first).all(axis=2) & np.isfinite(second).all(axis=2)
    noise = float(np.sqrt(np.mean((first[ok] - second[ok]) ** 2))) / 2.0
    return both, noise, secs


def run_config(ctx, name: str, pt_spp: int, spp: int | None = None, seed: int = 1,
               save_dir: str | None = None, return_images: bool = False):
    """Traces and renders setting `name` of CONFIGS on `ctx`, path-traces the reference
    image, and returns the record printed by the command line (with
    return_images: the record, the photon-mapping image and the path-traced
    image). With save_dir, both images are written there as .npy (raw
    linear radiance)."""
    from .integrator import PhotonMapping
    c = CONFIGS[name]
    spp = c["spp"] if spp is None else spp
    mesh = make_scene(c["scene"])
    sc = S.Scene(ctx)
    sc.setMesh(mesh)
    sc.build()
    cam = camera()
    pmi = PhotonMapping(c["photons"], c["k"], c["caustics_multiplier"], c["k"], c["fg"], MAX_DEPTH,
                        ctx=ctx)
    pmi.build(sc, seed=seed)                       # warm-up
    t0 = time.perf_counter()
    stats = pmi.build(sc, seed=seed)
    t_trace = time.perf_counter() - t0
    pmi.render(cam, c["width"], c["height"], spp, n_gather=c["n_gather"])   # warm-up
    t0 = time.perf_counter()
    img, rst = pmi.render(cam, c["width"], c["height"], spp, n_gather=c["n_gather"])
    t_render = time.perf_counter() - t0
    ref, noise, t_pt = path_traced_reference(ctx, cam, c["width"], c["height"], pt_spp)
    if save_dir:
        from pathlib import Path
        Path(save_dir).mkdir(parents=True, exist_ok=True)
        np.save(Path(save_dir) / f"{name}_photon_mapping.npy", img)
        np.save(Path(save_dir) / f"{name}_path_tracing.npy", ref)
    n = c["width"] * c["height"] * spp
    rec = {
        "name": name, **c, "spp": spp, "triangles": int(mesh.n_faces),
        "photons_stored": {k: int(v["stored"]) for k, v in stats.items()},
        "trace_s": t_trace, "render_s": t_render, "samples_per_s": n / t_render,
        "render_stats": rst,
        "path_tracing": {"spp": 2 * pt_spp, "seconds": t_pt,
                         "samples_per_s": c["width"] * c["height"] * 2 * pt_spp / t_pt},
        "error_vs_path_tracing": image_error(img, ref, noise),
    }
    return (rec, img, ref) if return_images else rec


def main(argv=None) -> None:
    from . import Context
    ap = argparse.ArgumentParser(description=__doc__,
                                 formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--config", nargs="+", choices=NAMES, default=NAMES)
    ap.add_argument("--pt-spp", type=int, default=4096,
                    help="the path-traced reference uses twice this many samples")
    ap.add_argument("--spp", type=int, default=None, help="override the config's spp")
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("--save", default=None, help="directory for the images (.npy)")
    args = ap.parse_args(argv)
    ctx = Context(args.device)
    for name in args.config:
        print(json.dumps(run_config(ctx, name, args.pt_spp, args.spp, save_dir=args.save)), flush=True)
    ctx.close()


if __name__ == "__main__":
    main()

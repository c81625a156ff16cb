#!/usr/bin/env python
"""Benchmark of the photon-mapping hot path on B200.

Metric: kNN radiance queries/s at 1M photons, k=100 — the radiance estimate
of integrator.h:133-152 (k nearest photons + Lambert BRDF sum) for every
primary hit of a 512x512x4-spp frame, against a device-resident photon map.

One step = one pass of the estimate over the whole query set (inputs
already in HBM). L2 is flushed (256 MiB write) before each step, outside
the step's CUDA events. `e2e` times the same pass through the C ABI entry
point with pinned host buffers (host->device copy of the queries and the
device->host copy of the radiance inside the timed region).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

N > 1 runs under torchrun as N independent replicas (the photon map and
the queries are not exchanged between GPUs; each rank does the full
pass), timed as the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

K_NEAREST = 100
N_EMIT = 1_000_000          # photons emitted for the global map of the benchmark
TRACE_SEED = 1
MAX_DEPTH = 100
IMAGE_W = IMAGE_H = 512
SPP = 4                     # the query frame: primary hits of 512x512x4 spp
# algorithmic bytes per query: k photons x 36 B (position, throughput, wi),
# the 48-B radiance query record in (position, wo, shading normal, albedo)
# and the 12-B RGB out
BYTES_PER_QUERY = 36 * K_NEAREST + 48 + 12
METRIC = "kNN radiance queries/s at 1M photons k=100"
CPU_SAMPLE_QUERIES = 40000


def parse_args():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-render", action="store_true", help="skip the render-rate measurements")
    ap.add_argument("--no-grad", action="store_true", help="skip the gradient measurements")
    ap.add_argument("--no-batch", action="store_true", help="skip the batched-render measurements")
    ap.add_argument("--batch-scenes", type=int, default=64)
    ap.add_argument("--convergence", nargs="*", default=None, metavar="NAME",
                    help="instead of the benchmark: image error against the path tracer for "
                         "these settings of photon_mapping_b200.configs (default all: "
                         "cornell-256, cornell-512-final-gathering, caustics-512), beside the "
                         "reference integrator's")
    ap.add_argument("--pt-spp", type=int, default=4096)
    ap.add_argument("--batch-stages", type=int, default=None, metavar="N",
                    help="instead of the benchmark: build a batch of the first N random scenes "
                         "of the batched leg and print one step's stage times (a short run "
                         "for profiling the batched kernels)")
    ap.add_argument("--trace-render", choices=["cornell", "caustics"], default=None,
                    help="instead of the benchmark: trace the photon maps of this scene twice "
                         "(1M global photons, caustics x10 with the caustics scene) and render "
                         "one 256x256 frame at 2 spp with final gathering; prints the rays and "
                         "kernel times (a short run for profiling the trace and camera kernels)")
    return ap.parse_args()


def scene_and_camera():
    from photon_mapping_b200 import scene as S
    from photon_mapping_b200.camera import Camera
    return S.cornell_box(0), Camera(S.CAMERA["position"], S.CAMERA["forward"], S.CAMERA["fov"])


def config_dict(nq: int, n_stored: int) -> dict:
    return {
        "workload": (f"radiance estimate k={K_NEAREST} on the photon map traced from {N_EMIT} "
                     f"emitted photons in the procedural Cornell box (512x512 frame scene); queries = "
                     f"primary hits of a {IMAGE_W}x{IMAGE_H}x{SPP}spp frame in pixel order"),
        "photons_emitted": N_EMIT,
        "photons_stored": n_stored,
        "k": K_NEAREST,
        "queries_per_step": nq,
        "l2": "flushed before every step (256 MiB device write outside the step events)",
        "parallelism": "replicas",
    }


# ------------------------------------------------------------------ distributed

def dist_env():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def max_over_ranks(dist, value: float, device) -> float:
    """The largest `value` over all ranks (every rank gets it); the value
    itself without a process group."""
    if dist is None:
        return value
    import torch
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def dist_init(world: int, backend: str):
    if world <= 1:
        return None
    import datetime
    import torch.distributed as dist
    os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
    dist.init_process_group(backend=backend, timeout=datetime.timedelta(seconds=120))
    return dist


# ----------------------------------------------------------------------- clocks

class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.path = Path(tempfile.mkstemp(prefix="clocks_", suffix=".csv")[1])

    def start(self):
        try:
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=self.fh, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self) -> dict | None:
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.fh.close()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.path.read_text().splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for nm, val in zip(names, parts[5:9]):
                if val.lower() == "active":
                    reasons.add(nm)
        self.path.unlink(missing_ok=True)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


# ------------------------------------------------------------------ references

def measured_peak_hbm() -> tuple[float, str]:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            return float(json.loads(p.read_text())["hbm_gbs"]), "measured"
        except Exception:
            pass
    return 6650.0, "fallback"


def ncu_traffic() -> float | None:
    """DRAM bytes per launch of the kNN radiance kernel from the committed
    ncu summary (profiles/knn_radiance_traffic.json), scaled to this
    workload's query count when the capture ran a smaller case."""
    p = ROOT / "profiles" / "knn_radiance_traffic.json"
    if not p.exists():
        return None
    try:
        d = json.loads(p.read_text())
        return float(d["dram_bytes_per_launch_full_workload"])
    except Exception:
        return None


def cpu_reference_rate(photons, queries, n_queries: int, repeats: int = 1):
    """The reference's own photon map + radiance loop (oracle/_ref, compiled
    from the reference headers) on a bounded sample of the same queries,
    with every host thread. Returns (queries/s, threads, seconds)."""
    from oracle import oracle as O
    if not O.ref_available():
        return None
    ref = O.RefPhotonMap(photons)
    sample = np.ascontiguousarray(queries[:n_queries])
    t0 = time.perf_counter()
    for _ in range(repeats):
        ref.radiance(sample, K_NEAREST, N_EMIT)
    dt = time.perf_counter() - t0
    threads = O.ref_threads()
    ref.close()
    return n_queries * repeats / dt, threads, dt


# ---------------------------------------------------------------- render rates

RENDER_CONFIGS = {
    # 256^2, 100k photons, k=100, 16 spp, no final gathering
    "cornell_256_100k_direct": dict(width=256, height=256, spp=16, photons=100_000, k=100, fg=0, n_gather=1),
    # 512^2, 1M photons, k=100, final gathering with 16 gather rays; timed on
    # 2 of the setting's 100 spp (samples/s is per sample)
    "cornell_512_1M_fg16": dict(width=512, height=512, spp=2, photons=1_000_000, k=100, fg=1, n_gather=16),
    # the same with the reference integrator's single gather ray per hit
    # (integrator.h:292-309), the setting its CPU time is taken on
    "cornell_512_1M_fg1": dict(width=512, height=512, spp=4, photons=1_000_000, k=100, fg=1,
                            n_gather=1),
    # caustics scene (mirror and glass icospheres, 512x512 water heightfield;
    # 563,238 triangles), 1M global + 10M caustics photons, k=100, final
    # gathering; timed on 2 of the setting's 64 spp
    "caustics_512_11M_fg1": dict(width=512, height=512, spp=2, photons=1_000_000, k=100, fg=1, n_gather=1,
                    scene="caustics", caustics_multiplier=10.0),
}
RENDER_REPEATS = 3           # timed renders per setting (median reported)
CPU_RENDER_BUDGET_S = 6.0   # per config, for the reference integrator's bounded sample


def cpu_render_rate(mesh, pmi, c) -> dict | None:
    """The reference's own PhotonMapping::integrate in the loop of
    examples/main.cpp (oracle/_ref, compiled from the reference headers),
    over the same photon maps, on a bounded band of rows in the middle of
    the image. Returns the samples/s record."""
    from oracle import oracle as O
    from photon_mapping_b200 import scene as S
    if c["n_gather"] != 1 or not O.ref_integrator_available():
        return None
    with tempfile.TemporaryDirectory() as td:
        path = Path(td) / "scene.obj"
        S.write_obj(mesh, path)
        ref = O.RefIntegrator(path)
    ref.set_maps(pmi.global_map.photons(), pmi.caustics_map.photons(), c["photons"], c["k"],
                 1.0, c["k"], c["fg"], MAX_DEPTH)
    cam = S.CAMERA
    w, h, spp = c["width"], c["height"], c["spp"]
    args = (cam["position"], cam["forward"], cam["fov"], w, h, spp)
    rows = 2
    _, secs = ref.render(*args, h // 2 - 1, h // 2 + 1)
    rows = int(min(max(rows * CPU_RENDER_BUDGET_S / max(secs, 1e-3), 2), h))
    row0 = (h - rows) // 2
    _, secs = ref.render(*args, row0, row0 + rows)
    ref.close()
    return {"value": rows * w * spp / secs, "unit": "samples/s", "cores": O.RefIntegrator.threads(),
            "kind": "reference",
            "sample": (f"rows {row0}-{row0 + rows - 1} of {w}x{h} at {spp} spp through the "
                       f"reference's Scene + PhotonMapping (scene.h, integrator.h, g++ -O3 "
                       f"-fopenmp) over the same photon maps, {secs:.1f} s")}


def knn_uniform_cube(ctx, d_q, nq: int, flush, stream, steps: int, warmup: int, dev) -> dict:
    """The kNN radiance kernel on a second photon set: 1,000,000 photons
    uniform in the unit cube (a volume, where the traced map lies on
    surfaces), answering the same primary-hit queries at k = 100, timed like
    the headline step (CUDA events on the launching stream, L2 flushed)."""
    import torch
    from photon_mapping_b200 import PhotonMap
    from photon_mapping_b200 import _native as N
    from photon_mapping_b200 import workloads as W
    n = 1_000_000
    pm = PhotonMap(ctx, map_id=N.PM_MAP_CAUSTICS)
    pm.setPhotons(W.uniform_photons(n, seed=0))
    pm.build()
    out = torch.empty((nq, 3), dtype=torch.float32, device=dev)

    def step():
        ctx.check(ctx.lib.pm_photonmap_radiance_device(
            ctx.handle, N.PM_MAP_CAUSTICS, d_q.data_ptr(), nq, K_NEAREST, n, out.data_ptr(),
            stream.cuda_stream), "pm_photonmap_radiance_device")

    for _ in range(max(warmup, 0)):
        flush.zero_()
        step()
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
           for _ in range(steps)]
    torch.cuda.synchronize(dev)
    for e0, e1 in evs:
        flush.zero_()
        e0.record(stream)
        step()
        e1.record(stream)
    torch.cuda.synchronize(dev)
    ms = sum(e0.elapsed_time(e1) for e0, e1 in evs) / len(evs)
    ctx.set_stats(True)
    step()
    torch.cuda.synchronize(dev)
    st = ctx.get_stats(reset=True)
    ctx.set_stats(False)
    peak, _ = measured_peak_hbm()
    achieved = nq * BYTES_PER_QUERY / (ms / 1e3) / 1e9
    return {
        "workload": "1000000 photons uniform in the unit cube, the same primary-hit queries, k=100",
        "photons": n, "k": K_NEAREST, "queries": nq, "ms_per_step": ms,
        "queries_per_s": nq / (ms / 1e3), "achieved_gbs": achieved, "frac": achieved / peak,
        "knn_per_query": {k2: v / max(st["queries"], 1) for k2, v in st.items() if k2 != "queries"},
    }


def workload_parity(ctx, photons, queries, rgb) -> dict:
    """Exactness of the timed workload on a sample of its queries (outside
    the timed region): the neighbour lists of the same query stream (every
    query, in pixel order, through pm_photonmap_knn) against the oracle's
    brute-force exact kNN, and the timed steps' radiance `rgb` against the
    FP64 recomputation on the oracle's neighbour sets."""
    from oracle import oracle as O
    from photon_mapping_b200 import PM_MAP_GLOBAL, PhotonMap
    from photon_mapping_b200 import workloads as W
    pm = PhotonMap(ctx, PM_MAP_GLOBAL)
    idx, cnt, md2 = pm.query_knn(queries[:, :3], K_NEAREST)
    s = W.parity_sample(queries.shape[0])
    t0 = time.perf_counter()
    oidx, ocnt, omd2 = O.knn(photons, queries[s, :3], K_NEAREST)
    secs = time.perf_counter() - t0
    mism = int(((idx[s] != oidx).any(axis=1) | (md2[s] != omd2) | (cnt[s] != ocnt)).sum())
    want = O.radiance_fp64(photons, oidx, ocnt, omd2, queries[s], N_EMIT)
    err = np.abs(rgb[s] - want) / np.maximum(np.abs(want), 1e-30)
    return {"sample": int(s.size), "mismatches": mism, "max_rel_err": float(err.max()),
            "tolerance": 1e-5,
            "oracle": ("brute-force exact kNN over every photon (FP32 distance in the reference's "
                       "order, ties to the smaller index), radiance recomputed in FP64"),
            "sample_kind": ("runs of 64 consecutive queries from work-item starts, the last 64, "
                            "first queries of 512 work items, 1024 random"),
            "oracle_s": secs}


def render_rates(ctx, sc, mesh, camera, dev, cpu: bool) -> dict:
    """Camera samples per second of pm_render (host API, wall clock) for
    the configs above, photon maps traced beforehand; beside each, the
    reference integrator's CPU rate where its settings match."""
    import torch
    from photon_mapping_b200 import scene as S
    from photon_mapping_b200.integrator import PhotonMapping
    out = {}
    for name, c in RENDER_CONFIGS.items():
        mult = c.get("caustics_multiplier", 1.0)
        scene_mesh, scene_dev = mesh, sc
        trace_s = None
        if c.get("scene") == "caustics":
            scene_mesh = S.caustics_scene(0)
            scene_dev = S.Scene(ctx)
            scene_dev.setMesh(scene_mesh)
            scene_dev.build()
        pmi = PhotonMapping(c["photons"], c["k"], mult, c["k"], c["fg"], MAX_DEPTH, ctx=ctx)
        pmi.build(scene_dev, seed=TRACE_SEED)
        if c.get("scene") == "caustics":
            torch.cuda.synchronize(dev)
            t0 = time.perf_counter()
            trace = pmi.build(scene_dev, seed=TRACE_SEED)
            trace_s = time.perf_counter() - t0
        # warm-up at the same setting (the render buffers reach their size)
        pmi.render(camera, c["width"], c["height"], c["spp"], n_gather=c["n_gather"])
        times = []
        for _ in range(RENDER_REPEATS):
            torch.cuda.synchronize(dev)
            t0 = time.perf_counter()
            img, st = pmi.render(camera, c["width"], c["height"], c["spp"],
                                 n_gather=c["n_gather"])
            times.append(time.perf_counter() - t0)
        dt = statistics.median(times)
        n = c["width"] * c["height"] * c["spp"]
        out[name] = {"samples_per_s": n / dt, "seconds": dt, "repeats": RENDER_REPEATS, **c,
                     "queries_global": st["queries_global"],
                     "queries_caustics": st["queries_caustics"], "passes": st["passes"],
                     "mean_radiance": float(img.mean()),
                     # closest-hit queries of the camera pass (camera, specular,
                     # shadow and gather rays) over its kernels' device time
                     "camera_rays": st["rays"], "camera_ms": st["camera_ms"],
                     "camera_rays_per_s": st["rays"] / (st["camera_ms"] / 1e3)
                     if st["camera_ms"] > 0 else None,
                     "estimate_ms": st["estimate_ms"]}
        if trace_s is not None:
            rays = sum(int(v["rays"]) for v in trace.values())
            kms = sum(float(v["trace_ms"]) for v in trace.values())
            out[name]["photon_trace"] = {
                "seconds": trace_s, "triangles": int(scene_mesh.n_faces),
                "emitted": c["photons"] + int(c["photons"] * mult),
                "stored": {k: int(v["stored"]) for k, v in trace.items()},
                "photons_per_s": (c["photons"] + c["photons"] * mult) / trace_s,
                "rays": rays, "trace_kernel_ms": kms,
                "rays_per_s": rays / (kms / 1e3) if kms > 0 else None}
        if cpu and c.get("scene") != "caustics":
            out[name]["cpu_reference"] = cpu_render_rate(mesh, pmi, c)
        if scene_dev is not sc:
            sc.build()   # the bench scene back on the context
    return out


# ------------------------------------------------------------------ gradients

# The Cornell box at 256^2, 1M photons, k = 50, final
# gathering, 16 spp; loss = MSE against a render with seed-perturbed albedos
# (8 materials x RGB) and emission
GRAD_CONFIG = dict(width=256, height=256, spp=16, photons=1_000_000, k=50, fg=1, n_gather=1)
GRAD_STEPS = 5


def gradient_rates(ctx, mesh, camera, dev) -> dict:
    """Gradient evaluations per second (forward render + device adjoint,
    photon maps traced in every evaluation) against the plain per-scene
    loop (PhotonMapping.build + render) on the same setting, and central
    finite differences (decisions frozen) of 4 parameter channels against
    the adjoint at full size."""
    import torch
    from photon_mapping_b200 import differentiable as D
    from photon_mapping_b200.integrator import PhotonMapping
    c = GRAD_CONFIG
    r = D.DiffRenderer(ctx, mesh, camera, c["width"], c["height"], c["spp"], c["photons"],
                       c["k"], final_gathering_depth=c["fg"], max_depth=MAX_DEPTH,
                       n_gather=c["n_gather"], seed=TRACE_SEED)
    a0, e0 = r.base()
    ta, te = D.perturbed_parameters(a0, e0, seed=0)
    target = r.forward(ta, te).astype(np.float64)
    for _ in range(2):
        r.loss_and_grad(a0, e0, target)
    torch.cuda.synchronize(dev)
    t_fwd, t_bwd = [], []
    for _ in range(GRAD_STEPS):
        t0 = time.perf_counter()
        img = r.forward(a0, e0)
        t1 = time.perf_counter()
        diff = img.astype(np.float64) - target
        loss = float(np.mean(diff * diff))
        ga, ge = r.backward((2.0 / diff.size) * diff)
        t2 = time.perf_counter()
        t_fwd.append(t1 - t0)
        t_bwd.append(t2 - t1)
    grad_s = (sum(t_fwd) + sum(t_bwd)) / GRAD_STEPS
    pmi = PhotonMapping(c["photons"], c["k"], 1.0, c["k"], c["fg"], MAX_DEPTH, ctx=ctx)
    pmi.build(r.scene, seed=TRACE_SEED)
    plain, _ = pmi.render(camera, c["width"], c["height"], c["spp"], n_gather=c["n_gather"])
    t_plain = []
    for _ in range(GRAD_STEPS):
        t0 = time.perf_counter()
        pmi.build(r.scene, seed=TRACE_SEED)
        pmi.render(camera, c["width"], c["height"], c["spp"], n_gather=c["n_gather"])
        t_plain.append(time.perf_counter() - t0)
    plain_s = sum(t_plain) / GRAD_STEPS
    which = [(2, 0), (3, 1), (6, 2), (len(a0), 0)]   # floor R, leftWall G, shortBox B, Le R
    fd = r.finite_differences(a0, e0, target, h=1e-3, which=which)
    g = np.concatenate([ga, ge[None]])
    fd_err = max(abs(g[p, ch] - fd[p, ch]) / max(abs(fd[p, ch]), 1e-30) for p, ch in which)
    return {
        "workload": ("Cornell box (8 material albedos x RGB + emission RGB = 27 "
                     f"parameters), {c['width']}x{c['height']}, {c['spp']} spp, "
                     f"{c['photons']} photons, k={c['k']}, final gathering; MSE loss against "
                     "a render with seed-perturbed parameters"),
        "grad_evals_per_s": 1.0 / grad_s,
        "forward_s": sum(t_fwd) / GRAD_STEPS,
        "backward_s": sum(t_bwd) / GRAD_STEPS,
        "plain_evals_per_s": 1.0 / plain_s,
        "grad_vs_plain": plain_s / grad_s,
        "image_rmse_vs_plain": float(np.sqrt(np.mean((img.astype(np.float64) - plain) ** 2))),
        "loss": loss,
        "fd_check": {"channels": which, "h": 1e-3, "max_rel_err": fd_err},
        "timing": "host wall clock per evaluation (photon trace + map build + render "
                  "[+ adjoint]), inputs and image on the host",
    }


# ------------------------------------------------------------- batched render

BATCH_STEPS = 3


def batched_rates(n_scenes: int, dev) -> dict:
    """n_scenes random scenes rendered as one batch (one step =
    every scene's photon trace, map build, camera pass, kNN estimates and
    resolve; CUDA graph, autotuned launch shapes) against the per-scene
    sequential loop over the same scenes; the images must be identical."""
    import torch
    from photon_mapping_b200 import batch as B
    scenes = [B.random_scene(1000 + s) for s in range(n_scenes)]
    samples = sum(sc["width"] * sc["height"] * sc["spp"] for sc in scenes)
    seq = B.Sequential(scenes)
    seq.render()                                   # warm-up
    seq_s = []
    for _ in range(BATCH_STEPS):
        imgs, secs = seq.render()
        seq_s.append(secs)
    seq.close()
    del seq
    torch.cuda.synchronize(dev)
    br = B.BatchRenderer(scenes)
    t0 = time.perf_counter()
    best, tune_ms = br.autotune()
    tune_s = time.perf_counter() - t0
    br.render(use_graph=True)                      # capture + warm-up
    br.render(use_graph=True)
    dev_ms, wall_s = [], []
    for _ in range(BATCH_STEPS):
        t0 = time.perf_counter()
        dev_ms.append(br.render(use_graph=True))
        wall_s.append(time.perf_counter() - t0)
    nograph_ms = br.render(use_graph=False)
    stage_ms = [br.stage_times() for _ in range(3)]
    stages = {k: min(st[k] for st in stage_ms) for k in stage_ms[0]}
    max_diff = max(float(np.abs(br.image(i) - imgs[i]).max()) for i in range(n_scenes))
    stored, queries = br.counts()
    br.close()
    step_s = sum(wall_s) / len(wall_s)
    seq_step = sum(seq_s) / len(seq_s)
    tris = [sc["mesh"].n_faces for sc in scenes]
    return {
        "workload": (f"{n_scenes} random Cornell variants (1-40 boxes, displaced "
                     "heightfield floor, triangles log-uniform 1k-500k), photons log-uniform "
                     "100k-4M, k in {50,100}, square images side log-uniform 128-1024, "
                     f"{scenes[0]['spp']} spp, photon-map estimate at the first diffuse hit"),
        "scenes": n_scenes,
        "triangles": {"min": min(tris), "max": max(tris), "total": sum(tris)},
        "photons_emitted": sum(sc["photons"] for sc in scenes),
        "photons_stored": int(stored.sum()),
        "queries": int(queries.sum()),
        "samples_per_step": samples,
        "batched": {"step_ms_device": sum(dev_ms) / len(dev_ms), "step_s_wall": step_s,
                    "samples_per_s": samples / step_s, "scenes_per_s": n_scenes / step_s,
                    "step_ms_without_graph": nograph_ms},
        "sequential": {"step_s_wall": seq_step, "samples_per_s": samples / seq_step,
                       "scenes_per_s": n_scenes / seq_step},
        "batched_vs_sequential": seq_step / step_s,
        "max_abs_image_difference": max_diff,
        "tuning": best,
        "autotune_stage_ms": {"trace": tune_ms[0], "camera": tune_ms[1], "knn": tune_ms[2]},
        "stage_ms": stages,
        "autotune_s": tune_s,
    }


# -------------------------------------------------------------------- our arm

def run_ours(args) -> None:
    import torch
    world, rank, local = dist_env()
    torch.cuda.set_device(local)
    dist = dist_init(world, "nccl")
    dev = torch.device("cuda", local)

    from photon_mapping_b200 import Context
    from photon_mapping_b200 import scene as S
    from photon_mapping_b200 import workloads as W
    from photon_mapping_b200.integrator import PhotonMapping
    mesh, camera = scene_and_camera()
    ctx = Context(local)
    lib = ctx.lib
    sc = S.Scene(ctx)
    sc.setMesh(mesh)
    sc.build()
    pmi = PhotonMapping(N_EMIT, K_NEAREST, 1.0, K_NEAREST, 0, MAX_DEPTH, ctx=ctx)
    pmi.build(sc, seed=TRACE_SEED)            # warm-up trace
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    trace_stats = pmi.build(sc, seed=TRACE_SEED)["global"]
    trace_s = time.perf_counter() - t0
    photons = pmi.global_map.photons()
    o, d = W.camera_rays(camera, IMAGE_W, IMAGE_H, SPP)
    queries = W.hit_queries(mesh, o, d, sc.intersect(o, d))
    nq = queries.shape[0]

    d_q = torch.from_numpy(queries).to(dev)
    d_out = torch.empty((nq, 3), dtype=torch.float32, device=dev)
    flush = torch.empty(64 << 20, dtype=torch.float32, device=dev)  # 256 MiB > L2
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)

    def step():
        st = lib.pm_photonmap_radiance_device(ctx.handle, 0, d_q.data_ptr(), nq, K_NEAREST,
                                              N_EMIT, d_out.data_ptr(), stream.cuda_stream)
        ctx.check(st, "pm_photonmap_radiance_device")

    for _ in range(max(args.warmup, 0)):
        flush.zero_()
        step()
    torch.cuda.synchronize(dev)

    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
           for _ in range(args.steps)]
    clocks = ClockSampler(local)
    if dist:
        dist.barrier()
    torch.cuda.synchronize(dev)
    clocks.start()
    t_wall = time.perf_counter()
    for e0, e1 in evs:
        flush.zero_()
        e0.record(stream)
        step()
        e1.record(stream)
    torch.cuda.synchronize(dev)
    t_wall = time.perf_counter() - t_wall
    if dist:
        dist.barrier()
    times = [e0.elapsed_time(e1) for e0, e1 in evs]
    ms = max_over_ranks(dist, sum(times) / len(times), dev)
    value = world * nq / (ms / 1e3)

    # e2e through the C ABI with pinned host buffers
    h_q = torch.from_numpy(queries).pin_memory()
    h_out = torch.empty((nq, 3), dtype=torch.float32).pin_memory()

    def e2e_step():
        st = lib.pm_photonmap_radiance(ctx.handle, 0, h_q.data_ptr(), nq, K_NEAREST, N_EMIT,
                                       h_out.data_ptr())
        ctx.check(st, "pm_photonmap_radiance")

    for _ in range(max(args.warmup, 1)):
        e2e_step()
    if dist:
        dist.barrier()
    e2e_times = []
    for _ in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        e2e_step()
        e2e_times.append(time.perf_counter() - t0)
    e2e_s = max_over_ranks(dist, sum(e2e_times) / len(e2e_times), dev)
    e2e_value = world * nq / e2e_s
    clk = clocks.stop()  # sampled over the timed steps and the e2e steps

    parity = None
    if rank == 0:
        parity = workload_parity(ctx, photons, queries, d_out.cpu().numpy())

    # one more (untimed) pass with the kernel's counters on
    ctx.set_stats(True)
    step()
    torch.cuda.synchronize(dev)
    st = ctx.get_stats(reset=True)
    ctx.set_stats(False)
    per_q = {k2: v / max(st["queries"], 1) for k2, v in st.items() if k2 != "queries"}
    uniform = knn_uniform_cube(ctx, d_q, nq, flush, stream, args.steps, args.warmup, dev)

    render = {} if args.no_render else render_rates(
        ctx, sc, mesh, camera, dev, cpu=(rank == 0 and world == 1 and not args.no_cpu_baseline))

    grad = None if args.no_grad else gradient_rates(ctx, mesh, camera, dev)
    batched = None if args.no_batch else batched_rates(args.batch_scenes, dev)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        r = cpu_reference_rate(photons, queries, CPU_SAMPLE_QUERIES)
        if r:
            rate, threads, secs = r
            cpu = {"value": rate, "unit": "queries/s", "cores": threads, "kind": "reference",
                   "sample": (f"{CPU_SAMPLE_QUERIES} of the {nq} queries through the reference's "
                              f"PhotonMap + radiance loop (photon_map.h, integrator.h:133-152 "
                              f"compiled with g++ -O3 -fopenmp), {secs:.1f} s")}

    peak, peak_kind = measured_peak_hbm()
    achieved = nq * BYTES_PER_QUERY / (ms / 1e3) / 1e9
    traffic = ncu_traffic()
    line = {
        "metric": METRIC,
        "value": value,
        "unit": "queries/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic (procedural Cornell box, seeded photon tracing and camera jitter)",
        "config": config_dict(nq, int(photons.shape[0])),
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic,
                     "peak_source": ("measured (MEASURED_PEAKS.json hbm_gbs)"
                                     if peak_kind == "measured" else
                                     "fallback 6650 GB/s (MEASURED_PEAKS.json absent)"),
                     "bytes_per_query": BYTES_PER_QUERY},
        "cpu_baseline": cpu,
        "e2e": {"value": e2e_value, "unit": "queries/s",
                "h2d_bytes_per_step": int(queries.nbytes),
                "d2h_bytes_per_step": int(nq * 3 * 4)},
        "gpu_launches": args.steps,
        "parity": parity,
        "knn_per_query": per_q,
        "knn_uniform_cube": uniform,
        "photon_trace": {"emitted": N_EMIT, "stored": trace_stats["stored"],
                         "seconds": trace_s, "photons_per_s": N_EMIT / trace_s,
                         "includes": "emission, tracing, ordering and the map build",
                         "rays": trace_stats["rays"],
                         "trace_kernel_ms": trace_stats["trace_ms"],
                         "build_ms": trace_stats["build_ms"],
                         "rays_per_s": trace_stats["rays"] / (trace_stats["trace_ms"] / 1e3)
                         if trace_stats["trace_ms"] > 0 else None},
        "render": render,
        "gradient": grad,
        "batched": batched,
        "clocks": clk,
        "wall_s_timed_region": t_wall,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    ctx.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()


# ------------------------------------------------------------------ convergence

REF_BAND_BUDGET_S = 20.0


def run_convergence(args) -> None:
    """One JSON line per render setting: the device render's error against the
    path-traced image (photon_mapping_b200.configs), and on a band of rows
    the same error of the reference's own PhotonMapping (its own photon
    tracing and camera pass, oracle/_ref, on the host cores) against the
    same path-traced image. The reference integrator has one gather ray per
    hit, so settings with more are reported without it."""
    from oracle import oracle as O
    from photon_mapping_b200 import Context
    from photon_mapping_b200 import configs as CF
    from photon_mapping_b200 import scene as S
    ctx = Context(0)
    for name in (args.convergence or CF.NAMES):
        rec, img, pt = CF.run_config(ctx, name, args.pt_spp, return_images=True)
        c = CF.CONFIGS[name]
        rec["reference"] = None
        if c["n_gather"] == 1 and O.ref_integrator_available():
            with tempfile.TemporaryDirectory() as td:
                path = Path(td) / "scene.obj"
                S.write_obj(CF.make_scene(c["scene"]), path)
                ref = O.RefIntegrator(path)
            t_build = ref.build(c["photons"], c["k"], c["caustics_multiplier"], c["k"], c["fg"],
                                CF.MAX_DEPTH)
            cam = S.CAMERA
            w, h, spp = c["width"], c["height"], c["spp"]
            a = (cam["position"], cam["forward"], cam["fov"], w, h, spp)
            _, secs = ref.render(*a, h // 2 - 1, h // 2 + 1)
            rows = int(min(max(2 * REF_BAND_BUDGET_S / max(secs, 1e-3), 2), h))
            r0 = (h - rows) // 2
            band, secs = ref.render(*a, r0, r0 + rows)
            rec["reference"] = {
                "rows": [r0, r0 + rows], "build_s": t_build, "render_s": secs,
                "samples_per_s": rows * w * spp / secs, "cores": O.RefIntegrator.threads(),
                "photons_stored_global": ref.n_photons(),
                "error_vs_path_tracing": CF.image_error(band, pt[r0:r0 + rows]),
                "ours_on_same_rows": CF.image_error(img[r0:r0 + rows], pt[r0:r0 + rows]),
            }
            ref.close()
        print(json.dumps(rec), flush=True)
    ctx.close()


# -------------------------------------------------------------- reference arm

def run_reference(args) -> None:
    world, rank, local = dist_env()
    if rank != 0:
        return
    from oracle import oracle as O
    if not O.ref_available():
        try:
            O.build()
        except Exception as e:  # pragma: no cover
            print(json.dumps({"impl": "reference", "unavailable": f"reference build failed: {e}"}))
            return
    from photon_mapping_b200 import workloads as W
    mesh, camera = scene_and_camera()
    osc = O.OracleScene(mesh)
    photons, _ = osc.trace(0, TRACE_SEED, 0, N_EMIT, MAX_DEPTH)   # same photons as the GPU trace
    o, d = W.camera_rays(camera, IMAGE_W, IMAGE_H, SPP)
    queries = W.hit_queries(mesh, o, d, osc.intersect(W.rays8(o, d)))
    nq = queries.shape[0]
    ref = O.RefPhotonMap(photons)
    sample = np.ascontiguousarray(queries[:CPU_SAMPLE_QUERIES // 2])
    for _ in range(max(args.warmup, 0)):
        ref.radiance(sample[:2000], K_NEAREST, N_EMIT)
    times = []
    for s in range(args.steps):
        off = (s * sample.shape[0]) % max(nq - sample.shape[0], 1)
        chunk = np.ascontiguousarray(queries[off: off + sample.shape[0]])
        t0 = time.perf_counter()
        ref.radiance(chunk, K_NEAREST, N_EMIT)
        times.append(time.perf_counter() - t0)
    threads = O.ref_threads()
    ref.close()
    secs = sum(times) / len(times)
    value = sample.shape[0] / secs
    line = {
        "impl": "reference",
        "metric": METRIC,
        "value": value,
        "unit": "queries/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": secs * 1e3,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic (procedural Cornell box, seeded photon tracing and camera jitter)",
        "config": config_dict(nq, int(photons.shape[0])),
        "cpu_baseline": {"value": value, "unit": "queries/s", "cores": threads, "kind": "reference",
                         "sample": (f"{sample.shape[0]} queries per step through the reference's "
                                    "PhotonMap + radiance loop (g++ -O3 -fopenmp)")},
        "e2e": {"value": value, "unit": "queries/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_trace_render(args) -> None:
    from photon_mapping_b200 import Context
    from photon_mapping_b200 import scene as S
    from photon_mapping_b200.integrator import PhotonMapping
    caustics = args.trace_render == "caustics"
    mesh = S.caustics_scene(0) if caustics else S.cornell_box(0)
    _, camera = scene_and_camera()
    ctx = Context(0)
    sc = S.Scene(ctx)
    sc.setMesh(mesh)
    sc.build()
    pmi = PhotonMapping(N_EMIT, K_NEAREST, 10.0 if caustics else 1.0, K_NEAREST, 1, MAX_DEPTH,
                        ctx=ctx)
    pmi.build(sc, seed=TRACE_SEED)
    trace = pmi.build(sc, seed=TRACE_SEED)
    img, st = pmi.render(camera, 256, 256, 2)
    print(json.dumps({"scene": args.trace_render, "triangles": int(mesh.n_faces),
                      "trace": trace, "render": st, "mean_radiance": float(img.mean())}),
          flush=True)
    ctx.close()


def run_batch_stages(args) -> None:
    from photon_mapping_b200 import batch as B
    scenes = [B.random_scene(1000 + s) for s in range(args.batch_stages)]
    br = B.BatchRenderer(scenes)
    stored, queries = br.counts()
    print(json.dumps({"scenes": len(scenes), "photons_stored": int(stored.sum()),
                      "queries": int(queries.sum()), "stage_ms": br.stage_times()}), flush=True)
    br.close()


def main():
    args = parse_args()
    if args.batch_stages is not None:
        run_batch_stages(args)
    elif args.trace_render is not None:
        run_trace_render(args)
    elif args.convergence is not None:
        run_convergence(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()

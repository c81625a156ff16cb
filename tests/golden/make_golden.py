"""Generates tests/golden/knn_cases.npz from the reference's own code.

Run in a tree where the reference is present (oracle/Makefile compiles its
photon_map.h unchanged into oracle/_ref). For each case the file holds the
photon set, the query points, k, and what the reference returned:
PhotonMap::queryKNearestPhotons (photon_map.h:208-211) indices in its
return order, their count and maxDist2, plus the FP32 radiance estimate of
integrator.h:133-152 for the cases that carry radiance queries.

    python tests/golden/make_golden.py
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle import oracle as O  # noqa: E402
from photon_mapping_b200 import workloads as W  # noqa: E402

OUT = Path(__file__).resolve().parent / "knn_cases.npz"


def cases():
    rng = np.random.default_rng(20261203)
    lat = W.lattice_photons(12)
    yield "uniform", W.uniform_photons(2000, 0), rng.uniform(-0.2, 2.2, (256, 3)), 100, None
    wq = W.wall_queries(256, 1)
    yield "walls", W.wall_photons(2500, 0), wq[:, :3], 50, wq
    yield "lattice", lat, np.concatenate([lat[::9, 3:6], lat[::13, 3:6] + 0.0625]), 27, None
    yield "lattice_k100", lat, lat[::17, 3:6], 100, None
    yield "small_n_lt_k", W.uniform_photons(37, 3), rng.uniform(0, 2, (64, 3)), 100, None
    yield "k1", W.wall_photons(2500, 7), W.wall_queries(256, 8)[:, :3], 1, None
    dup = W.wall_photons(600, 9)
    dup = np.concatenate([dup, dup, dup[:200]])  # coincident photons
    dq = W.wall_queries(128, 10)
    dq[:64, 0:3] = dup[:64, 3:6]  # queries exactly on photons: dist2 == 0
    yield "duplicates", dup, dq[:, :3], 40, dq


def main() -> None:
    O.build()
    assert O.ref_available(), "reference tree not built into oracle/_ref"
    blob = {}
    names = []
    for name, ph, q, k, rq in cases():
        ph = np.ascontiguousarray(ph, np.float32)
        q = np.ascontiguousarray(q, np.float32)
        ref = O.RefPhotonMap(ph)
        idx, cnt, md2 = ref.knn(q, k)
        blob[f"{name}/photons"] = ph
        blob[f"{name}/queries"] = q
        blob[f"{name}/k"] = np.int32(k)
        blob[f"{name}/ref_idx"] = idx
        blob[f"{name}/ref_cnt"] = cnt
        blob[f"{name}/ref_maxd2"] = md2
        if rq is not None:
            rq = np.ascontiguousarray(rq, np.float32)
            n_emitted = 100000
            blob[f"{name}/rq"] = rq
            blob[f"{name}/n_emitted"] = np.int64(n_emitted)
            blob[f"{name}/ref_rgb"] = ref.radiance(rq, k, n_emitted)
        ref.close()
        names.append(name)
    blob["names"] = np.array(names)
    np.savez_compressed(OUT, **blob)
    print(f"wrote {OUT} ({OUT.stat().st_size} bytes): {names}")


if __name__ == "__main__":
    main()

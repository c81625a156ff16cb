"""Parity on the benchmarked kNN workload itself.

The benchmark times the radiance estimate (k = 100) over the global photon
map traced from 1,000,000 emitted photons in the procedural Cornell box
(3.26M stored photons on planar walls, with many exact distance ties) for
the primary hits of a 512x512x4-spp frame, answered in pixel order. This
test runs that workload through the same entry points and checks a sample
of over 4,000 queries (runs of consecutive queries, first queries of work
items, the end of the stream and random ones) against brute force:

* neighbour lists and maxDist2 bit-exact against the oracle's exact kNN
  (ties broken by the smaller photon index, photon_map.h:107-147,
  :166-183);
* radiance within 1e-5 relative of the FP64 recomputation on those
  neighbour sets (integrator.h:133-152);
* the reference's own KdTree (photon_map.h, compiled unchanged) on the
  same sample: its lists differ from the oracle's only among photons at the
  k-th distance (its pruning keeps another subset of tied photons).
"""
from __future__ import annotations

import numpy as np
import pytest

from oracle import oracle as O
from photon_mapping_b200 import workloads as W

pytestmark = pytest.mark.gpu

K = 100
N_EMIT = 1_000_000
RTOL = 1e-5


@pytest.fixture(scope="module")
def workload(ctx):
    sc, mesh, camera, photons, queries, stats = W.traced_cornell_knn_workload(ctx, N_EMIT)
    return photons, queries, stats


def test_workload_shape(workload):
    photons, queries, stats = workload
    assert photons.shape[0] == stats["stored"] > 3_000_000
    assert queries.shape[0] > 900_000


def test_sampled_queries_exact(ctx, workload):
    from photon_mapping_b200 import PM_MAP_GLOBAL, PhotonMap
    photons, queries, _ = workload
    pm = PhotonMap(ctx, PM_MAP_GLOBAL)         # the traced map, as the benchmark uses it
    nq = queries.shape[0]
    idx, cnt, md2 = pm.query_knn(queries[:, :3], K)     # every query, in pixel order
    rad = pm.radiance(queries, K, N_EMIT)
    s = W.parity_sample(nq)
    assert s.size >= 4096
    oidx, ocnt, omd2 = O.knn(photons, queries[s, :3], K)
    bad = np.flatnonzero((idx[s] != oidx).any(axis=1) | (md2[s] != omd2) | (cnt[s] != ocnt))
    assert bad.size == 0, f"{bad.size} of {s.size} sampled queries differ, first {s[bad[:5]]}"
    want = O.radiance_fp64(photons, oidx, ocnt, omd2, queries[s], N_EMIT)
    err = np.abs(rad[s] - want) / np.maximum(np.abs(want), 1e-30)
    assert err.max() <= RTOL, f"radiance max rel err {err.max():.3e}"


@pytest.mark.skipif(not O.ref_available(), reason="reference photon map not built")
def test_reference_kdtree_agrees_up_to_ties(workload):
    photons, queries, _ = workload
    s = W.parity_sample(queries.shape[0])[::4]
    q = queries[s, :3]
    oidx, ocnt, omd2 = O.knn(photons, q, K)
    ref = O.RefPhotonMap(photons)
    try:
        ridx, rcnt, rmd2 = ref.knn(q, K)
    finally:
        ref.close()
    np.testing.assert_array_equal(rcnt, ocnt)
    np.testing.assert_array_equal(rmd2, omd2)
    differ = np.flatnonzero((ridx != oidx).any(axis=1))
    pos = photons[:, 3:6]
    for i in differ:
        a, b = set(oidx[i].tolist()), set(ridx[i].tolist())
        if a == b:
            continue     # same set, another order among equal distances
        d = q[i] - pos[np.array(sorted(a ^ b))]
        d2 = ((d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1]) + d[:, 2] * d[:, 2]).astype(np.float32)
        assert (d2 == omd2[i]).all(), f"query {s[i]}: lists differ below the k-th distance"
    print(f"reference KdTree: {s.size - differ.size} of {s.size} lists identical, "
          f"{differ.size} differ among photons at the k-th distance")

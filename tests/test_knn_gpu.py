"""Parity of the device photon map (pm_photonmap_* through the C ABI) with
the oracle and with the reference's golden vectors.

Bar: neighbour index lists bit-exact (same indices, same order, same
maxDist2) against exact kNN with ties broken by the smaller photon index;
radiance within 1e-5 relative of the FP64 recomputation on the same
neighbour sets.
"""
from __future__ import annotations

import numpy as np
import pytest

from oracle import oracle as O
from photon_mapping_b200 import PhotonMap, PMError
from photon_mapping_b200 import workloads as W

pytestmark = pytest.mark.gpu

RTOL = 1e-5  # radiance vs FP64, relative


def gpu_map(ctx, photons, map_id=0):
    pm = PhotonMap(ctx, map_id)
    pm.setPhotons(photons)
    pm.build()
    return pm


def assert_radiance_close(got, want, rtol=RTOL, what=""):
    want = np.asarray(want, np.float64)
    got = np.asarray(got, np.float64)
    fin = np.isfinite(want)
    np.testing.assert_array_equal(np.isfinite(got), fin, err_msg=what)
    scale = np.maximum(np.abs(want[fin]), 1e-30)
    err = np.abs(got[fin] - want[fin]) / scale
    assert err.max(initial=0.0) <= rtol, f"{what}: max rel err {err.max():.3e}"


def test_golden_knn_exact(ctx, golden_knn):
    for name, c in golden_knn.items():
        ph, q, k = c["photons"], c["queries"], int(c["k"])
        pm = gpu_map(ctx, ph)
        idx, cnt, md2 = pm.query_knn(q, k)
        oidx, ocnt, omd2 = O.knn(ph, q, k)
        np.testing.assert_array_equal(cnt, ocnt, err_msg=name)
        np.testing.assert_array_equal(md2, omd2, err_msg=name)
        np.testing.assert_array_equal(idx, oidx, err_msg=name)
        # and the reference itself wherever it did not break a tie differently
        same_ref = (oidx == c["ref_idx"]).all(axis=1)
        np.testing.assert_array_equal(idx[same_ref], c["ref_idx"][same_ref], err_msg=name)
        np.testing.assert_array_equal(md2, c["ref_maxd2"], err_msg=name)


def test_golden_radiance(ctx, golden_knn):
    for name, c in golden_knn.items():
        if "rq" not in c:
            continue
        ph, rq, k, ne = c["photons"], c["rq"], int(c["k"]), int(c["n_emitted"])
        pm = gpu_map(ctx, ph)
        got = pm.radiance(rq, k, ne)
        oidx, ocnt, omd2 = O.knn(ph, rq[:, :3], k)
        want = O.radiance_fp64(ph, oidx, ocnt, omd2, rq, ne)
        assert_radiance_close(got, want, what=name)
        assert_radiance_close(got, c["ref_rgb"], rtol=2e-5, what=name + " vs reference fp32")


@pytest.mark.parametrize("k", [1, 7, 32, 50, 100, 256, 300, 1024])
def test_random_walls_all_k(ctx, k):
    ph = W.wall_photons(30000, 100 + k)
    q = W.wall_queries(3000, 200 + k)
    pm = gpu_map(ctx, ph)
    idx, cnt, md2 = pm.query_knn(q[:, :3], k)
    oidx, ocnt, omd2 = O.knn(ph, q[:, :3], k)
    np.testing.assert_array_equal(idx, oidx)
    np.testing.assert_array_equal(cnt, ocnt)
    np.testing.assert_array_equal(md2, omd2)
    got = pm.radiance(q, k, 30000)
    assert_radiance_close(got, O.radiance_fp64(ph, oidx, ocnt, omd2, q, 30000), what=f"k={k}")


def test_query_order_does_not_change_results(ctx):
    """Coherent (warm-start) and shuffled (cold-start) query streams agree."""
    ph = W.wall_photons(50000, 5)
    rng = np.random.default_rng(6)
    q = W.wall_queries(4000, 7)
    q = q[np.lexsort((q[:, 2], q[:, 1], q[:, 0]))]  # spatially coherent order
    pm = gpu_map(ctx, ph)
    a = pm.query_knn(q[:, :3], 100)
    perm = rng.permutation(q.shape[0])
    b = pm.query_knn(q[perm, :3], 100)
    for x, y in zip(a, b):
        np.testing.assert_array_equal(x[perm], y)
    ra = pm.radiance(q, 100, 50000)
    rb = pm.radiance(q[perm], 100, 50000)
    assert_radiance_close(ra[perm], rb, rtol=1e-6, what="order")


def test_uniform_cube_and_far_queries(ctx):
    ph = W.uniform_photons(40000, 8)
    rng = np.random.default_rng(9)
    q = np.concatenate([rng.uniform(0, 2, (1500, 3)), rng.uniform(-5, 7, (500, 3))]).astype(np.float32)
    pm = gpu_map(ctx, ph)
    got = pm.query_knn(q, 64)
    want = O.knn(ph, q, 64)
    for g, w in zip(got, want):
        np.testing.assert_array_equal(g, w)


def test_edge_cases(ctx):
    # empty map: no neighbours, zero radiance (integrator.h:148 guard)
    pm = gpu_map(ctx, np.zeros((0, 9), np.float32))
    idx, cnt, md2 = pm.query_knn(np.zeros((5, 3), np.float32), 10)
    assert (cnt == 0).all() and (idx == -1).all() and (md2 == 0).all()
    assert (pm.radiance(W.wall_queries(5, 1), 10, 1000) == 0).all()
    assert pm.getNPhotons() == 0
    # fewer photons than k
    ph = W.uniform_photons(5, 2)
    pm = gpu_map(ctx, ph)
    idx, cnt, md2 = pm.query_knn(np.full((2, 3), 0.5, np.float32), 8)
    oidx, ocnt, omd2 = O.knn(ph, np.full((2, 3), 0.5, np.float32), 8)
    np.testing.assert_array_equal(idx, oidx)
    assert (cnt == 5).all()
    # a NaN query finds nothing
    idx, cnt, md2 = pm.query_knn(np.array([[np.nan, 0, 0]], np.float32), 3)
    assert cnt[0] == 0 and (idx == -1).all()
    # invalid k is an argument error, not a crash
    for bad_k in (0, -1, 1025):
        with pytest.raises(PMError) as e:
            pm.query_knn(np.zeros((1, 3), np.float32), bad_k)
        assert e.value.status == 1
    # single-photon queries mirror the reference interface
    ph = W.wall_photons(1000, 3)
    pm = gpu_map(ctx, ph)
    ids, md2 = pm.queryKNearestPhotons(ph[17, 3:6], 1)
    assert ids == [17] and md2 == 0.0
    np.testing.assert_array_equal(pm.getIthPhoton(17), ph[17])
    np.testing.assert_array_equal(pm.photons(), ph)


def test_map_not_built_is_reported(ctx):
    from photon_mapping_b200 import PM_MAP_CAUSTICS, Context
    c2 = Context(0)
    try:
        pm = PhotonMap(c2, PM_MAP_CAUSTICS)
        with pytest.raises(PMError) as e:
            pm.query_knn(np.zeros((1, 3), np.float32), 3)
        assert e.value.status == 4
    finally:
        c2.close()


def test_large_map_properties(ctx):
    """Full-size map (1.3M photons on the walls, more than 256 sort tiles):
    exactness on a sample against brute force, size-independent properties
    on all queries."""
    n = 1_300_000
    ph = W.wall_photons(n, 21)
    q = W.wall_queries(1 << 18, 22)
    pm = gpu_map(ctx, ph)
    idx, cnt, md2 = pm.query_knn(q[:, :3], 100)
    assert (cnt == 100).all()
    # maxDist2 is the distance of the first (farthest) photon returned
    p = ph[idx[:, 0], 3:6]
    d = q[:, :3] - p
    d2 = (d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1]) + d[:, 2] * d[:, 2]
    np.testing.assert_array_equal(d2.astype(np.float32), md2)
    # no duplicates in any list
    s = np.sort(idx, axis=1)
    assert (s[:, 1:] != s[:, :-1]).all()
    sample = np.random.default_rng(23).choice(q.shape[0], 512, replace=False)
    oidx, ocnt, omd2 = O.knn(ph, q[sample, :3], 100)
    np.testing.assert_array_equal(idx[sample], oidx)
    rad = pm.radiance(q, 100, n)
    assert_radiance_close(rad[sample], O.radiance_fp64(ph, oidx, ocnt, omd2, q[sample], n),
                          what="1M sample")


def test_page_locked_host_buffers(ctx):
    """Host-pointer calls with page-locked (mapped) buffers read the
    radiance queries in place (the index search: through a copy kernel) and
    write the results straight into the host buffers; the results equal
    those of pageable buffers, also for buffers that start off a 16-byte
    boundary and for a query count that is not a multiple of 8."""
    import ctypes as C
    import torch
    ph = W.wall_photons(100000, seed=7)
    pm = gpu_map(ctx, ph)
    q = W.wall_queries(70001, seed=8)
    want = pm.radiance(q, 50, 100000)
    widx, wcnt, wmd2 = pm.query_knn(q[:, :3], 30)
    hq = torch.from_numpy(np.ascontiguousarray(q)).pin_memory()
    hout = torch.zeros((q.shape[0], 3), dtype=torch.float32).pin_memory()
    ctx.check(ctx.lib.pm_photonmap_radiance(ctx.handle, 0, hq.data_ptr(), q.shape[0], 50, 100000,
                                            hout.data_ptr()), "pm_photonmap_radiance")
    np.testing.assert_array_equal(hout.numpy(), want)
    hp = torch.from_numpy(np.ascontiguousarray(q[:, :3])).pin_memory()
    hidx = torch.zeros((q.shape[0], 30), dtype=torch.int32).pin_memory()
    hcnt = torch.zeros(q.shape[0], dtype=torch.int32).pin_memory()
    hmd2 = torch.zeros(q.shape[0], dtype=torch.float32).pin_memory()
    ctx.check(ctx.lib.pm_photonmap_knn(ctx.handle, 0, hp.data_ptr(), q.shape[0], 30,
                                       hidx.data_ptr(), hcnt.data_ptr(), hmd2.data_ptr()),
              "pm_photonmap_knn")
    np.testing.assert_array_equal(hidx.numpy(), widx)
    np.testing.assert_array_equal(hcnt.numpy(), wcnt)
    np.testing.assert_array_equal(hmd2.numpy(), wmd2)
    # a query array whose size is not a multiple of 16 bytes (3 floats each)
    hp1 = torch.from_numpy(np.ascontiguousarray(q[:5, :3])).pin_memory()
    i1, c1, m1 = (np.zeros((5, 30), np.int32), np.zeros(5, np.int32), np.zeros(5, np.float32))
    ctx.check(ctx.lib.pm_photonmap_knn(ctx.handle, 0, hp1.data_ptr(), 5, 30, i1.ctypes.data,
                                       c1.ctypes.data, m1.ctypes.data), "pm_photonmap_knn")
    np.testing.assert_array_equal(i1, widx[:5])
    # mapped buffers 4 bytes off a 16-byte boundary: the queries are copied
    # first, the results are stored word by word
    n = q.shape[0]
    qbig = torch.zeros(q.size + 1, dtype=torch.float32).pin_memory()
    qbig[1:] = torch.from_numpy(np.ascontiguousarray(q).reshape(-1))
    obig = torch.zeros(3 * n + 1, dtype=torch.float32).pin_memory()
    ctx.check(ctx.lib.pm_photonmap_radiance(ctx.handle, 0, qbig[1:].data_ptr(), n, 50, 100000,
                                            obig[1:].data_ptr()), "pm_photonmap_radiance")
    np.testing.assert_array_equal(obig[1:].numpy().reshape(n, 3), want)
    assert obig[0].item() == 0.0
    # device buffers, output 4 bytes off a 16-byte boundary
    dq = torch.from_numpy(np.ascontiguousarray(q)).cuda()
    dout = torch.zeros(3 * n + 1, dtype=torch.float32, device="cuda")
    ctx.check(ctx.lib.pm_photonmap_radiance_device(ctx.handle, 0, dq.data_ptr(), n, 50, 100000,
                                                   dout[1:].data_ptr(), None),
              "pm_photonmap_radiance_device")
    torch.cuda.synchronize()
    np.testing.assert_array_equal(dout[1:].cpu().numpy().reshape(n, 3), want)
    assert dout[0].item() == 0.0


def test_ragged_query_counts_all_paths(ctx):
    """Query counts below one work item, ending inside a group of 8 or just
    past one: the pageable, page-locked and device paths give the same
    radiance, equal to the FP64 recomputation on the oracle's neighbours,
    and write nothing past the last query."""
    import torch
    ph = W.wall_photons(20000, 31)
    pm = gpu_map(ctx, ph)
    qall = W.wall_queries(80, 32)
    for n in (1, 3, 7, 8, 9, 15, 16, 17, 23, 33, 80):
        q = np.ascontiguousarray(qall[:n])
        want = pm.radiance(q, 30, 20000)
        oidx, ocnt, omd2 = O.knn(ph, q[:, :3], 30)
        assert_radiance_close(want, O.radiance_fp64(ph, oidx, ocnt, omd2, q, 20000),
                              what=f"n={n}")
        hq = torch.from_numpy(q).pin_memory()
        hout = torch.full((n + 1, 3), -7.0, dtype=torch.float32).pin_memory()
        ctx.check(ctx.lib.pm_photonmap_radiance(ctx.handle, 0, hq.data_ptr(), n, 30, 20000,
                                                hout.data_ptr()), "pm_photonmap_radiance")
        np.testing.assert_array_equal(hout[:n].numpy(), want)
        assert (hout[n].numpy() == -7.0).all()
        dq = torch.from_numpy(q).cuda()
        dout = torch.full((n + 1, 3), -7.0, dtype=torch.float32, device="cuda")
        ctx.check(ctx.lib.pm_photonmap_radiance_device(ctx.handle, 0, dq.data_ptr(), n, 30,
                                                       20000, dout.data_ptr(), None),
                  "pm_photonmap_radiance_device")
        torch.cuda.synchronize()
        np.testing.assert_array_equal(dout[:n].cpu().numpy(), want)
        assert (dout[n].cpu().numpy() == -7.0).all()


def test_stats_counters(ctx):
    """pm_ctx_set_stats / pm_ctx_get_stats: per-query counters of the
    radiance kernel are consistent and reset on request; disabled counters
    stay at zero."""
    ph = W.wall_photons(50000, 41)
    pm = gpu_map(ctx, ph)
    q = W.wall_queries(3000, 42)
    ctx.get_stats(reset=True)
    ctx.set_stats(True)
    try:
        pm.radiance(q, 50, 50000)
        st = ctx.get_stats(reset=True)
    finally:
        ctx.set_stats(False)
    assert st["queries"] == q.shape[0]
    assert st["walks"] >= st["queries"]
    assert st["candidates"] >= 50 * st["queries"]
    assert st["leaves"] > 0 and st["nodes"] > 0
    assert 0 < st["cold_starts"] <= st["queries"]
    assert st["selects"] >= 1
    pm.radiance(q, 50, 50000)
    assert all(v == 0 for v in ctx.get_stats().values())

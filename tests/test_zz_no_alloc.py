"""The allocation-free entry point, pm_photonmap_radiance_noalloc.

It serves callers that cannot call cudaMalloc (a plug-in whose host
application owns all device memory, a real-time loop that cannot take the
synchronisation an allocation implies): the caller hands over device
buffers and the library keeps its intermediates in a static device array.
These tests call it through the C ABI, several times in a row on different
inputs, and check each result against the context-based
pm_photonmap_radiance on the same inputs: the same kernels run on the same
photon set, so the results must be identical, bit for bit. The file is
collected last; it also passes alone in a fresh process.
"""
from __future__ import annotations

import numpy as np
import pytest

from photon_mapping_b200 import Context, PhotonMap
from photon_mapping_b200 import _native as N
from photon_mapping_b200 import workloads as W

pytestmark = pytest.mark.gpu


def noalloc_call(lib, photons_t, queries_t, out_t, k, n_emitted, stream):
    return lib.pm_photonmap_radiance_noalloc(
        photons_t.data_ptr(), photons_t.shape[0], queries_t.data_ptr(), queries_t.shape[0],
        int(k), int(n_emitted), out_t.data_ptr(), stream)


def test_noalloc_matches_context_entry_point():
    import torch
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    lib = N.load()
    stream = torch.cuda.current_stream(dev).cuda_stream
    cases = [
        # the largest photon set accepted
        (W.wall_photons(N.PM_NOALLOC_MAX_PHOTONS, 31), W.wall_queries(6000, 32), 100, 250000),
        # a second, smaller set right after it (the array keeps the last contents)
        (W.wall_photons(9000, 33), W.wall_queries(3000, 34), 40, 12345),
        # a query count that ends inside a group of 8
        (W.wall_photons(5000, 35), W.wall_queries(13, 36), 50, 5000),
        # k above the photon count: every photon is a neighbour
        (W.wall_photons(37, 37), W.wall_queries(100, 38), 64, 37),
        # no photons at all: zero radiance
        (np.zeros((0, 9), np.float32), W.wall_queries(21, 39), 10, 1000),
    ]
    with Context(0) as ctx:
        for ph, q, k, n_emit in cases:
            ph_t = torch.from_numpy(np.ascontiguousarray(ph)).to(dev)
            q_t = torch.from_numpy(q).to(dev)
            out_t = torch.full((q.shape[0], 3), float("nan"), device=dev)
            st = noalloc_call(lib, ph_t, q_t, out_t, k, n_emit, stream)
            assert st == N.PM_OK, N.status_string(st)
            torch.cuda.synchronize(dev)
            got = out_t.cpu().numpy()
            pm = PhotonMap(ctx)
            pm.setPhotons(ph)
            pm.build()
            want = pm.radiance(q, k, n_emit)
            np.testing.assert_array_equal(got, want, err_msg=f"{ph.shape[0]} photons, k={k}")
            if ph.shape[0] == 0:
                assert (got == 0).all()


def test_noalloc_rejects_oversized_photon_sets():
    import torch
    dev = torch.device("cuda", 0)
    lib = N.load()
    ph_t = torch.zeros((N.PM_NOALLOC_MAX_PHOTONS + 1, 9), device=dev)
    q_t = torch.zeros((4, 12), device=dev)
    out_t = torch.zeros((4, 3), device=dev)
    st = noalloc_call(lib, ph_t, q_t, out_t, 10, 100, None)
    assert st == N.PM_ERR_INVALID_ARGUMENT
    st = lib.pm_photonmap_radiance_noalloc(ph_t.data_ptr(), 100, q_t.data_ptr(), 4, 0, 100,
                                           out_t.data_ptr(), None)
    assert st == N.PM_ERR_INVALID_ARGUMENT

"""The batched renderer (pm_batch_*) against the oracle, scene by scene.

Each scene of a small batch (random Cornell variants and a small caustics
scene with a mirror and a glass sphere) must store exactly the photons the
oracle's restatement of PhotonMapping::build stores for it
(integrator.h:406-469, bit for bit), and render the image the oracle's
restatement of the render loop gives with those photons (examples/main.cpp
:26-64 with integrate at finalGatheringDepth 0), per pixel within the
render tests' tolerance (float summation order only). Checked for the
first step, for graph replays and again after autotuning.
"""
from __future__ import annotations

import numpy as np
import pytest

from oracle import oracle as O
from photon_mapping_b200 import batch as B
from photon_mapping_b200 import scene as S
from photon_mapping_b200.camera import Camera

pytestmark = pytest.mark.gpu

RTOL = 2e-5   # per pixel and channel, relative
ATOL = 1e-6


def scenes():
    out = [B.random_scene(s, tri_range=(600, 6000), photon_range=(3000, 20000),
                          side_range=(16, 48), ks=(10, 40), spp=2, max_depth=12)
           for s in (11, 12, 13)]
    cam = Camera(S.CAMERA["position"], S.CAMERA["forward"], S.CAMERA["fov"])
    out.append(dict(mesh=S.caustics_scene(0, grid=10, subdiv=1), camera=cam, width=32,
                    height=24, spp=2, k=16, photons=15000, seed=21, max_depth=12))
    return out


@pytest.fixture(scope="module")
def batch_and_oracle():
    scs = scenes()
    want = []
    for sc in scs:
        osc = O.OracleScene(sc["mesh"])
        ph, _ = osc.trace(0, sc["seed"], 0, sc["photons"], sc["max_depth"])
        img, _ = osc.render(ph, sc["photons"], np.zeros((0, 9), np.float32), 0,
                            sc["camera"].as_array(), sc["width"], sc["height"], sc["spp"],
                            sc["k"], sc["k"], 0, sc["max_depth"])
        want.append((ph, img))
    br = B.BatchRenderer(scs)
    yield scs, br, want
    br.close()


def check(br, scs, want):
    stored, queries = br.counts()
    for i, (ph, img) in enumerate(want):
        assert stored[i] == ph.shape[0], f"scene {i}"
        np.testing.assert_array_equal(br.photons(i), ph, err_msg=f"scene {i} photons")
        got = br.image(i)
        np.testing.assert_array_equal(np.isfinite(got), np.isfinite(img))
        np.testing.assert_allclose(got, img, rtol=RTOL, atol=ATOL, err_msg=f"scene {i} image")
        assert queries[i] > 0 and img.mean() > 0


def test_batch_matches_oracle(batch_and_oracle):
    scs, br, want = batch_and_oracle
    check(br, scs, want)          # the planning step
    for use_graph in (False, True, True):
        br.render(use_graph=use_graph)
        check(br, scs, want)


def test_batch_matches_oracle_after_autotune(batch_and_oracle):
    scs, br, want = batch_and_oracle
    br.autotune()
    for use_graph in (True, False):
        br.render(use_graph=use_graph)
        check(br, scs, want)

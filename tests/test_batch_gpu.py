"""The batched render (pm_batch_*) against the per-scene loop it replaces:
every scene's image bit-identical to PhotonMapping.build + render of that
scene on its own context, without and with the CUDA graph, before and after
autotuning; photons stored per scene equal to the per-scene trace."""
from __future__ import annotations

import numpy as np
import pytest

from photon_mapping_b200 import batch as B
from photon_mapping_b200 import scene as S
from photon_mapping_b200._native import PMError
from photon_mapping_b200.camera import Camera

pytestmark = pytest.mark.gpu


def small_scenes():
    scenes = [B.random_scene(s, tri_range=(600, 20000), photon_range=(3000, 40000),
                             side_range=(16, 72), ks=(10, 40), spp=2, max_depth=20)
              for s in range(5)]
    # one scene with a mirror and glass: specular branching in the camera pass
    cam = Camera(S.CAMERA["position"], S.CAMERA["forward"], S.CAMERA["fov"])
    scenes.append(dict(mesh=S.caustics_scene(0, grid=10, subdiv=1), camera=cam, width=40,
                       height=30, spp=2, k=16, photons=20000, seed=9, max_depth=12))
    return scenes


@pytest.fixture(scope="module")
def batch_and_reference():
    scenes = small_scenes()
    seq = B.Sequential(scenes)
    want, _ = seq.render()
    stored_seq = [pmi.stats["global"]["stored"] for pmi in seq.pmis]
    seq.close()
    br = B.BatchRenderer(scenes)
    yield scenes, br, want, stored_seq
    br.close()


def test_batch_matches_per_scene_loop(batch_and_reference):
    scenes, br, want, stored_seq = batch_and_reference
    stored, queries = br.counts()
    assert list(stored) == stored_seq
    assert (queries > 0).all()
    for use_graph in (False, True, True):
        ms = br.render(use_graph=use_graph)
        assert ms > 0
        for i in range(len(scenes)):
            np.testing.assert_array_equal(br.image(i), want[i])


def test_autotune_keeps_the_images(batch_and_reference):
    scenes, br, want, _ = batch_and_reference
    best, ms = br.autotune()
    assert best == br.tuning()
    assert best["bvh_stack"] in (16, 32, 64) and best["knn_warps"] in (4, 8)
    assert all(t > 0 for t in ms)
    for use_graph in (True, False):
        br.render(use_graph=use_graph)
        for i in range(len(scenes)):
            np.testing.assert_array_equal(br.image(i), want[i])
    # any valid setting renders the same images
    br.set_tuning(knn_warps=4, knn_chunk=7, knn_buffer=2048, bvh_stack=64, block=64)
    br.render(use_graph=True)
    for i in range(len(scenes)):
        np.testing.assert_array_equal(br.image(i), want[i])


def test_stage_times_cover_a_step(batch_and_reference):
    """pm_batch_stage_times runs one step stage by stage: six positive times
    whose sum is about one step's device time, and the images of that step
    are the per-scene loop's."""
    scenes, br, want, _ = batch_and_reference
    step = min(br.render(use_graph=False) for _ in range(3))
    st = br.stage_times()
    assert list(st) == ["trace", "maps", "camera", "sort", "knn", "resolve"]
    assert all(v > 0.0 for v in st.values()), st
    assert 0.5 * step < sum(st.values()) < 2.0 * step + 1.0, (st, step)
    for i in range(len(scenes)):
        np.testing.assert_array_equal(br.image(i), want[i])


def test_batch_scenes_with_no_or_few_photons():
    """The segmented map build with empty and nearly empty maps among full
    ones: a scene that emits no photons (its estimates are 0), scenes whose
    few stored photons fill less than one 8-photon group, and ordinary
    scenes. Images bit-identical to the per-scene loop; stored counts equal."""
    base = dict(tri_range=(600, 5000), side_range=(16, 40), ks=(10, 40), spp=2, max_depth=20)
    scenes = []
    for s, photons in enumerate([0, 1, 3, 20000, 7, 30000]):
        sc = B.random_scene(50 + s, photon_range=(1000, 2000), **base)
        sc["photons"] = photons
        scenes.append(sc)
    seq = B.Sequential(scenes)
    want, _ = seq.render()
    stored_seq = [pmi.stats["global"]["stored"] for pmi in seq.pmis]
    seq.close()
    br = B.BatchRenderer(scenes)
    try:
        stored, _ = br.counts()
        assert list(stored) == stored_seq
        assert stored[0] == 0
        for use_graph in (False, True):
            br.render(use_graph=use_graph)
            for i in range(len(scenes)):
                np.testing.assert_array_equal(br.image(i), want[i])
        for i in (1, 2, 4):
            ph = br.photons(i)
            assert ph.shape == (stored[i], 9)
    finally:
        br.close()


def test_batch_errors(batch_and_reference):
    scenes, br, _, _ = batch_and_reference
    with pytest.raises(PMError):
        br.set_tuning(knn_warps=9)
    with pytest.raises(PMError):
        br.set_tuning(bvh_stack=48)
    bad = dict(scenes[0], k=0)
    with pytest.raises(PMError):
        B.BatchRenderer([bad])

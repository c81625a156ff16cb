"""Output and fixture formats (no GPU): PFM images and binary photon files."""
from __future__ import annotations

import numpy as np
import pytest

from photon_mapping_b200 import workloads as W
from photon_mapping_b200.camera import Image
from photon_mapping_b200.photon_map import load_photons, save_photons


def test_pfm_round_trip(tmp_path):
    rng = np.random.default_rng(0)
    px = rng.uniform(0, 20, (7, 5, 3)).astype(np.float32)
    px[0, 0] = [np.inf, 0.0, 1e-30]
    img = Image(5, 7, px)
    img.writePFM(tmp_path / "a.pfm")
    back = Image.readPFM(tmp_path / "a.pfm")
    assert (back.width, back.height) == (5, 7)
    np.testing.assert_array_equal(back.pixels, px)
    # header and bottom-to-top rows as the format defines
    raw = (tmp_path / "a.pfm").read_bytes()
    assert raw.startswith(b"PF\n5 7\n-1.0\n")
    first_row = np.frombuffer(raw[len(b"PF\n5 7\n-1.0\n"):][:60], "<f4").reshape(5, 3)
    np.testing.assert_array_equal(first_row, px[-1])


def test_photon_file_round_trip(tmp_path):
    ph = W.wall_photons(1000, seed=2)
    save_photons(tmp_path / "m.pmph", ph, 777)
    got, emitted = load_photons(tmp_path / "m.pmph")
    assert emitted == 777
    np.testing.assert_array_equal(got, ph)
    save_photons(tmp_path / "e.pmph", np.zeros((0, 9), np.float32), 0)
    got, emitted = load_photons(tmp_path / "e.pmph")
    assert got.shape == (0, 9) and emitted == 0


def test_photon_file_rejects_bad_input(tmp_path):
    (tmp_path / "x").write_bytes(b"nonsense" * 4)
    with pytest.raises(ValueError):
        load_photons(tmp_path / "x")
    save_photons(tmp_path / "t.pmph", W.wall_photons(10, seed=1), 10)
    data = (tmp_path / "t.pmph").read_bytes()
    (tmp_path / "t.pmph").write_bytes(data[:-4])  # truncated
    with pytest.raises(ValueError):
        load_photons(tmp_path / "t.pmph")

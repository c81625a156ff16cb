"""The drop-in C++ headers: the reference's own programs compile unchanged
against them, and the camera / image programs produce the same files as
the reference's headers do (no GPU needed)."""
from __future__ import annotations

import subprocess
from pathlib import Path

import pytest

from tests.dropin_build import ROOT, compile_dropin, CXX, reference_dir

REF = reference_dir()
needs_ref = pytest.mark.skipif(not (REF / "include" / "camera.h").exists(),
                               reason="reference tree not present")


def test_driver_compiles(tmp_path):
    compile_dropin(ROOT / "tests" / "cpp" / "dropin_render.cpp", tmp_path / "dropin_render")


@needs_ref
@pytest.mark.parametrize("src", ["examples/main.cpp", "tests/test_camera.cpp", "tests/test_image.cpp",
                                 "tests/test_intersector.cpp", "tests/test_path_tracing.cpp",
                                 "tests/visualize_photon_map.cpp"])
def test_reference_sources_compile_unchanged(tmp_path, src):
    compile_dropin(REF / src, tmp_path / "prog")


@needs_ref
@pytest.mark.parametrize("prog", ["test_camera", "test_image"])
def test_camera_and_image_match_reference(tmp_path, prog):
    src = REF / "tests" / f"{prog}.cpp"
    dropin = tmp_path / "dropin"
    dropin.mkdir()
    compile_dropin(src, dropin / prog)
    subprocess.run([str(dropin / prog)], cwd=dropin, check=True)
    ref = tmp_path / "ref"
    ref.mkdir()
    # the reference's headers rely on transitive includes for <cstdint> and
    # <algorithm>; force them in without touching its sources
    cmd = [CXX, "-std=c++20", "-O2", "-include", "cstdint", "-include", "algorithm",
           "-I", str(ROOT / "oracle" / "shim"), "-I", str(REF / "include"), str(src),
           "-o", str(ref / prog)]
    subprocess.run(cmd, check=True, capture_output=True)
    subprocess.run([str(ref / prog)], cwd=ref, check=True)
    assert (dropin / "output.ppm").read_bytes() == (ref / "output.ppm").read_bytes()

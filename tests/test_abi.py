"""The C ABI library loads and exports every entry point include/pm_cuda.h
declares (no GPU needed; no compute call is made)."""
from __future__ import annotations

import ctypes
import re
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
HEADER = ROOT / "include" / "pm_cuda.h"
LIB = ROOT / "photon_mapping_b200" / "_lib" / "libpm_cuda.so"


def declared_functions() -> set[str]:
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return set(re.findall(r"\b(pm_[a-z0-9_]+)\s*\(", text))


@pytest.fixture(scope="module")
def lib_path():
    if not LIB.exists():
        from photon_mapping_b200.build import build_cuda
        build_cuda()
    return LIB


def test_header_declares_entry_points():
    names = declared_functions()
    assert {"pm_ctx_create", "pm_photonmap_build", "pm_photonmap_knn",
            "pm_photonmap_radiance"} <= names


def test_library_exports_every_declared_symbol(lib_path):
    out = subprocess.run(["nm", "-D", "--defined-only", str(lib_path)],
                         capture_output=True, text=True, check=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if " T " in line}
    missing = declared_functions() - exported
    assert not missing, f"declared but not exported: {sorted(missing)}"


def test_library_loads_and_symbols_resolve(lib_path):
    lib = ctypes.CDLL(str(lib_path))
    for name in declared_functions():
        assert getattr(lib, name) is not None


def test_status_strings_and_null_context(lib_path):
    lib = ctypes.CDLL(str(lib_path))
    lib.pm_status_string.restype = ctypes.c_char_p
    assert lib.pm_status_string(0) == b"PM_OK"
    assert lib.pm_status_string(4) == b"PM_ERR_NOT_BUILT"
    # null context: an argument error, never a crash
    assert lib.pm_ctx_synchronize(None) == 1
    assert lib.pm_photonmap_build(None, 0, None, ctypes.c_int64(0)) == 1
    # null batch: the same
    assert lib.pm_batch_render(None, 0, None) == 1
    assert lib.pm_batch_photons(None, 0, None) == 1
    assert lib.pm_batch_stage_times(None, None, 6) == 1


def test_radiance_query_record_is_48_bytes():
    from photon_mapping_b200 import _native
    assert _native.RADIANCE_QUERY_FLOATS * 4 == 48


def test_struct_layouts_match_the_header(tmp_path):
    """The ctypes mirrors of the statistics records have the C sizes and
    field offsets of include/pm_cuda.h."""
    import ctypes as C
    from photon_mapping_b200 import _native as N
    from photon_mapping_b200.integrator import RenderStats, TraceStats
    src = tmp_path / "sizes.c"
    src.write_text('#include <stddef.h>\n#include <stdio.h>\n#include "pm_cuda.h"\n'
                   'int main(void) {\n'
                   '  printf("%zu %zu %zu %zu %zu\\n", sizeof(pm_trace_stats),\n'
                   '         offsetof(pm_trace_stats, rays), sizeof(pm_render_stats),\n'
                   '         offsetof(pm_render_stats, rays), sizeof(pm_knn_stats));\n'
                   '  return 0;\n}\n')
    exe = tmp_path / "sizes"
    subprocess.run(["gcc", "-I", str(ROOT / "include"), str(src), "-o", str(exe)], check=True)
    got = [int(x) for x in subprocess.run([str(exe)], capture_output=True, text=True,
                                          check=True).stdout.split()]
    assert got == [C.sizeof(TraceStats), TraceStats.rays.offset, C.sizeof(RenderStats),
                   RenderStats.rays.offset, 8 * len(N.Context.STAT_FIELDS)]

"""Compiles C++ programs against the drop-in headers and libpm_cuda.so."""
from __future__ import annotations

import os
import subprocess
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]
DROPIN = ROOT / "photon_mapping_b200" / "cpp" / "include"
LIBDIR = ROOT / "photon_mapping_b200" / "_lib"
CXX = "/usr/bin/g++" if Path("/usr/bin/g++").exists() else "g++"


def reference_dir() -> Path:
    """The reference tree: PM_REFERENCE_DIR when set, else the directory
    `reference` beside the repository root (as in oracle/Makefile)."""
    env = os.environ.get("PM_REFERENCE_DIR")
    return Path(env) if env else ROOT.parent / "reference"


def compile_dropin(src: Path, out: Path, include=DROPIN) -> None:
    if not (LIBDIR / "libpm_cuda.so").exists():
        from photon_mapping_b200.build import build_cuda
        build_cuda()
    cmd = [CXX, "-std=c++20", "-O2", "-fopenmp", "-I", str(include), "-I", str(ROOT / "include"),
           str(src), "-L", str(LIBDIR), "-lpm_cuda", f"-Wl,-rpath,{LIBDIR}", "-o", str(out)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, f"compile failed: {' '.join(cmd)}\n{r.stderr}"

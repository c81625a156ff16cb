"""Build recipe of the native parts of photon_mapping_b200.

* ``libpm_cuda.so``: every ``csrc/*.cu`` compiled by nvcc for sm_100a and
  linked into one shared library with the C ABI of ``include/pm_cuda.h``.
  Device code is compiled with ``-fmad=false`` so that every float
  operation rounds on its own, as the reference's x86-64 build does.

The outputs stay in the source tree (``photon_mapping_b200/_lib``) so that
they travel with a snapshot of the repository.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
LIBDIR = PKG / "_lib"
OBJDIR = PKG / "_lib" / "obj"
LIB = LIBDIR / "libpm_cuda.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + [
    "-lineinfo", "-O3", "-std=c++17", "-fmad=false",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
    "-I", str(ROOT / "include"),
]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def _sources() -> list[Path]:
    return sorted(CSRC.glob("*.cu"))


def _headers() -> list[Path]:
    return sorted(CSRC.glob("*.cuh")) + sorted((ROOT / "include").glob("*.h"))


def _stale(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def _compile(src: Path, verbose: bool) -> Path:
    obj = OBJDIR / (src.stem + ".o")
    if _stale(obj, [src] + _headers()):
        cmd = [nvcc(), *NVCC_FLAGS, "-c", str(src), "-o", str(obj)]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed on {src.name}:\n{r.stdout}\n{r.stderr}")
    return obj


def build_cuda(force: bool = False, verbose: bool = False) -> Path:
    """Compiles csrc/*.cu for sm_100a and links libpm_cuda.so."""
    OBJDIR.mkdir(parents=True, exist_ok=True)
    if force:
        for o in OBJDIR.glob("*.o"):
            o.unlink()
    srcs = _sources()
    with cf.ThreadPoolExecutor(max_workers=min(8, len(srcs))) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose), srcs))
    if force or _stale(LIB, objs):
        cmd = [nvcc(), *ARCH, "-shared", "-o", str(LIB), *map(str, objs), "-lcudart"]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    return LIB


def build_oracle(verbose: bool = False) -> None:
    """Builds the CPU oracle (test infrastructure, under oracle/)."""
    cmd = ["make", "-s", "-C", str(ROOT / "oracle")]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"oracle build failed:\n{r.stdout}\n{r.stderr}")


if __name__ == "__main__":
    build_cuda(force="--force" in sys.argv, verbose=True)
    if "--oracle" in sys.argv:
        build_oracle(verbose=True)
    print(LIB)

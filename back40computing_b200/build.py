"""Builds libb40c_bfs.so in-tree with nvcc for sm_100a.

The library holds every CUDA kernel and the C ABI declared in include/b40c_bfs.h.
Run as ``python -m back40computing_b200.build`` or call :func:`build`.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
INCLUDE = ROOT / "include"
LIB = PKG / "libb40c_bfs.so"

ARCH_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a"]
SOURCES = ["bfs_kernels.cu", "bfs_host.cu", "ms_kernels.cu", "ms_host.cu", "server_host.cu", "no_alloc.cu",
           "graph_gen.cpp", "graph_io.cpp"]
DRIVER = PKG / "test_bfs"


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found: the BFS library needs the CUDA toolkit to build")


def _stale(out: Path, deps) -> bool:
    if not out.exists():
        return True
    t = out.stat().st_mtime
    return any(Path(d).stat().st_mtime > t for d in deps)


def build(force: bool = False, verbose: bool = False, extra_flags=None) -> Path:
    """Compiles the library if any source is newer than the .so; returns its path."""
    deps = [CSRC / s for s in SOURCES] + list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.h")) + [
        INCLUDE / "b40c_bfs.h"]
    if not force and not _stale(LIB, deps):
        if _stale(DRIVER, [LIB, CSRC / "test_bfs_main.cpp"] + list((INCLUDE / "b40c").rglob("*.hpp"))):
            build_driver(verbose=verbose)
        return LIB
    tmp = LIB.with_suffix(".so.tmp")
    cmd = [_nvcc(), *ARCH_FLAGS, "-lineinfo", "-O3", "-std=c++17", "--shared",
           "-Xcompiler", "-fPIC,-O3,-fvisibility=default", "-Xptxas", "-O3",
           f"-I{INCLUDE}", f"-I{CSRC}", "-o", str(tmp), *[str(CSRC / s) for s in SOURCES],
           "-lpthread", *(extra_flags or [])]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True, cwd=str(ROOT))
    os.replace(tmp, LIB)
    build_driver(verbose=verbose)
    return LIB


def build_driver(verbose: bool = False) -> Path:
    """The test_bfs command-line driver: plain C++ over the C ABI (no nvcc)."""
    src = CSRC / "test_bfs_main.cpp"
    cuda_inc = Path(_nvcc()).resolve().parent.parent / "include"
    cmd = [os.environ.get("CXX", "g++"), "-O2", "-std=c++17", f"-I{INCLUDE}", f"-I{cuda_inc}", "-o", str(DRIVER),
           str(src), f"-L{PKG}", "-lb40c_bfs", "-Wl,-rpath,$ORIGIN"]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True, cwd=str(ROOT))
    return DRIVER


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True,
          extra_flags=["-Xptxas", "-v"] if "--ptxas-v" in sys.argv else None)
    print(LIB)

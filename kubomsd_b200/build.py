"""Build libkmsd_b200.so (the engine's C ABI) in-tree with nvcc for sm_100a.

The library is written to ``kubomsd_b200/_lib/libkmsd_b200.so`` next to the
package so that it travels with the source tree; ``python -m
kubomsd_b200.build`` rebuilds it when a source is newer than the library.
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
INCLUDE = ROOT / "include"
LIBDIR = PKG / "_lib"
LIBNAME = "libkmsd_b200.so"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
              "-Xcompiler", "-Wall", "-Xcompiler", "-Wno-unused-function"]
SOURCES = ["kmsd_engine.cu", "kmsd_metric.cu", "kmsd_ops.cu", "kmsd_noalloc.cu", "kmsd_batch.cu", "kmsd_corr.cu", "kmsd_stats.cu"]


def nvcc() -> str:
    path = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(path).exists():
        raise RuntimeError("nvcc not found; the CUDA toolkit is required to build libkmsd_b200.so")
    return path


def library_path() -> Path:
    return LIBDIR / LIBNAME


def _stale(target: Path, deps) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def build(force: bool = False, verbose: bool = False, jobs: int | None = None) -> Path:
    """Compile every .cu source to an object and link the shared library."""
    LIBDIR.mkdir(exist_ok=True)
    objdir = LIBDIR / "obj"
    objdir.mkdir(exist_ok=True)
    headers = list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.h")) + list(INCLUDE.glob("*.h"))
    compiler = nvcc()

    def compile_one(src: str) -> Path:
        s = CSRC / src
        o = objdir / (Path(src).stem + ".o")
        if force or _stale(o, [s, *headers]):
            cmd = [compiler, *ARCH, *NVCC_FLAGS, "-I", str(INCLUDE), "-I", str(CSRC), "-c", str(s), "-o", str(o)]
            if verbose:
                cmd.insert(1, "-Xptxas=-v")
            run = subprocess.run(cmd, capture_output=True, text=True)
            if run.returncode != 0:
                raise RuntimeError(f"nvcc failed for {src}:\n{run.stdout}\n{run.stderr}")
            if verbose:
                sys.stderr.write(run.stderr)
        return o

    with cf.ThreadPoolExecutor(max_workers=jobs or len(SOURCES)) as pool:
        objects = list(pool.map(compile_one, SOURCES))
    lib = library_path()
    if force or _stale(lib, objects):
        cmd = [compiler, *ARCH, "-shared", "-o", str(lib), *map(str, objects), "-lcudart"]
        run = subprocess.run(cmd, capture_output=True, text=True)
        if run.returncode != 0:
            raise RuntimeError(f"link failed:\n{run.stdout}\n{run.stderr}")
    return lib


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))

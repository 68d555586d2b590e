"""Builds libsppgpu.so (the CUDA library behind the C ABI in include/sppgpu.h).

nvcc cross-compiles for sm_100a only; the shared object is written in-tree
next to this file so it travels with the package.  The build is skipped when
the library is newer than every source.
"""

from __future__ import annotations

import os
import shutil
import subprocess
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
INCLUDE = PKG.parent / "include"
LIB = PKG / "libsppgpu.so"

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC", "-shared",
    "--expt-relaxed-constexpr",
]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found; set NVCC or install the CUDA toolkit")


def sources() -> list[Path]:
    return sorted(CSRC.glob("*.cu"))


def _stale() -> bool:
    if not LIB.exists():
        return True
    t = LIB.stat().st_mtime
    deps = list(CSRC.glob("*.cu")) + list(CSRC.glob("*.cuh")) + list(INCLUDE.glob("*.h"))
    return any(p.stat().st_mtime > t for p in deps)


def build(force: bool = False, verbose: bool = False, extra: list[str] | None = None) -> Path:
    """Compile each .cu to an object in parallel (no device code crosses files),
    then link the shared library."""
    if not force and not _stale():
        return LIB
    from concurrent.futures import ThreadPoolExecutor

    objdir = PKG / "_build"
    objdir.mkdir(exist_ok=True)
    compile_flags = [f for f in NVCC_FLAGS if f != "-shared"]
    jobs = []
    for src in sources():
        obj = objdir / (src.stem + ".o")
        jobs.append((obj, [_nvcc(), *compile_flags, *(extra or []), "-c", "-o", str(obj), str(src)]))

    def run(job):
        if verbose:
            print(" ".join(job[1]))
        subprocess.run(job[1], check=True)
        return job[0]

    with ThreadPoolExecutor(max_workers=min(len(jobs), os.cpu_count() or 1)) as ex:
        objs = list(ex.map(run, jobs))
    tmp = LIB.with_suffix(".so.tmp")
    subprocess.run([_nvcc(), "-gencode", "arch=compute_100a,code=sm_100a", "-shared",
                    "-o", str(tmp), *map(str, objs)], check=True)
    tmp.replace(LIB)
    return LIB


if __name__ == "__main__":
    import sys

    build(force="--force" in sys.argv, verbose=True,
          extra=["-Xptxas", "-v"] if "--ptxas" in sys.argv else None)

"""Build libporerad.so (the sm_100a CUDA library behind porerad_b200) in-tree.

    python -m porerad_b200.build [-v] [--force]

Each csrc/*.cu compiles to an object with nvcc for sm_100a only; the traversal
file additionally gets -fmad=false (its arithmetic is written with explicit
round-to-nearest intrinsics as well).  Objects go to porerad_b200/_build/, the
library to porerad_b200/libporerad.so.
"""

from __future__ import annotations

import concurrent.futures
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
OUT = PKG / "libporerad.so"
BUILD = PKG / "_build"
INCLUDE = PKG.parent / "include"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
         "--expt-relaxed-constexpr", "-I", str(INCLUDE)]
SOURCES = ["patches.cu", "trace.cu", "operator.cu", "radiosity.cu", "capi.cu", "timers.cu", "arena.cu", "coupled.cu", "multibounce.cu", "descriptors.cu", "generate.cu", "archetypes.cu", "hostcopy.cu"]
STRICT_FP = {"trace.cu", "patches.cu", "multibounce.cu", "generate.cu", "archetypes.cu"}


def nvcc() -> str:
    path = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(path).exists():
        raise RuntimeError("nvcc not found: the CUDA toolkit is required to build libporerad")
    return path


def _deps() -> list[Path]:
    return sorted(CSRC.glob("*.cuh")) + [INCLUDE / "porerad.h"]


def _stale(target: Path, inputs: list[Path]) -> bool:
    if not target.is_file():
        return True
    t = target.stat().st_mtime
    return any(p.stat().st_mtime > t for p in inputs)


def _compile(src: str, verbose: bool, extra: list[str]) -> Path:
    obj = BUILD / (Path(src).stem + ".o")
    inputs = [CSRC / src] + _deps()
    if not _stale(obj, inputs):
        return obj
    cmd = [nvcc(), *ARCH, *FLAGS, *extra, "-c", str(CSRC / src), "-o", str(obj)]
    if src in STRICT_FP:
        cmd.insert(-4, "-fmad=false")
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    return obj


def build(verbose: bool = False, force: bool = False, extra: list[str] | None = None) -> Path:
    """Compile every CUDA source for sm_100a and link libporerad.so; returns its path."""

    BUILD.mkdir(exist_ok=True)
    if force:
        for o in BUILD.glob("*.o"):
            o.unlink()
    extra = list(extra or [])
    workers = min(len(SOURCES), os.cpu_count() or 1)
    with concurrent.futures.ThreadPoolExecutor(workers) as pool:
        objs = list(pool.map(lambda s: _compile(s, verbose, extra), SOURCES))
    if force or _stale(OUT, objs):
        cmd = [nvcc(), *ARCH, "-shared", "-Xcompiler", "-fPIC", *[str(o) for o in objs], "-o", str(OUT),
               "-lcudart"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return OUT


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, force="--force" in sys.argv))

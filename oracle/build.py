"""Build recipe for the oracle's C kernels (test infrastructure only).

    python oracle/build.py

Compiles oracle/dda.c into oracle/liboracle_dda.so and oracle/multibounce.c into
oracle/liboracle_mb.so with gcc, OpenMP and -ffp-contract=off (every binary64 operation rounds
once, no FMA contraction).
"""

from __future__ import annotations

import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent


def _compile(name: str, verbose: bool) -> Path:
    src = HERE / f"{name}.c"
    out = HERE / f"liboracle_{'dda' if name == 'dda' else 'mb'}.so"
    if out.is_file() and out.stat().st_mtime >= src.stat().st_mtime:
        return out
    cmd = ["gcc", "-O2", "-ffp-contract=off", "-fno-fast-math", "-fopenmp", "-fPIC", "-shared",
           str(src), "-o", str(out), "-lm"]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    return out


def build(verbose: bool = False) -> Path:
    """Both libraries; returns the traversal's."""

    _compile("multibounce", verbose)
    return _compile("dda", verbose)


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))

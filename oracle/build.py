"""Build recipe for the oracle's C traversal (test infrastructure only).

    python oracle/build.py

Compiles oracle/dda.c into oracle/liboracle_dda.so with gcc, OpenMP and
-ffp-contract=off (every binary64 operation rounds once, no FMA contraction).
"""

from __future__ import annotations

import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent


def build(verbose: bool = False) -> Path:
    src = HERE / "dda.c"
    out = HERE / "liboracle_dda.so"
    if out.is_file() and out.stat().st_mtime >= src.stat().st_mtime:
        return out
    cmd = ["gcc", "-O2", "-ffp-contract=off", "-fno-fast-math", "-fopenmp", "-fPIC", "-shared",
           str(src), "-o", str(out), "-lm"]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    return out


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))

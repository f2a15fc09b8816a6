"""Time the reference's own Numba first-hit counts beside the oracle port on the same sample.

    python oracle/compare_reference_counts.py --reference <checkout of porerad> [--width 256]

(or set PORERAD_REFERENCE to the checkout.)  Test infrastructure: it runs where the reference
package and Numba are importable, never on the GPU path.  The workload is the c2 count stage
(OF N=128^3, phi 0.10, geometry seed 1, 1000 rays per patch, sets A and B); the sample is the
one the bench's CPU arm uses, 16 blocks of ``width`` consecutive origin patches spread evenly
over the patches, traced for both sets.  Each block is one chunk of the reference's
``first_hit_counts`` (porerad/view_factors.py:273-287): ``generate_rays`` + ``trace_first_hit``
(the Numba kernel, all cores) + ``np.unique`` of the edge keys; the port runs
``oracle.porerad_oracle.first_hit_counts`` on the same patch ranges with the same threads.
Prints one JSON line: rays/s of each, the thread counts, and whether one block's counts agree.
"""

from __future__ import annotations

import argparse
import json
import os
import sys
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]


def main() -> None:
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--reference", default=os.environ.get("PORERAD_REFERENCE"),
                    help="checkout of the reference (the directory holding the porerad package)")
    ap.add_argument("--width", type=int, default=256, help="consecutive origin patches per block")
    args = ap.parse_args()
    if not args.reference:
        ap.error("--reference (or PORERAD_REFERENCE) is required")
    sys.path.insert(0, str(Path(args.reference).resolve()))
    sys.path.insert(0, str(ROOT))

    import numba
    import numpy as np
    from porerad import view_factors as rvf

    import bench
    from oracle import build as ob
    from oracle import porerad_oracle as orc

    ob.build()
    threads = orc.set_threads()
    cfg = bench.WORKLOADS["c2"]
    seeds = bench.ray_seeds(cfg)
    phases = bench.make_phases(cfg)
    rp = rvf.build_surface_patches(phases, cfg["H"])
    op = orc.build_surface_patches(phases, cfg["H"])
    P, R, blocks, width = rp.n_patches, cfg["rays"], 16, args.width
    starts = [int(b * P // blocks) for b in range(blocks)]

    def reference_block(seed, p0, p1):
        origins, directions = rvf.generate_rays(rp, p0, p1, R, seed)
        receiver = rvf.trace_first_hit(rp, origins, directions)
        origin = np.repeat(np.arange(p0, p1, dtype=np.int64), R)
        return np.unique(origin * P + receiver.astype(np.int64), return_counts=True)

    def port_block(seed, p0, p1):
        return orc.first_hit_counts(op, R, seed, patch_start=p0, patch_end=p1)

    reference_block(seeds[0], 0, 8)  # Numba compiles outside the timing
    out = {"workload": "c2 count stage sample", "blocks": blocks, "width": width, "threads": threads,
           "numba_threads": numba.get_num_threads()}
    for name, fn in (("reference_numba", reference_block), ("oracle_port", port_block)):
        t0 = time.perf_counter()
        for seed in seeds:
            for p0 in starts:
                fn(seed, p0, p0 + width)
        dt = time.perf_counter() - t0
        out[name] = {"rays_per_s": len(seeds) * blocks * width * R / dt, "s": dt}
    pair, count = reference_block(seeds[0], starts[3], starts[3] + width)
    o, r, c = port_block(seeds[0], starts[3], starts[3] + width)
    out["same_counts"] = bool(np.array_equal(pair, o.astype(np.int64) * P + r) and np.array_equal(count, c))
    print(json.dumps(out))


if __name__ == "__main__":
    main()

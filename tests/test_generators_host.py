"""Host side of porerad_b200.generators on the CPU: the fiber parameters, lattice nodes and disk
offsets it hands to the device reproduce every archived FI/FA array of data/microstructures.csv
when stamped with NumPy (the device kernel's integer work), and the acceptance rules decide as
the reference's on the stored descriptor records."""

from __future__ import annotations

import hashlib
import json

import numpy as np
import pytest

from porerad_b200 import generators as gen
from tests.helpers import GOLDEN, descriptor_records

ROWS = [r for r in json.loads((GOLDEN / "microstructures.json").read_text())["rows"] if r["structure"] in ("FI", "FA")]


def _stamp(N, fibers, r):
    ph = np.zeros(N ** 3, np.uint8)
    for f in fibers:
        idx = (f.nodes[:, None, :] + f.disk(r)[None, :, :]) % N
        ph[((idx[..., 0] * N + idx[..., 1]) * N + idx[..., 2]).ravel()] = 1
    return ph.reshape(N, N, N)


def _bisect(render, target, lo, hi, tol, max_iter):
    best = None
    for _ in range(max_iter):
        mid = 0.5 * (lo + hi)
        ph = render(mid)
        phi = float(np.count_nonzero(ph == 1) / ph.size)
        err = abs(phi - target)
        if best is None or err < best[0]:
            best = (err, ph)
        if err <= tol:
            break
        lo, hi = (mid, hi) if phi < target else (lo, mid)
    return best[1]


@pytest.mark.parametrize("row", ROWS, ids=[r["id"] for r in ROWS])
def test_fiber_nodes_and_disks(row):
    N = row["N"]
    if row["set"] == "matched":
        seed, n_lines = gen.MATCHED_PAIRS[int(row["id"][-1])][row["structure"]]
        aligned = row["structure"] == "FA"
        centers = [tuple(float(v) for v in c)
                   for c in (np.random.default_rng(seed + 1000003).random((64, 3)) * N)[:n_lines]]
        rng = np.random.default_rng(seed + (3000003 if aligned else 2000003))
        rots = []
        for _ in range(n_lines):
            v = gen._fiber_axis(rng, aligned)
            rots.append(gen._frame(v / np.linalg.norm(v), gen._EZ))
        fibers = [gen._long_fiber(N, c, 0.5 * 9.0 * N, R) for c, R in zip(centers, rots)]
        ph = _bisect(lambda r: _stamp(N, fibers, r), 0.1, 0.12, 7.0, 5e-4, 32)
    else:
        phi = round(row["target_phi"], 2)
        centers, rots = gen.fiber_lines(N, row["seed"], gen.FIBER_LINES[row["structure"]][phi],
                                        row["structure"] == "FA", row["set"] == "canonical")
        half = 0.5 * gen.FIBER_LENGTH[row["structure"]] * N
        fibers = [gen._long_fiber(N, c, half, R) for c, R in zip(centers, rots)]
        ph = _bisect(lambda r: _stamp(N, fibers, r), row["target_phi"], 0.1, 4.0, gen.PHI_TOL, 24)
    assert hashlib.sha256(ph.tobytes()).hexdigest() == row["phase_sha256"]


def test_acceptance_rules_on_stored_descriptors():
    recs = descriptor_records()["stored"]
    for name, rec in recs.items():
        a = rec["archived"]
        if a["set"] != "core":
            continue
        d = dict(rec["scalar"])
        assert gen.accepted(a["structure"], d, a["target_phi"]), name  # every stored core array was accepted
    d = dict(recs["OF_core_phi0.10_s2"]["scalar"])
    assert not gen.accepted("OF", {**d, "pore_percolates": [True, False, True]}, 0.10)
    assert not gen.accepted("OF", d, 0.10 + 2 * gen.PHI_TOL)
    with pytest.raises(ValueError):
        gen.accepted("XX", d, 0.10)

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
        draws = gen.draw_matched_fibers(N, int(row["id"][-1]), row["structure"])
        half, target, lo, hi, tol, its = 0.5 * 9.0 * N, 0.1, 0.12, 7.0, 5e-4, 32
    else:
        phi = round(row["target_phi"], 2)
        draws = gen.draw_library_fibers(N, row["seed"], gen.FIBER_LINES[row["structure"]][phi],
                                        row["structure"] == "FA", row["set"] == "canonical")
        half = 0.5 * gen.FIBER_LENGTH[row["structure"]] * N
        target, lo, hi, tol, its = row["target_phi"], 0.1, 4.0, gen.PHI_TOL, 24
    fibers = [gen.LatticeCylinder(N, c, half, f) for c, f in zip(draws.centres, draws.frames)]
    ph = _bisect(lambda r: _stamp(N, fibers, r), target, lo, hi, tol, its)
    assert hashlib.sha256(ph.tobytes()).hexdigest() == row["phase_sha256"]


def test_public_fiber_lines_and_foam_graph_forms():
    """fiber_lines and foam_graph return the reference's forms (tuples of floats, 3 x 3 frames,
    sorted (i, j) edges with i < j) built from the recorded draws."""

    centres, frames = gen.fiber_lines(64, 3, 5, False)
    d = gen.draw_library_fibers(64, 3, 5, False, False)
    assert centres == [tuple(float(v) for v in c) for c in d.centres]
    assert all(np.array_equal(a, b) for a, b in zip(frames, d.frames))
    assert all(float(v).is_integer() for c in centres for v in c)
    for f in frames:
        assert np.allclose(f.T @ f, np.eye(3), atol=1e-14)
    nodes, edges = gen.foam_graph(48, 2, 20)
    assert nodes.shape == (20, 3) and edges == sorted(set(edges))
    assert all(i < j for i, j in edges) and len(edges) >= 20 * gen.FOAM_NEIGHBOURS // 2


def test_foam_edges_and_layer_field_against_oracle():
    """The foam's draws (nodes, the periodic k-nearest-neighbour edges) and TL's host field equal
    the oracle's restatement of the reference's generator, value for value."""

    from scipy.spatial import cKDTree

    from oracle import generators as og

    for N, seed, n in ((128, 0, 32), (128, 5, 24), (160, 0, 32)):
        foam = gen.draw_foam(N, seed, n)
        pts = np.random.default_rng(seed).uniform(0, N, size=(n, 3))
        _, nn = cKDTree(pts, boxsize=N).query(pts, k=4)
        want = sorted({tuple(sorted((int(i), int(j)))) for i, row in enumerate(nn) for j in row[1:] if i != j})
        assert np.array_equal(foam.nodes, pts) and [tuple(e) for e in foam.edges.tolist()] == want
    for N, seed, layers, wav in ((48, 0, 7, 1.7), (40, 3, 9, 1.55)):
        assert np.array_equal(gen.lamellar_field(N, seed, layers, wav), og.layered_field(N, seed, layers, wav))


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

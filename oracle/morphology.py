"""ORACLE — test infrastructure only.

CPU restatement of the morphology descriptors of porerad (porerad/descriptors.py), the
checker of ``porerad_b200.descriptors`` in ``tests/``.  Counts are NumPy reductions over
shifted copies of the phase masks; runs and chords come from the run boundaries of each
axis-parallel line; 26-connected pore clusters use ``scipy.ndimage.label`` with a full
3x3x3 structuring element, the labelling the reference itself calls.  Pinned by
tests/test_oracle_golden.py against the reference's outputs stored in
tests/golden/descriptors.json and the archived columns of data/microstructures.csv.
"""

from __future__ import annotations

import numpy as np
from scipy.ndimage import label

QUANTILES = (0.5, 0.75, 0.9, 0.95, 0.99)  # descriptors.py:15
LINEAL_SAMPLES = (1, 2, 4, 8, 16, 32, 64, 128)  # descriptors.py:16


def _axis_lines(mask, axis):
    """Rows = the axis-parallel lines of a 3-D mask, in index order of the other two axes."""
    m = np.moveaxis(np.asarray(mask, bool), axis, -1)
    return m.reshape(-1, m.shape[-1])


def _line_runs(rows):
    """(row, start, length) of every run of True cells, rows in order, runs in order along a row."""
    M, N = rows.shape
    edge = np.zeros((M, N + 1), np.int8)
    edge[:, :N] += rows
    edge[:, 1:] -= rows  # +1 where a run starts, -1 one past where it ends
    r0, c0 = np.nonzero(edge == 1)
    _, c1 = np.nonzero(edge == -1)
    return r0, c0, c1 - c0


def interface_area(solid):  # descriptors.py:38-43
    m = np.asarray(solid, bool)
    return int(sum(np.count_nonzero(np.diff(m.astype(np.int8), axis=a)) for a in range(3)))


def mean_pore_chords(pore):  # descriptors.py:46-48
    out = []
    for a in range(3):
        _, _, length = _line_runs(_axis_lines(pore, a))
        out.append(float(np.mean(length)) if len(length) else float("nan"))
    return tuple(out)


def pore_connectivity(pore):  # descriptors.py:51-60
    lbl, n = label(np.asarray(pore, bool), structure=np.ones((3, 3, 3), bool))
    perc = []
    for a in range(3):
        low = set(np.unique(np.take(lbl, 0, axis=a)).tolist()) - {0}
        high = set(np.unique(np.take(lbl, lbl.shape[a] - 1, axis=a)).tolist()) - {0}
        perc.append(bool(low & high))
    sizes = np.bincount(lbl.ravel(), minlength=n + 1)[1:]
    largest = int(sizes.max()) if len(sizes) else 0
    return tuple(perc), float(largest / max(1, int(np.count_nonzero(pore))))


def scalar_descriptors(phases):  # descriptors.py:63-77
    p = np.asarray(phases)
    solid, pore = p == 1, p == 0
    perc, largest = pore_connectivity(pore)
    area = interface_area(solid)
    return {
        "phi_solid": float(np.count_nonzero(solid) / p.size),
        "interfacial_area_density": float(area / p.size),
        "mean_beam_length": float(4.0 * float(np.count_nonzero(pore)) / float(area)),
        "mean_pore_chord": mean_pore_chords(pore),
        "pore_percolates": perc,
        "pore_largest_cluster_fraction": largest,
    }


def periodic_chord_histogram(pore, axis):
    """Chord-length histogram (0..N) of one axis of the periodic cell, all-pore lines, lines, N
    (descriptors.py:82-109: the first and last runs of a line touching both ends are one
    chord; an all-pore line is one chord of length N)."""
    rows = _axis_lines(pore, axis)
    M, N = rows.shape
    full = rows.all(axis=1)
    row, start, length = _line_runs(rows)
    hist = np.zeros(N + 1, np.int64)
    keep = ~full[row]
    wraps = rows[:, 0] & rows[:, -1] & ~full
    first = keep & wraps[row] & (start == 0)
    last = keep & wraps[row] & (start + length == N)
    np.add.at(hist, length[keep & ~first & ~last], 1)
    merged = np.zeros(M, np.int64)
    np.add.at(merged, row[first | last], length[first | last])
    np.add.at(hist, merged[wraps], 1)
    hist[N] += int(full.sum())
    return hist, int(full.sum()), M, N


def lineal_path(counts, n_all_pore, n_lines, N):  # descriptors.py:112-117
    counts = np.asarray(counts, np.int64)
    seg = np.arange(1, N + 1, dtype=np.int64)
    lengths = np.arange(len(counts), dtype=np.int64)
    hits = np.array([int(np.sum(np.maximum(lengths - l + 1, 0) * counts)) for l in seg], np.int64)
    return (hits + n_all_pore * (seg - 1)) / (n_lines * N)


def interface_face_counts(solid):  # descriptors.py:120-123
    s = np.asarray(solid, bool)
    return np.array([np.count_nonzero(s ^ np.roll(s, -1, axis=a)) for a in range(3)], np.int64)


def directional_descriptors(phases):  # descriptors.py:135-180
    pore = np.asarray(phases) == 0
    N = pore.shape[0]
    fc = interface_face_counts(~pore)
    f = fc / fc.sum()
    out = []
    for axis in range(3):
        hist, allp, nlines, n = periodic_chord_histogram(pore, axis)
        counts = np.zeros(N + 1, np.int64)
        m = min(N + 1, len(hist))
        counts[:m] = hist[:m]
        lp = lineal_path(counts, allp, nlines, n)
        vals = np.repeat(np.arange(len(hist), dtype=np.float64), hist)
        q = np.quantile(vals, list(QUANTILES))
        below = lp <= np.exp(-1)
        row = {
            "interface_face_count_axis": int(fc[axis]),
            "interface_face_count_total": int(fc.sum()),
            "interface_normal_fraction_axis": float(f[axis]),
            "interface_normal_anisotropy": float(f.max() / f.min()),
            "all_pore_line_count": allp,
            "total_axis_lines": nlines,
            "all_pore_line_fraction": float(allp / nlines),
            "lineal_integral_cells": float(lp.sum()),
            "lineal_1e_length_cells": float(np.where(below)[0][0] + 1) if np.any(below) else float(N),
            "pore_chord_cells_count": int(len(vals)),
            "pore_chord_cells_mean": float(vals.mean()),
            "pore_chord_cells_std": float(vals.std()),
            "pore_chord_cells_max": float(vals.max()),
            "pore_chord_cells_cv": float(vals.std() / vals.mean()),
        }
        for qq, v in zip(QUANTILES, q):
            row[f"pore_chord_cells_q{int(round(100 * qq))}"] = float(v)
        row["pore_chord_cells_q95_over_mean"] = float(q[3] / vals.mean())
        row["pore_chord_cells_q99_over_mean"] = float(q[4] / vals.mean())
        for l in LINEAL_SAMPLES:
            row[f"lineal_path_L{l:03d}"] = float(lp[l - 1])
        row["lineal_path"] = lp
        row["chord_counts"] = counts
        out.append(row)
    return out

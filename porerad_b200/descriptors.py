"""Morphology descriptors of a two-phase digital microstructure, on a B200.

Mirrors ``porerad.descriptors`` (porerad/descriptors.py).  Phase arrays hold 1 for solid and
0 for pore; lengths are in cells.  The scalar descriptors (phi_s, A_s, L_m, mean axial pore
chords, pore percolation and the largest 26-connected pore cluster) treat the box faces as
ends of the sample; the directional descriptors (periodic chord-length distribution,
lineal-path function L_a(l), interface-normal fractions f_a) use the periodic cell.

Every count behind them (cells, interface faces, pore runs, periodic chord histograms,
all-pore lines, pore clusters) comes from one call of libporerad (``pr_morphology_counts``);
what remains here is arithmetic on those integers and on histograms of N + 1 entries, in
the reference's own formulas.  ``periodic_chords`` returns the chord lengths in ascending
order (the reference lists them line by line): every statistic taken of them is the same.
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass
from fractions import Fraction

import numpy as np

from . import _lib

QUANTILES = (0.5, 0.75, 0.9, 0.95, 0.99)
LINEAL_SAMPLES = (1, 2, 4, 8, 16, 32, 64, 128)

CHORDS = 1
CONNECTIVITY = 2


@dataclass
class MorphologyCounts:
    """The integer counts of one phase array (``pr_morphology``); -1 where not asked for."""

    shape: tuple
    cells: int
    solid_cells: int
    pore_cells: int
    interface_faces: tuple      # solid/non-solid faces inside the box, normals x, y, z
    periodic_faces: tuple       # pore/non-pore faces of the periodic cell, normals x, y, z
    pore_runs: tuple            # pore runs along x, y, z ending at the box faces
    all_pore_lines: tuple       # periodic-cell lines entirely in the pore, along x, y, z
    pore_clusters: int
    largest_pore_cluster: int
    pore_percolates: tuple
    chord_counts: tuple | None  # per axis: chords of each length 0..n_a of the periodic cell


def _phase_buffer(phases):
    """(pointer, shape, keep-alive) of a C-ordered uint8 3-D phase array, host or CUDA."""

    try:
        import torch
    except ImportError:  # pragma: no cover - torch is part of the runtime image
        torch = None
    if torch is not None and isinstance(phases, torch.Tensor):
        t = phases
        if t.dim() != 3:
            raise ValueError("phase array must be 3-D")
        if t.dtype == torch.bool:
            t = t.to(torch.uint8)
        if t.dtype != torch.uint8:
            raise ValueError("phase tensor must hold uint8 or bool")
        t = t.contiguous()
        return t.data_ptr(), tuple(int(s) for s in t.shape), t
    a = np.asarray(phases)
    if a.ndim != 3:
        raise ValueError("phase array must be 3-D")
    if a.dtype == bool:
        a = a.astype(np.uint8)
    elif a.dtype != np.uint8:
        if not np.issubdtype(a.dtype, np.integer):
            raise ValueError("phase array must hold integers")
        # values other than 0 and 1 are neither phase, as in the reference's masks
        a = np.where(a == 1, 1, np.where(a == 0, 0, 2)).astype(np.uint8)
    a = np.ascontiguousarray(a)
    return a.ctypes.data, tuple(int(s) for s in a.shape), a


def morphology_counts(phases, *, chords: bool = True, connectivity: bool = True) -> MorphologyCounts:
    """Every count behind the descriptors of ``phases`` from one device pass."""

    ptr, shape, keep = _phase_buffer(phases)
    if min(shape) <= 0:
        raise ValueError("phase array must not be empty")
    m = _lib.Morphology()
    what = (CHORDS if chords else 0) | (CONNECTIVITY if connectivity else 0)
    hists = [np.zeros(n + 1, np.int64) for n in shape] if chords else [None, None, None]
    ptrs = [h.ctypes.data if h is not None else None for h in hists]
    _lib.check(_lib.load().pr_morphology_counts(ptr, shape[0], shape[1], shape[2], what, ctypes.byref(m), *ptrs,
                                                _lib.stream()))
    del keep
    return MorphologyCounts(
        shape=shape, cells=int(m.cells), solid_cells=int(m.solid_cells), pore_cells=int(m.pore_cells),
        interface_faces=tuple(int(v) for v in m.interface_faces),
        periodic_faces=tuple(int(v) for v in m.periodic_faces), pore_runs=tuple(int(v) for v in m.pore_runs),
        all_pore_lines=tuple(int(v) for v in m.all_pore_lines), pore_clusters=int(m.pore_clusters),
        largest_pore_cluster=int(m.largest_pore_cluster),
        pore_percolates=tuple(int(v) for v in m.pore_percolates),
        chord_counts=tuple(hists) if chords else None)


def _mask_phases(mask, solid: bool):
    """Phase array whose solid (or pore) cells are the True cells of a boolean mask."""

    m = np.asarray(mask, bool)
    return (m if solid else ~m).astype(np.uint8)


# Scalar descriptors

def interface_area(solid) -> int:
    """Number of cell faces between solid and pore inside the box, A_int (descriptors.py:38-43)."""

    return int(sum(morphology_counts(_mask_phases(solid, True), chords=False,
                                     connectivity=False).interface_faces))


def _mean_chords(c: MorphologyCounts) -> tuple:
    with np.errstate(invalid="ignore", divide="ignore"):
        return tuple(float(np.float64(c.pore_cells) / np.float64(r)) if r else float("nan") for r in c.pore_runs)


def mean_pore_chords(pore) -> tuple:
    """Mean length of the pore runs along x, y and z, runs ending at the box faces (descriptors.py:46-48)."""

    return _mean_chords(morphology_counts(_mask_phases(pore, False), chords=False, connectivity=False))


def _connectivity(c: MorphologyCounts) -> tuple:
    perc = tuple(bool(p) for p in c.pore_percolates)
    return perc, float(max(c.largest_pore_cluster, 0) / max(1, c.pore_cells))


def pore_connectivity(pore) -> tuple:
    """Pore percolation along x, y, z and the largest-cluster fraction, 26-connected (descriptors.py:51-60)."""

    return _connectivity(morphology_counts(_mask_phases(pore, False), chords=False))


def scalar_descriptors(phases) -> dict:
    """phi_s, A_s = A_int/N^3, L_m = 4 V_pore/A_int, mean axial pore chords and pore connectivity
    (descriptors.py:63-77).  Like the reference, a box without interface faces raises
    ZeroDivisionError."""

    return scalar_values(morphology_counts(phases, chords=False))


def scalar_values(c: MorphologyCounts) -> dict:
    """The dict of ``scalar_descriptors`` from the counts of one phase array."""

    area = sum(c.interface_faces)
    perc, largest = _connectivity(c)
    return {
        "phi_solid": float(c.solid_cells / c.cells),
        "interfacial_area_density": float(area / c.cells),
        "mean_beam_length": float(4.0 * float(c.pore_cells) / float(area)),
        "mean_pore_chord": _mean_chords(c),
        "pore_percolates": perc,
        "pore_largest_cluster_fraction": largest,
    }


# Directional descriptors

def periodic_chords(pore, axis: int) -> tuple:
    """Pore chords along one axis of the periodic cell (descriptors.py:82-109): the chord
    lengths (ascending), the number of all-pore lines, the number of lines and N."""

    c = morphology_counts(_mask_phases(pore, False), connectivity=False)
    counts = c.chord_counts[axis]
    N = c.shape[axis]
    return (np.repeat(np.arange(N + 1, dtype=np.int32), counts), int(c.all_pore_lines[axis]),
            int(c.cells // N), int(N))


def lineal_path(counts, n_all_pore, n_lines, N) -> np.ndarray:
    """L_a(l), l = 1..N, from the chord-count histogram of the periodic cell (descriptors.py:112-117)."""

    # hits(l) = sum over chords of length L >= l of (L - l + 1) = T1(l) - (l - 1) T0(l), with the
    # tail sums T0(l) = sum_{L >= l} c_L and T1(l) = sum_{L >= l} L c_L (exact integers)
    counts = np.asarray(counts, np.int64)
    m = len(counts)
    lengths = np.arange(m, dtype=np.int64)
    t0 = np.zeros(m + 1, np.int64)
    t1 = np.zeros(m + 1, np.int64)
    t0[:m] = np.cumsum(counts[::-1])[::-1]
    t1[:m] = np.cumsum((lengths * counts)[::-1])[::-1]
    seg = np.arange(1, N + 1, dtype=np.int64)
    at = np.minimum(seg, m)  # index m holds the empty tail
    hits = t1[at] - (seg - 1) * t0[at]
    return (hits + n_all_pore * (seg - 1)) / (n_lines * N)


def interface_face_counts(solid) -> np.ndarray:
    """Solid-pore faces of the periodic cell with normals along x, y and z (descriptors.py:120-123)."""

    c = morphology_counts(_mask_phases(solid, True), chords=False, connectivity=False)
    return np.array(c.periodic_faces, dtype=np.int64)


def chord_length_distribution(counts):
    """Chord probability, survival probability and pore-length fraction for l = 1..N (descriptors.py:126-132)."""

    counts = np.asarray(counts)
    n = counts.sum()
    total_length = np.sum(np.arange(len(counts)) * counts)
    surv = np.cumsum(counts[::-1])[::-1]
    seg = np.arange(1, len(counts), dtype=np.int64)
    return counts[1:] / n, surv[1:] / n, seg * counts[1:] / total_length


def histogram_quantiles(hist, quantiles=QUANTILES) -> np.ndarray:
    """Quantiles of the sample whose value l occurs hist[l] times, by numpy's default rule.

    numpy's "linear" method (Hyndman and Fan's 7th): virtual index v = (n - 1) q; between
    the sorted values a = x[floor v] and b = x[floor v + 1] with weight g = v - floor v it
    returns a + (b - a) g, or b - (b - a)(1 - g) when g >= 0.5; v >= n - 1 gives the
    largest value.  The sorted values at any position come from the cumulative histogram.
    """

    hist = np.asarray(hist, np.int64)
    n = int(hist.sum())
    if n == 0:
        raise IndexError("quantiles of an empty sample")
    cum = np.cumsum(hist)
    q = np.asarray(quantiles, dtype=np.float64)
    v = float(n - 1) * q
    top = v >= n - 1
    lo = np.where(top, float(n - 1), np.floor(v))
    lo_i = lo.astype(np.int64)
    a = np.searchsorted(cum, lo_i, side="right").astype(np.float64)
    b = np.searchsorted(cum, np.where(top, lo_i, lo_i + 1), side="right").astype(np.float64)
    g = v - lo
    d = b - a
    out = np.where(g >= 0.5, b - d * (1.0 - g), a + d * g)
    return np.where(top, a, out)


def _chord_stats(hist) -> tuple:
    """count, mean, std (population), max of the sample with histogram hist."""

    hist = np.asarray(hist, np.int64)
    n = int(hist.sum())
    if n == 0:
        return 0, float("nan"), float("nan"), float("nan")
    lengths = np.arange(len(hist), dtype=np.int64)
    s1 = int(np.dot(lengths, hist))  # exact: at most 1290 x 2^31
    s2 = int(np.dot(lengths * lengths, hist))
    mean = float(s1) / float(n)
    var = Fraction(n * s2 - s1 * s1, n * n)
    std = float(np.sqrt(float(var)))
    top = int(np.flatnonzero(hist)[-1])
    return n, mean, std, float(top)


def directional_descriptors(phases) -> list:
    """Per-axis directional descriptors for x, y, z (descriptors.py:135-180): three dicts with
    the summary values, the lineal-path function ``lineal_path`` (l = 1..N) and the chord-count
    histogram ``chord_counts`` (index = chord length in cells)."""

    return directional_rows(morphology_counts(phases, connectivity=False))


def directional_rows(c: MorphologyCounts) -> list:
    """The rows of ``directional_descriptors`` from the counts of one phase array."""

    N = c.shape[0]
    fc = np.array(c.periodic_faces, dtype=np.int64)
    with np.errstate(divide="ignore", invalid="ignore"):
        f = fc / fc.sum()
    out = []
    for axis in range(3):
        full = np.asarray(c.chord_counts[axis], np.int64)
        n_axis = c.shape[axis]
        counts = np.zeros(N + 1, np.int64)
        m = min(N + 1, len(full))
        counts[:m] = full[:m]
        allp, nlines = int(c.all_pore_lines[axis]), int(c.cells // n_axis)
        lp = lineal_path(counts, allp, nlines, n_axis)
        n_chords, mean, std, top = _chord_stats(full)
        q = histogram_quantiles(full)
        below = lp <= np.exp(-1)
        with np.errstate(divide="ignore", invalid="ignore"):
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
                "pore_chord_cells_count": int(n_chords),
                "pore_chord_cells_mean": mean,
                "pore_chord_cells_std": std,
                "pore_chord_cells_max": top,
                "pore_chord_cells_cv": float(np.float64(std) / np.float64(mean)),
            }
            for qq, v in zip(QUANTILES, q):
                row[f"pore_chord_cells_q{int(round(100 * qq))}"] = float(v)
            row["pore_chord_cells_q95_over_mean"] = float(np.float64(q[3]) / np.float64(mean))
            row["pore_chord_cells_q99_over_mean"] = float(np.float64(q[4]) / np.float64(mean))
        for l in LINEAL_SAMPLES:
            row[f"lineal_path_L{l:03d}"] = float(lp[l - 1])
        row["lineal_path"] = lp
        row["chord_counts"] = counts
        out.append(row)
    return out


def all_descriptors(phases) -> tuple:
    """``(scalar_descriptors(phases), directional_descriptors(phases))`` from one device pass."""

    c = morphology_counts(phases)
    return scalar_values(c), directional_rows(c)


def all_descriptors_many(arrays) -> list:
    """``all_descriptors`` of many phase arrays, on worker threads with their own streams (the host
    arithmetic of one overlaps the device passes of the others); in order."""

    from .streams import run_concurrently

    return run_concurrently([(all_descriptors, (a,), {}) for a in arrays])

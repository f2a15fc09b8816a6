"""Morphology descriptors on the CPU: the oracle against the reference's stored outputs, and the
host arithmetic of porerad_b200.descriptors (scalar values, directional rows, histogram
quantiles) fed with counts taken on the CPU.  No GPU needed."""

from __future__ import annotations

import math

import numpy as np
import pytest
from scipy.ndimage import label

from tests.helpers import descriptor_phases, descriptor_records
from oracle import morphology as om
from porerad_b200 import descriptors as dm

STD_RTOL = 1.0e-12  # population std and cv: summation order differs (the chords are listed differently)
RECORDS = descriptor_records()
ALL = [(g, n) for g in ("stored", "small") for n in RECORDS[g]]


def _plain(v):
    if isinstance(v, np.ndarray):
        return v.tolist()
    if isinstance(v, tuple):
        return [_plain(x) for x in v]
    return v


def check_directional(rows, golden):
    assert len(rows) == 3
    for row, g in zip(rows, golden):
        assert set(row) == set(g)
        for k, v in row.items():
            v = _plain(v)
            if k in ("pore_chord_cells_std", "pore_chord_cells_cv"):
                assert v == pytest.approx(g[k], rel=STD_RTOL, abs=0.0), k
            else:
                assert v == g[k], k


def check_scalar(values, golden):
    assert {k: _plain(v) for k, v in values.items()} == golden


def cpu_counts(ph: np.ndarray) -> dm.MorphologyCounts:
    """The counts of pr_morphology_counts, taken with NumPy/SciPy on the CPU."""

    solid, pore = ph == 1, ph == 0
    inner = tuple(int(np.count_nonzero(np.diff(solid.astype(np.int8), axis=a))) for a in range(3))
    periodic = tuple(int(np.count_nonzero(pore ^ np.roll(pore, -1, axis=a))) for a in range(3))
    runs = []
    for a in range(3):
        p = np.moveaxis(pore, a, 0)
        prev = np.concatenate([np.zeros((1,) + p.shape[1:], bool), p[:-1]], axis=0)
        runs.append(int(np.count_nonzero(p & ~prev)))
    hists, allp = [], []
    for a in range(3):
        h, n_all, _, _ = om.periodic_chord_histogram(pore, a)
        hists.append(h)
        allp.append(n_all)
    lbl, n = label(pore, structure=np.ones((3, 3, 3), bool))
    sizes = np.bincount(lbl.ravel(), minlength=n + 1)[1:]
    perc = []
    for a in range(3):
        lo = set(np.unique(np.take(lbl, 0, axis=a)).tolist()) - {0}
        hi = set(np.unique(np.take(lbl, lbl.shape[a] - 1, axis=a)).tolist()) - {0}
        perc.append(int(bool(lo & hi)))
    return dm.MorphologyCounts(
        shape=ph.shape, cells=ph.size, solid_cells=int(solid.sum()), pore_cells=int(pore.sum()),
        interface_faces=inner, periodic_faces=periodic, pore_runs=tuple(runs), all_pore_lines=tuple(allp),
        pore_clusters=int(n), largest_pore_cluster=int(sizes.max()) if n else 0, pore_percolates=tuple(perc),
        chord_counts=tuple(hists))


@pytest.mark.parametrize("group,name", ALL)
def test_oracle_descriptors_against_reference(group, name):
    rec = RECORDS[group][name]
    ph = descriptor_phases(name, rec)
    if "scalar" in rec:
        check_scalar(om.scalar_descriptors(ph), rec["scalar"])
    else:
        with pytest.raises(ZeroDivisionError):
            om.scalar_descriptors(ph)
    for a in range(3):
        h, allp, M, N = om.periodic_chord_histogram(ph == 0, a)
        g = rec["chords"][a]
        assert (h.tolist(), allp, M, N) == (g["hist"], g["all_pore"], g["lines"], g["N"])
    assert om.interface_face_counts(ph == 1).tolist() == rec["interface_face_counts"]
    if "directional" in rec:
        check_directional(om.directional_descriptors(ph), rec["directional"])


@pytest.mark.parametrize("name", sorted(RECORDS["stored"]))
def test_oracle_against_archived_microstructure_table(name):
    """data/microstructures.csv: realized phi, A_s, L_m and mean axial pore chords."""

    rec = RECORDS["stored"][name]
    a = rec["archived"]
    d = om.scalar_descriptors(descriptor_phases(name, rec))
    assert d["phi_solid"] == a["realized_phi"]
    assert d["interfacial_area_density"] == a["interfacial_area_density_per_cell"]
    assert d["mean_beam_length"] == a["mean_beam_length_cells"]
    assert list(d["mean_pore_chord"]) == [a["mean_pore_chord_x_cells"], a["mean_pore_chord_y_cells"],
                                          a["mean_pore_chord_z_cells"]]


@pytest.mark.parametrize("group,name", ALL)
def test_host_arithmetic_from_cpu_counts(group, name):
    """scalar_values and directional_rows reproduce the reference from the integer counts alone."""

    rec = RECORDS[group][name]
    c = cpu_counts(descriptor_phases(name, rec))
    if "scalar" in rec:
        check_scalar(dm.scalar_values(c), rec["scalar"])
    else:
        with pytest.raises(ZeroDivisionError):
            dm.scalar_values(c)
    if "directional" in rec:
        check_directional(dm.directional_rows(c), rec["directional"])


def test_histogram_quantiles_match_numpy():
    rng = np.random.default_rng(5)
    for trial in range(400):
        n_bins = int(rng.integers(1, 40))
        hist = rng.integers(0, 4, n_bins)
        if trial % 7 == 0:
            hist[:] = 0
            hist[int(rng.integers(0, n_bins))] = int(rng.integers(1, 3))
        if hist.sum() == 0:
            hist[-1] = 1
        vals = np.repeat(np.arange(n_bins, dtype=np.float64), hist)
        qs = (0.5, 0.75, 0.9, 0.95, 0.99, 0.0, 1.0, 0.3333)
        got = dm.histogram_quantiles(hist, qs)
        want = np.quantile(vals, list(qs))
        assert got.tolist() == want.tolist()
    with pytest.raises(IndexError):
        dm.histogram_quantiles(np.zeros(5, np.int64))


def test_lineal_path_and_distribution_against_oracle():
    rng = np.random.default_rng(9)
    for _ in range(50):
        N = int(rng.integers(1, 30))
        counts = rng.integers(0, 50, N + 1)
        allp, lines = int(rng.integers(0, 5)), int(rng.integers(5, 100))
        assert dm.lineal_path(counts, allp, lines, N).tolist() == om.lineal_path(counts, allp, lines, N).tolist()
        prob, surv, frac = dm.chord_length_distribution(counts)
        n = counts.sum()
        assert prob.tolist() == (counts[1:] / n).tolist()
        assert surv[0] == pytest.approx(counts[1:].sum() / n)
        assert math.isclose(float(frac.sum()), 1.0, rel_tol=1e-12) or counts[1:].sum() == 0

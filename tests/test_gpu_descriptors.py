"""Morphology descriptors on the device (pr_morphology_counts through porerad_b200.descriptors)
against the reference's outputs stored in tests/golden/descriptors.json, the archived columns of
data/microstructures.csv, and counts taken on the CPU for seeded arrays of many shapes."""

from __future__ import annotations

import numpy as np
import pytest

from tests.helpers import descriptor_phases, descriptor_records, random_phases
from tests.test_descriptors_host import ALL, RECORDS, check_directional, check_scalar, cpu_counts

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def dm():
    from porerad_b200 import descriptors

    return descriptors


@pytest.mark.parametrize("group,name", ALL)
def test_descriptors_against_reference(dm, group, name):
    rec = RECORDS[group][name]
    ph = descriptor_phases(name, rec)
    if "scalar" in rec:
        check_scalar(dm.scalar_descriptors(ph), rec["scalar"])
    else:
        with pytest.raises(ZeroDivisionError):
            dm.scalar_descriptors(ph)
    for a in range(3):
        chords, allp, M, N = dm.periodic_chords(ph == 0, a)
        g = rec["chords"][a]
        assert (np.bincount(chords, minlength=N + 1).tolist(), allp, M, N) == (
            g["hist"], g["all_pore"], g["lines"], g["N"])
    assert dm.interface_face_counts(ph == 1).tolist() == rec["interface_face_counts"]
    if "directional" in rec:
        check_directional(dm.directional_descriptors(ph), rec["directional"])


@pytest.mark.parametrize("name", sorted(descriptor_records()["stored"]))
def test_archived_microstructure_table(dm, name):
    """data/microstructures.csv: realized phi, A_s, L_m and mean axial pore chords, exactly."""

    rec = RECORDS["stored"][name]
    a = rec["archived"]
    ph = descriptor_phases(name, rec)
    d = dm.scalar_descriptors(ph)
    assert d["phi_solid"] == a["realized_phi"]
    assert d["interfacial_area_density"] == a["interfacial_area_density_per_cell"]
    assert d["mean_beam_length"] == a["mean_beam_length_cells"]
    assert list(d["mean_pore_chord"]) == [a["mean_pore_chord_x_cells"], a["mean_pore_chord_y_cells"],
                                          a["mean_pore_chord_z_cells"]]
    assert dm.interface_area(ph == 1) == round(a["interfacial_area_density_per_cell"] * ph.size)
    assert dm.mean_pore_chords(ph == 0) == tuple(d["mean_pore_chord"])
    assert dm.pore_connectivity(ph == 0) == (tuple(d["pore_percolates"]), d["pore_largest_cluster_fraction"])


SHAPES = [((1, 1, 1), 0.0), ((1, 1, 1), 1.0), ((2, 3, 4), 0.5), ((5, 1, 9), 0.3), ((33, 17, 65), 0.25),
          ((64, 200, 33), 0.45), ((127, 31, 3), 0.7), ((40, 40, 40), 0.8), ((96, 96, 96), 0.65),
          ((256, 256, 256), 0.3), ((200, 150, 260), 0.1)]


@pytest.mark.parametrize("shape,phi", SHAPES)
def test_counts_against_cpu(dm, shape, phi):
    """Every count (faces, runs, chord histograms, all-pore lines, clusters, percolation) equals
    the one taken on the CPU, for boxes from one cell to 17M cells and percolating or broken pores."""

    ph = random_phases(shape, phi, 100 + len(shape) + int(100 * phi)) if 0.0 < phi < 1.0 else np.full(
        shape, int(phi), np.uint8)
    same_counts(dm.morphology_counts(ph), cpu_counts(ph))


def same_counts(a, b):
    for k, v in vars(b).items():
        if k == "chord_counts":
            assert all(np.array_equal(x, y) for x, y in zip(a.chord_counts, v))
        else:
            assert getattr(a, k) == v, k


def test_device_and_other_inputs(dm):
    import torch

    ph = descriptor_phases("OF_canonical_phi0.10_N128", RECORDS["stored"]["OF_canonical_phi0.10_N128"])
    host = dm.morphology_counts(ph)
    same_counts(dm.morphology_counts(torch.from_numpy(ph).cuda()), host)
    assert dm.scalar_descriptors(ph.astype(np.int64)) == dm.scalar_descriptors(ph)
    assert dm.scalar_descriptors(torch.from_numpy(ph == 1).cuda()) == dm.scalar_descriptors(ph)
    odd = ph.copy()
    odd[0, 0, :5] = 7  # neither phase, as in the reference's masks p == 1 and p == 0
    c = dm.morphology_counts(odd)
    w = cpu_counts(odd)
    assert (c.solid_cells, c.pore_cells, c.interface_faces, c.periodic_faces, c.pore_runs) == (
        w.solid_cells, w.pore_cells, w.interface_faces, w.periodic_faces, w.pore_runs)
    partial = dm.morphology_counts(ph, chords=False, connectivity=False)
    assert partial.chord_counts is None and partial.pore_clusters == -1 and partial.all_pore_lines == (-1, -1, -1)
    with pytest.raises(ValueError):
        dm.morphology_counts(np.zeros((4, 4), np.uint8))
    with pytest.raises(ValueError):
        dm.morphology_counts(np.zeros((4, 0, 4), np.uint8))


def test_many_at_once_equals_one_by_one(dm):
    arrays = [descriptor_phases(n, RECORDS["stored"][n]) for n in sorted(RECORDS["stored"])[:6]]
    many = dm.all_descriptors_many(arrays)
    for a, (sc, rows) in zip(arrays, many):
        s1, r1 = dm.all_descriptors(a)
        assert sc == s1
        for x, y in zip(rows, r1):
            assert {k: v for k, v in x.items() if k not in ("lineal_path", "chord_counts")} == \
                   {k: v for k, v in y.items() if k not in ("lineal_path", "chord_counts")}
            assert np.array_equal(x["chord_counts"], y["chord_counts"])

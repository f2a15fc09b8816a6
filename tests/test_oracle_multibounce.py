"""The multi-bounce oracle (oracle/multibounce.c) against archived rows of
results/radiative_properties.csv and results/penetration_response.csv (CPU)."""

from __future__ import annotations

import math

import numpy as np
import pytest

from oracle import multibounce as om
from tests.helpers import load_canonical, multibounce_rows

ROWS = multibounce_rows()
NAME = "FI_core_phi0.05_s3"


def _one_per_microstructure(kind):
    seen, out = set(), []
    for r in ROWS[kind]:
        if r["microstructure"] not in seen:
            seen.add(r["microstructure"])
            out.append(r)
    return out


def _solid(name, axis):
    ph = load_canonical(name)
    return np.ascontiguousarray(np.moveaxis(ph == 1, "xyz".index(axis), 0)).astype(np.uint8)


@pytest.mark.parametrize("row", [r for r in ROWS["penetration"] if r["microstructure"] == NAME][:3])
def test_penetration_counts(row):
    n = 500_000
    counts = sum(om.run(_solid(NAME, row["transfer_axis"]), row["epsilon"], n, s, penetration=True) for s in (321, 654))
    for k, key in enumerate(("reflectance", "transmittance", "absorptance")):
        assert counts[k] / (2 * n) == pytest.approx(row[key], abs=1e-12)


@pytest.mark.parametrize("row", [r for r in ROWS["properties"] if r["microstructure"] == NAME][:3])
def test_property_estimates(row):
    tal = [om.run(_solid(NAME, row["transfer_axis"]), row["epsilon"], 200_000, s, penetration=False)
           for s in (123, 456)]
    beta = np.mean([t[0] / (t[1] + t[3]) for t in tal])
    omega = np.mean([t[5] / t[4] for t in tal])
    g = np.mean([t[6] / t[5] for t in tal])
    assert math.isclose(beta, row["beta_per_cell"], rel_tol=1e-12)
    assert math.isclose(omega, row["omega"], rel_tol=1e-12)
    assert math.isclose(g, row["g"], rel_tol=1e-10)


@pytest.mark.parametrize("row", _one_per_microstructure("penetration"), ids=lambda r: r["microstructure"])
def test_penetration_every_microstructure(row):
    n = 500_000
    solid = _solid(row["microstructure"], row["transfer_axis"])
    counts = sum(om.run(solid, row["epsilon"], n, s, penetration=True) for s in (321, 654))
    assert counts[1] / (2 * n) == pytest.approx(row["transmittance"], abs=1e-12)


@pytest.mark.parametrize("row", _one_per_microstructure("properties"), ids=lambda r: r["microstructure"])
def test_properties_every_microstructure(row):
    solid = _solid(row["microstructure"], row["transfer_axis"])
    tal = [om.run(solid, row["epsilon"], 200_000, s, penetration=False) for s in (123, 456)]
    assert math.isclose(np.mean([t[0] / (t[1] + t[3]) for t in tal]), row["beta_per_cell"], rel_tol=1e-12)
    assert math.isclose(np.mean([t[5] / t[4] for t in tal]), row["omega"], rel_tol=1e-12)


@pytest.mark.parametrize("row", [r for r in ROWS["penetration_hit_point"]][::9], ids=lambda r: r["microstructure"])
def test_penetration_hit_point_restart(row):
    """results/hit_point_restart/penetration_response.csv: the other restart rule."""

    n = 500_000
    solid = _solid(row["microstructure"], row["transfer_axis"])
    counts = sum(om.run(solid, row["epsilon"], n, s, penetration=True, restart="hit_point") for s in (321, 654))
    for k, key in enumerate(("reflectance", "transmittance", "absorptance")):
        assert counts[k] / (2 * n) == pytest.approx(row[key], abs=1e-12)


@pytest.mark.parametrize("row", [r for r in ROWS["properties_hit_point"]][::9], ids=lambda r: r["microstructure"])
def test_properties_hit_point_restart(row):
    """results/hit_point_restart/radiative_properties.csv: the other restart rule."""

    solid = _solid(row["microstructure"], row["transfer_axis"])
    tal = [om.run(solid, row["epsilon"], 200_000, s, penetration=False, restart="hit_point") for s in (123, 456)]
    assert math.isclose(np.mean([t[0] / (t[1] + t[3]) for t in tal]), row["beta_per_cell"], rel_tol=1e-12)
    assert math.isclose(np.mean([t[5] / t[4] for t in tal]), row["omega"], rel_tol=1e-12)
    assert math.isclose(np.mean([t[6] / t[5] for t in tal]), row["g"], rel_tol=1e-10)

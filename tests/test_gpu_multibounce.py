"""GPU parity of the multi-bounce ray statistics: radiative properties and penetration response.

The kernels follow the reference's rays one for one (same hash generator, traversal and
Lambertian sampling), so against the archived rows of results/radiative_properties.csv and
results/penetration_response.csv (every stored microstructure x axis x emissivity, 2 seeds
each): the penetration fractions are equal (they are counts of rays), the reflected and
interacting counts behind omega are equal, and beta and g (ratios of sums of lengths and
cosines, which the reference adds with atomics in thread order) agree to 1e-12 relative (the
standard error of g, a difference of nearly equal sums, to 1e-9).
"""

from __future__ import annotations

import pytest

from tests.helpers import load_canonical, multibounce_rows

pytestmark = pytest.mark.gpu

SUM_RTOL = 1e-12  # summation order of lengths and cosines
VAR_RTOL = 1e-9   # g_se: sum(mu^2) - n g^2 cancels, amplifying the summation-order differences


def _rows(kind):
    return multibounce_rows()[kind]


@pytest.mark.parametrize("row", _rows("properties"), ids=lambda r: f"{r['microstructure']}-{r['transfer_axis']}-{r['epsilon']}")
def test_properties_against_archived(row):
    from porerad_b200 import properties

    got = properties.identify_properties(load_canonical(row["microstructure"]), row["transfer_axis"], row["epsilon"])
    assert got["n_rays"] == int(row["n_rays"])
    for key, ref in (("beta", "beta_per_cell"), ("beta_se", "beta_se_per_cell"), ("omega", "omega"),
                     ("omega_se", "omega_se"), ("g", "g"), ("g_se", "g_se"),
                     ("beta_ci95_low", "beta_ci95_low_per_cell"), ("beta_ci95_high", "beta_ci95_high_per_cell")):
        tol = VAR_RTOL if key == "g_se" else SUM_RTOL
        assert abs(got[key] - row[ref]) <= tol * abs(row[ref]), (key, got[key], row[ref])


@pytest.mark.parametrize("row", _rows("penetration"), ids=lambda r: f"{r['microstructure']}-{r['transfer_axis']}-{r['epsilon']}")
def test_penetration_against_archived(row):
    from porerad_b200 import penetration

    got = penetration.penetration_response(load_canonical(row["microstructure"]), row["transfer_axis"], row["epsilon"])
    assert got["n_rays"] == int(row["n_rays"])
    for key in ("reflectance", "transmittance", "absorptance"):
        assert got[key] == row[key], key
        assert abs(got[key + "_se"] - row[key + "_se"]) <= SUM_RTOL * row[key + "_se"], key


def test_restart_rules_and_errors():
    from porerad_b200 import penetration, properties

    row = _rows("properties")[0]
    ph = load_canonical(row["microstructure"])
    a = properties.trace_properties(ph, "x", 0.6, n_rays=20000, restart="article")
    b = properties.trace_properties(ph, "x", 0.6, n_rays=20000, restart="hit_point")
    assert a["beta"] == b["beta"]  # the first path segment does not depend on the rule
    assert a["omega"] != b["omega"] or a["g"] != b["g"]
    p = penetration.trace_penetration(ph, "x", 0.6, n_rays=20000, restart="hit_point")
    assert abs(p["reflectance"] + p["transmittance"] + p["absorptance"] + p["terminated"] / 20000 - 1.0) <= 1e-12
    with pytest.raises(ValueError):
        properties.trace_properties(ph, "x", 0.6, restart="nearest")

"""GPU parity of the multi-bounce ray statistics under the other restart rule ("hit_point": a
reflected ray restarts from its hit point) against results/hit_point_restart/ for every stored
microstructure x axis x emissivity, with the tolerances of the article-rule rows."""

from __future__ import annotations

import pytest

from tests.helpers import load_canonical, multibounce_rows
from tests.test_gpu_multibounce import SUM_RTOL, VAR_RTOL

pytestmark = pytest.mark.gpu


def _rows(kind):
    return multibounce_rows()[kind]


@pytest.mark.parametrize("row", _rows("properties_hit_point"),
                         ids=lambda r: f"{r['microstructure']}-{r['transfer_axis']}-{r['epsilon']}")
def test_properties_hit_point_against_archived(row):
    from porerad_b200 import properties

    got = properties.identify_properties(load_canonical(row["microstructure"]), row["transfer_axis"], row["epsilon"],
                                         restart="hit_point")
    assert got["n_rays"] == int(row["n_rays"])
    for key, ref in (("beta", "beta_per_cell"), ("omega", "omega"), ("omega_se", "omega_se"), ("g", "g"),
                     ("g_se", "g_se")):
        tol = VAR_RTOL if key == "g_se" else SUM_RTOL
        assert abs(got[key] - row[ref]) <= tol * abs(row[ref]), (key, got[key], row[ref])


@pytest.mark.parametrize("row", _rows("penetration_hit_point"),
                         ids=lambda r: f"{r['microstructure']}-{r['transfer_axis']}-{r['epsilon']}")
def test_penetration_hit_point_against_archived(row):
    from porerad_b200 import penetration

    got = penetration.penetration_response(load_canonical(row["microstructure"]), row["transfer_axis"],
                                           row["epsilon"], restart="hit_point")
    assert got["n_rays"] == int(row["n_rays"])
    for key in ("reflectance", "transmittance", "absorptance"):
        assert got[key] == row[key], key

"""Host helpers of porerad_b200.coupled against the oracle's restatement of coupled.py (no GPU)."""

from __future__ import annotations

from types import SimpleNamespace

import numpy as np
import pytest

from porerad_b200 import coupled


@pytest.mark.parametrize("shape", [(7, 5, 3), (16, 12, 9), (3, 20, 8), (64, 64, 64), (9, 1, 2)])
def test_coarse_source_and_linear_field(oracle, shape):
    a = np.random.default_rng(sum(shape)).standard_normal(shape)
    got, want = coupled.coarse_source(a), oracle.coarse_source(a)
    assert got.shape == want.shape
    assert np.max(np.abs(got - want)) <= 1e-14 * np.max(np.abs(want))
    assert np.array_equal(coupled.linear_cell_temperature(shape, 700.0, 20.0),
                          oracle.linear_cell_temperature(shape, 700.0, 20.0))


def test_ab_differences_and_append_rule(oracle):
    rng = np.random.default_rng(5)
    mk = lambda: SimpleNamespace(q_h=rng.normal(100, 1), q_c=rng.normal(-90, 1), q_i=0.0,
                                 coarse_source=rng.standard_normal((8, 8, 8)))
    a, b = [mk() for _ in range(3)], [mk() for _ in range(3)]
    assert coupled.ab_differences(a, b) == pytest.approx(oracle.ab_differences(a, b), rel=1e-15)
    for ch, src in ((0.005, 0.01), (0.02, 0.01), (0.005, 0.06), (0.01, 0.05)):
        assert coupled.append_required(ch, src) == oracle.append_required(ch, src)
    assert coupled.relative_difference(0.0, 0.0) == 0.0


def test_acceptance_failures_names():
    ok = SimpleNamespace(converged=True, linear_residuals_pass=True)
    m = dict(wall_flux_mismatch_rel=0.001, energy_residual_rel=1e-6, temperature_bound_violations=0)
    assert coupled.acceptance_failures(ok, m) == []
    bad = SimpleNamespace(converged=False, linear_residuals_pass=True)
    got = coupled.acceptance_failures(bad, {**m, "wall_flux_mismatch_rel": 0.01})
    assert got == ["Newton iteration converged", "wall-flux mismatch <= 0.5 %"]

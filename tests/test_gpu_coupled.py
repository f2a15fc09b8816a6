"""GPU parity of conduction and the strictly coupled Newton-Krylov solve.

The conduction system's diagonal and wall responses must equal the reference's bit for
bit (same face order of the sums).  Solves are compared with stated tolerances: the
pure-conduction field stops at a relative residual of 1e-11 and the Newton iteration at
1e-13 W; fields agree to about 1e-10 relative, the wall-flux metrics to 1e-8.  The
archived rows of results/coupled.csv (canonical microstructures, counts from the stored
seeds) are reproduced through the whole device path.
"""

from __future__ import annotations

import hashlib
import json

import numpy as np
import pytest

from tests.helpers import (GOLDEN, SMALL, case_phases, count_hash_cases, coupled_rows, load_canonical, load_coupled,
                           load_small)

pytestmark = pytest.mark.gpu

FIELD_RTOL = 1e-9     # final temperature fields (Newton converged to 1e-13 W, step 1e-10 K)
METRIC_RTOL = 1e-8    # wall fluxes, fractions, k_eff, T_min / T_max
ARCHIVE_RTOL = 1e-7   # archived rows: also carry the balancing tolerance of the operator (d to 1e-8)


def _rel(a, b):
    a, b = np.asarray(a, float), np.asarray(b, float)
    return float(np.max(np.abs(a - b)) / max(float(np.max(np.abs(b))), 1e-300))


def _small_setup(name):
    from porerad_b200 import conduction, exchange, view_factors as vf
    from porerad_b200.constants import K_GAS, K_SOLID

    case = load_small(name)
    ph = case["phases"]
    H = float(case["H_m"])
    n = case["patches_patch_class"].size
    R = int(case["rays_per_patch"]) * len(case["seeds"])
    op = exchange.ExchangeOperator(case["pooled_origin"], case["pooled_receiver"], case["pooled_count"],
                                   np.full(n, R, np.int64), case["patches_patch_area_m2"])
    p = vf.build_surface_patches(ph, H)
    system = conduction.assemble_conduction(np.where(ph == 1, K_SOLID, K_GAS), H)
    return case, op, p, system


@pytest.mark.parametrize("name", SMALL)
def test_conduction_system_bit_exact(name, oracle):
    case, op, p, system = _small_setup(name)
    g = load_coupled(name)
    assert np.array_equal(system.matrix.diagonal(), g["diag"])
    assert np.array_equal(system.hot_rhs, g["hot_rhs"]) and np.array_equal(system.cold_rhs, g["cold_rhs"])
    ref = oracle.assemble_conduction(system.conductivity, system.H_m)
    assert (system.matrix != ref.matrix).nnz == 0  # the materialised CSR is the reference's matrix
    x = np.random.default_rng(3).standard_normal(system.conductivity.size)
    assert _rel(system.apply(x), ref.matrix @ x) <= 1e-14
    T = 600.0 + 50.0 * np.random.default_rng(4).random(system.conductivity.size)
    got = system.wall_fluxes(T, 650.0, 550.0)
    want = oracle.wall_fluxes(ref, T, 650.0, 550.0)
    assert _rel(got, want) <= 1e-13


@pytest.mark.parametrize("name", SMALL)
def test_coupled_solve_against_reference(name):
    from porerad_b200 import conduction, coupled

    case, op, p, system = _small_setup(name)
    g = load_coupled(name)
    names = [str(x) for x in g["metric_names"]]
    for k, (Tm, dT, eps) in enumerate(g["conditions"]):
        Th, Tc = Tm + dT / 2.0, Tm - dT / 2.0
        T0 = conduction.solve_conduction(system, Th, Tc)
        assert _rel(T0, g[f"T_initial_{k}"]) <= 1e-10
        res = coupled.solve_coupled(system, op, p, Th, Tc, eps, g[f"T_initial_{k}"])
        m = coupled.wall_flux_metrics(system, p, res, Th, Tc)
        assert not coupled.acceptance_failures(res, m), coupled.acceptance_failures(res, m)
        assert res.newton_iterations == int(g["record"][k][0])
        assert res.preconditioner_steps == int(g["record"][k][1])
        assert _rel(res.temperature_K, g[f"T_final_{k}"]) <= FIELD_RTOL
        assert _rel(res.state.cell_net_power_W, g[f"cell_power_{k}"]) <= 1e-7
        for j, key in enumerate(names):
            want = g["metrics"][k][j]
            if key in ("wall_flux_mismatch_rel", "energy_residual_rel"):
                assert m[key] <= max(100 * want, 1e-10), key
            else:
                assert abs(m[key] - want) <= METRIC_RTOL * max(abs(want), 1.0), key


def test_newton_krylov_fixed_steps_and_errors():
    from porerad_b200 import conduction, coupled

    case, op, p, system = _small_setup("box12")
    g = load_coupled("box12")
    Tm, dT, eps = g["conditions"][0]
    Th, Tc = Tm + dT / 2.0, Tm - dT / 2.0
    res = coupled.newton_krylov(system, op, p, Th, Tc, eps, g["T_initial_0"], 20)
    assert res.converged and res.preconditioner_steps == 20
    assert res.linear_residuals_pass
    assert _rel(res.temperature_K, g["T_final_0"]) <= FIELD_RTOL
    with pytest.raises(ValueError):
        coupled.newton_krylov(system, op, p, Th, Tc, eps, g["T_initial_0"], 0)
    with pytest.raises(ValueError):
        coupled.solve_coupled(system, op, p, Tc, Th, eps, g["T_initial_0"])  # walls swapped


@pytest.mark.parametrize("case_id", [r["case_id"] for r in coupled_rows()])
def test_archived_coupled_rows(case_id):
    """results/coupled.csv through counts, operator, conduction and the coupled solve on the device."""

    from porerad_b200 import conduction, coupled, exchange, view_factors as vf
    from porerad_b200.constants import K_GAS, K_SOLID

    row = next(r for r in coupled_rows() if r["case_id"] == case_id)
    ph = vf.orient_along_x(case_phases(row["microstructure"]), row["axis"])
    ph = np.ascontiguousarray(np.concatenate([ph] * row["repeats"], axis=0))
    assert ph.shape[0] == row["N_axis"]
    assert hashlib.sha256(ph.tobytes()).hexdigest() == row["phase_sha256_x"]
    H = row["H_m"]
    Th, Tc = row["T_mean_K"] + row["delta_T_K"] / 2.0, row["T_mean_K"] - row["delta_T_K"] / 2.0
    p = vf.build_surface_patches(ph, H)
    seeds = row["seeds_A"] + row["seeds_B"]
    table = vf.first_hit_counts_pooled(p, row["rays_per_patch"], seeds)
    n = p.n_patches
    op = exchange.ExchangeOperator(table, None, None, np.full(n, row["rays_per_patch"] * len(seeds), np.int64),
                                   np.full(n, (H / ph.shape[0]) ** 2))
    system = conduction.assemble_conduction(np.where(ph == 1, K_SOLID, K_GAS), H)
    T0 = conduction.solve_conduction(system, Th, Tc)
    res = coupled.solve_coupled(system, op, p, Th, Tc, row["epsilon"], T0)
    m = coupled.wall_flux_metrics(system, p, res, Th, Tc)
    assert not coupled.acceptance_failures(res, m), coupled.acceptance_failures(res, m)
    assert res.newton_iterations == row["newton_updates"]
    for key in ("q_cond_hot_W_m2", "q_rad_hot_W_m2", "q_total_hot_W_m2", "q_cond_cold_W_m2", "q_rad_cold_W_m2",
                "q_total_cold_W_m2", "radiative_fraction_hot", "k_eff_apparent_W_mK", "T_min_K", "T_max_K"):
        want = row[key]
        if want is None:
            continue
        assert abs(m[key] - want) <= ARCHIVE_RTOL * abs(want), (key, m[key], want)
    assert m["wall_flux_mismatch_rel"] <= 0.005 and m["energy_residual_rel"] <= 1e-3
    op.close()
    table.close()


@pytest.mark.parametrize("case_id", ["coupled_TL_y_T700_eps0.6_N128", "coupled_FI_x_T400_eps0.6_N128"])
def test_coupled_case_driver(case_id):
    """cases.coupled_case (the run_coupled.py sequence) on archived rows: the stored count hashes
    of sets A and B reproduced, the archived row, and the A/B comparison."""

    from porerad_b200 import cases

    row = next(r for r in coupled_rows() if r["case_id"] == case_id)
    h = count_hash_cases()[f"{row['microstructure']}|{row['axis']}"]
    case = dict(case_id=case_id, group=row["group"], microstructure=row["microstructure"], transfer_axis=row["axis"],
                repeats_along_axis=row["repeats"], H_m=row["H_m"], N_axis=row["N_axis"], T_mean_K=row["T_mean_K"],
                delta_T_K=row["delta_T_K"], epsilon=row["epsilon"], rays_per_patch_per_block=row["rays_per_patch"],
                seeds_A=";".join(str(s) for s in row["seeds_A"]), seeds_B=row["seeds_B"],
                phase_sha256_x=row["phase_sha256_x"], raw_count_sha256_A=h["sha256_A"], raw_count_sha256_B=h["sha256_B"])
    out = cases.coupled_case(case, load_canonical(row["microstructure"]), ab=True)
    assert out.count_hashes == {"A": True, "B": True}
    assert out.row["newton_updates"] == row["newton_updates"]
    assert set(out.row) <= set(cases.COUPLED_COLUMNS)
    for key in ("q_total_hot_W_m2", "q_rad_hot_W_m2", "k_eff_apparent_W_mK", "T_min_K", "T_max_K"):
        assert abs(out.row[key] - row[key]) <= ARCHIVE_RTOL * abs(row[key]), key
    assert out.ab["max_temperature_difference_K"] >= 0.0 and out.ab["total_flux_rel_difference"] >= 0.0
    bad = dict(case, phase_sha256_x="0" * 64)
    with pytest.raises(ValueError):
        cases.coupled_case(bad, load_canonical(row["microstructure"]))


RAYSET = json.loads((GOLDEN / "ray_set_comparison.json").read_text())["rows"]


@pytest.mark.parametrize("ref", RAYSET, ids=lambda r: f"{r['microstructure']}-{r['axis']}")
def test_ray_set_comparison_rows(ref):
    """results/coupled_ray_set_comparison.csv (run_coupled.py --ab): the coupled solves with sets A
    and B on their own differ by the archived largest temperature difference and relative
    total-flux difference (the latter a difference of nearly equal fluxes: compared absolutely)."""

    from porerad_b200 import cases

    row = next(r for r in coupled_rows() if r["microstructure"] == ref["microstructure"] and r["axis"] == ref["axis"]
               and r["T_mean_K"] == ref["T_mean_K"] and r["epsilon"] == ref["epsilon"] and r["repeats"] == 1)
    case = dict(case_id=row["case_id"], transfer_axis=row["axis"], repeats_along_axis=row["repeats"], H_m=row["H_m"],
                N_axis=row["N_axis"], T_mean_K=row["T_mean_K"], delta_T_K=row["delta_T_K"], epsilon=row["epsilon"],
                rays_per_patch_per_block=row["rays_per_patch"], seeds_A=row["seeds_A"], seeds_B=row["seeds_B"],
                phase_sha256_x=row["phase_sha256_x"])
    out = cases.coupled_case(case, load_canonical(row["microstructure"]), ab=True)
    dT, dq = out.ab["max_temperature_difference_K"], out.ab["total_flux_rel_difference"]
    assert abs(dT - ref["max_temperature_difference_K"]) <= 1e-6 * ref["max_temperature_difference_K"] + 1e-9
    assert abs(dq - ref["total_flux_rel_difference"]) <= 1e-6


def test_conduction_system_from_reference_fields():
    """ConductionSystem built as the reference's dataclass (matrix, hot_rhs, cold_rhs, conductivity,
    H_m) from an assembled system's own arrays; arrays of another field are rejected."""

    from porerad_b200 import conduction
    from porerad_b200.constants import K_GAS, K_SOLID

    case = load_small("slab16")
    k = np.where(case["phases"] == 1, K_SOLID, K_GAS)
    ref = conduction.assemble_conduction(k, float(case["H_m"]))
    again = conduction.ConductionSystem(ref.matrix, ref.hot_rhs, ref.cold_rhs, k, float(case["H_m"]))
    assert (again.matrix != ref.matrix).nnz == 0
    assert np.array_equal(again.boundary_rhs(710.0, 690.0), ref.boundary_rhs(710.0, 690.0))
    with pytest.raises(ValueError):
        conduction.ConductionSystem(ref.matrix * 2.0, None, None, k, float(case["H_m"]))
    with pytest.raises(ValueError):
        conduction.ConductionSystem(None, ref.cold_rhs, None, k, float(case["H_m"]))

"""The oracle against the reference's golden vectors (CPU only).

The oracle must reproduce the reference module's outputs on the seeded fixtures, the
first-hit count hashes the reference stores in data/cases_coupled.csv, and the fluxes
it archives in results/prescribed_field.csv.
"""

from __future__ import annotations

import hashlib

import numpy as np
import pytest

from tests.helpers import SMALL, count_hash_cases, load_canonical, load_coupled, load_small, prescribed_case


def _rel(a, b):
    a, b = np.asarray(a, float), np.asarray(b, float)
    return float(np.max(np.abs(a - b)) / max(float(np.max(np.abs(b))), 1e-300))


@pytest.mark.parametrize("name", SMALL)
def test_oracle_patches_rays_counts(oracle, name):
    case = load_small(name)
    p = oracle.build_surface_patches(case["phases"], float(case["H_m"]))
    for field in ("solid", "patch_class", "patch_cell", "patch_face", "patch_origin", "patch_normal",
                  "patch_area_m2", "cell_face_patch", "hot_wall_patch", "cold_wall_patch"):
        got, want = getattr(p, field), case["patches_" + field]
        assert got.dtype == want.dtype and np.array_equal(got, want), field
    p0, p1 = (int(v) for v in case["ray_range"])
    R = int(case["rays_per_patch"])
    o, d = oracle.generate_rays(p, p0, p1, R, int(case["seeds"][0]))
    assert np.array_equal(o, case["ray_origins"]) and np.array_equal(d, case["ray_directions"])
    assert np.array_equal(oracle.trace_first_hit(p, o, d), case["ray_receivers"])
    tables = []
    for k, s in enumerate(int(x) for x in case["seeds"]):
        t = oracle.first_hit_counts(p, R, s, patch_chunk=97)
        for got, key in zip(t, ("origin", "receiver", "count")):
            assert np.array_equal(got, case[f"seed{k}_{key}"])
        tables.append(t)
    pooled = oracle.pool_counts(tables, p.n_patches)
    rays = np.full(p.n_patches, R * len(tables), np.int64)
    assert oracle.count_sha256(*pooled, rays) == case["count_hash"].item().decode()


@pytest.mark.parametrize("name", SMALL)
def test_oracle_operator_radiosity_channels(oracle, name):
    case = load_small(name)
    n = case["patches_patch_class"].size
    R = int(case["rays_per_patch"]) * len(case["seeds"])
    area = case["patches_patch_area_m2"]
    op = oracle.ExchangeOperator(case["pooled_origin"], case["pooled_receiver"], case["pooled_count"],
                                 np.full(n, R, np.int64), area)
    assert op.row_sum_error <= 1e-10
    assert _rel(op.scale, case["scale"]) <= 1e-12  # same SciPy Anderson iteration as the reference
    x = case["probe_x"]
    assert _rel(op.symmetric_matvec(x), case["probe_sym"]) <= 1e-14
    assert _rel(op.rmatvec(x), case["probe_rmatvec"]) <= 1e-12
    res = oracle.net_patch_power(op, case["T"], case["eps"], area, relative_tolerance=1e-13,
                                 reference_temperature_K=650.0)
    assert _rel(res.absorbed_power_W, case["ref_absorbed"]) <= 1e-12
    p = oracle.build_surface_patches(case["phases"], float(case["H_m"]))
    for row, coarse in zip(case["channels"], case["coarse"]):
        ch = oracle.prescribed_field_channels(op, p, *row[:3])
        scale = max(abs(row[3]), abs(row[4]), abs(row[5]))
        assert abs(ch.q_h - row[3]) <= 1e-12 * scale and abs(ch.q_c - row[4]) <= 1e-12 * scale
        assert abs(ch.q_i - row[5]) <= 1e-12 * scale
        assert _rel(ch.coarse_source, coarse) <= 1e-10


def test_oracle_stored_count_hash(oracle):
    """data/cases_coupled.csv raw_count_sha256_A of the OF canonical case along x (13.8 M rays)."""

    c = count_hash_cases()["OF_canonical_phi0.10_N128|x"]
    ph = oracle.orient_along_x(load_canonical(c["microstructure"]), c["axis"])
    assert hashlib.sha256(ph.tobytes()).hexdigest() == c["phase_sha256_x"]
    p = oracle.build_surface_patches(ph, c["H_m"])
    tables = [oracle.first_hit_counts(p, c["rays_per_patch"], s) for s in c["seeds_A"]]
    pooled = oracle.pool_counts(tables, p.n_patches)
    rays = np.full(p.n_patches, c["rays_per_patch"] * len(tables), np.int64)
    assert oracle.count_sha256(*pooled, rays) == c["sha256_A"]


def test_oracle_archived_prescribed_field_row(oracle):
    """results/prescribed_field.csv, pf_OF_core_phi0.05_s3_x at 700 K, eps 0.6."""

    c = prescribed_case()
    ph = oracle.orient_along_x(load_canonical(c["microstructure"]), c["axis"])
    p = oracle.build_surface_patches(ph, c["H_m"])
    tables = [oracle.first_hit_counts(p, c["rays_per_patch"], s) for s in c["seeds"]]
    pooled = oracle.pool_counts(tables, p.n_patches)
    rays = np.full(p.n_patches, c["rays_per_patch"] * len(tables), np.int64)
    op = oracle.ExchangeOperator(*pooled, rays, p.patch_area_m2)
    row = next(r for r in c["rows"] if r["T_mean_K"] == 700.0 and r["epsilon"] == 0.6)
    ch = oracle.prescribed_field_channels(op, p, 700.0, c["delta_T_K"], 0.6)
    scale = max(abs(row["q_h"]), abs(row["q_c"]), abs(row["q_i"]))
    for got, want in ((ch.q_h, row["q_h"]), (ch.q_c, row["q_c"]), (ch.q_i, row["q_i"])):
        assert abs(got - want) <= 1e-12 * scale


def test_oracle_errors(oracle):
    case = load_small("box12")
    n = case["patches_patch_class"].size
    bad = case["pooled_count"].copy()
    bad[3] += 2
    with pytest.raises(ValueError, match="account for every emitted ray"):
        oracle.ExchangeOperator(case["pooled_origin"], case["pooled_receiver"], bad, np.full(n, 32, np.int64),
                                case["patches_patch_area_m2"])
    p = oracle.build_surface_patches(case["phases"], float(case["H_m"]))
    o = case["ray_origins"][:2].copy()
    d = case["ray_directions"][:2].copy()
    d[0] = (0.0, 0.0, 1.0)
    with pytest.raises(RuntimeError, match="1 rays did not resolve"):
        oracle.trace_first_hit(p, o, d)


@pytest.mark.parametrize("name", SMALL)
def test_oracle_conduction_and_coupled_solve(oracle, name):
    """conduction.py and coupled.py:222-490 against the reference's outputs on the small cases."""

    case = load_small(name)
    g = load_coupled(name)
    ph = case["phases"]
    H = float(case["H_m"])
    system = oracle.assemble_conduction(np.where(ph == 1, oracle.K_SOLID, oracle.K_GAS), H)
    assert np.array_equal(system.matrix.diagonal(), g["diag"])
    assert np.array_equal(system.hot_rhs, g["hot_rhs"]) and np.array_equal(system.cold_rhs, g["cold_rhs"])
    n = case["patches_patch_class"].size
    R = int(case["rays_per_patch"]) * len(case["seeds"])
    op = oracle.ExchangeOperator(case["pooled_origin"], case["pooled_receiver"], case["pooled_count"],
                                 np.full(n, R, np.int64), case["patches_patch_area_m2"])
    p = oracle.build_surface_patches(ph, H)
    names = [str(x) for x in g["metric_names"]]
    for k, (Tm, dT, eps) in enumerate(g["conditions"]):
        Th, Tc = Tm + dT / 2.0, Tm - dT / 2.0
        T0 = oracle.solve_conduction(system, Th, Tc)
        assert _rel(T0, g[f"T_initial_{k}"]) <= 1e-12
        res = oracle.solve_coupled(system, op, p, Th, Tc, eps, T0)
        assert res.converged and oracle.linear_residuals_pass(res)
        assert [res.newton_iterations, res.preconditioner_steps, len(res.linear_solves)] == list(g["record"][k])
        assert _rel(res.temperature_K, g[f"T_final_{k}"]) <= 1e-11
        m = oracle.wall_flux_metrics(system, p, res, Th, Tc)
        for j, key in enumerate(names):
            want = g["metrics"][k][j]
            if key in ("wall_flux_mismatch_rel", "energy_residual_rel"):
                assert m[key] <= max(10 * want, 1e-11), key  # round-off quantities
            else:
                assert abs(m[key] - want) <= 1e-9 * max(abs(want), 1.0), key
        assert m["temperature_bound_violations"] == 0

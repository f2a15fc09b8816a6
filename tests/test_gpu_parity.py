"""GPU parity: libporerad (through porerad_b200 and its C-ABI) against the reference's outputs.

Integer and index results (patch tables, receivers, counts, count hashes) must be
bit-exact.  Floating-point results are compared with stated tolerances: the
operator scale d solves d * (S d) = A only to the balancing tolerance 1e-11, so
quantities downstream of d agree to about 1e-9 relative.
"""

from __future__ import annotations

import hashlib

import numpy as np
import pytest

from tests.helpers import SMALL, case_phases, count_hash_cases, load_canonical, load_small, prescribed_case

pytestmark = pytest.mark.gpu

SCALE_RTOL = 1e-8      # d of two balancing solvers that both stop at max|f| <= 1e-11
PRODUCT_RTOL = 1e-13   # products that do not depend on d (summation order only)
FLUX_RTOL = 1e-9       # radiosity / channel results downstream of d
MIXED_RTOL = 1e-8      # mixed-precision channels against the binary64 result


def _vf():
    from porerad_b200 import view_factors

    return view_factors


def _patches(case):
    return _vf().build_surface_patches(case["phases"], float(case["H_m"]))


def _rel(a, b):
    a, b = np.asarray(a, float), np.asarray(b, float)
    return float(np.max(np.abs(a - b)) / max(float(np.max(np.abs(b))), 1e-300))


@pytest.mark.parametrize("name", SMALL)
def test_patch_table_bit_exact(name):
    case = load_small(name)
    p = _patches(case)
    for field in ("solid", "patch_class", "patch_cell", "patch_face", "patch_origin", "patch_normal",
                  "patch_area_m2", "cell_face_patch", "hot_wall_patch", "cold_wall_patch"):
        got, want = getattr(p, field), case["patches_" + field]
        assert got.dtype == want.dtype and got.shape == want.shape, field
        assert np.array_equal(got, want), field
    assert p.n_patches == case["patches_patch_class"].size


@pytest.mark.parametrize("name", SMALL)
def test_rays(name):
    case = load_small(name)
    p = _patches(case)
    p0, p1 = (int(v) for v in case["ray_range"])
    o, d = _vf().generate_rays(p, p0, p1, int(case["rays_per_patch"]), int(case["seeds"][0]))
    assert np.array_equal(o, case["ray_origins"])
    # directions: own sin/cos is correctly rounded; glibc misrounds ~0.14% of azimuths by 1 ulp
    same = np.all(d == case["ray_directions"], axis=1)
    assert same.mean() >= 0.98
    assert np.allclose(d, case["ray_directions"], rtol=1e-15, atol=1e-16)


@pytest.mark.parametrize("name", SMALL)
def test_trace_given_rays_bit_exact(name):
    case = load_small(name)
    p = _patches(case)
    rec = _vf().trace_first_hit(p, case["ray_origins"], case["ray_directions"])
    assert rec.dtype == np.int32
    assert np.array_equal(rec, case["ray_receivers"])


@pytest.mark.parametrize("name", SMALL)
def test_first_hit_counts_bit_exact(name):
    vf = _vf()
    case = load_small(name)
    p = _patches(case)
    R = int(case["rays_per_patch"])
    seeds = [int(s) for s in case["seeds"]]
    tables = []
    for k, s in enumerate(seeds):
        o, r, c = vf.first_hit_counts(p, R, s)
        assert o.dtype == np.int32 and r.dtype == np.int32 and c.dtype == np.int64
        assert np.array_equal(o, case[f"seed{k}_origin"])
        assert np.array_equal(r, case[f"seed{k}_receiver"])
        assert np.array_equal(c, case[f"seed{k}_count"])
        tables.append((o, r, c))
    pooled = vf.pool_counts(tables, p.n_patches)
    for got, key in zip(pooled, ("pooled_origin", "pooled_receiver", "pooled_count")):
        assert np.array_equal(got, case[key])
    rays = np.full(p.n_patches, R * len(seeds), np.int64)
    assert vf.count_sha256(*pooled, rays) == case["count_hash"].item().decode()
    fused = vf.first_hit_counts_pooled(p, R, seeds)
    assert fused.sha256() == case["count_hash"].item().decode()
    assert fused.rays_traced == p.n_patches * R * len(seeds)
    assert fused.dda_steps >= fused.rays_traced


@pytest.mark.parametrize("name", SMALL)
def test_exchange_operator(name):
    from porerad_b200 import exchange

    case = load_small(name)
    n = case["patches_patch_class"].size
    R = int(case["rays_per_patch"]) * len(case["seeds"])
    rays = np.full(n, R, np.int64)
    area = case["patches_patch_area_m2"]
    op = exchange.ExchangeOperator(case["pooled_origin"], case["pooled_receiver"], case["pooled_count"], rays, area)
    assert op.balance_method in ("anderson", "multiplicative")
    assert op.row_sum_error <= 1e-10
    assert _rel(op.scale, case["scale"]) <= SCALE_RTOL
    # both sides form the same products of the same scale d; the defect stays at rounding level
    assert op.reciprocity_error() <= 1e-12
    assert abs(op.reciprocity_error() - float(case["reciprocity_error"])) <= 4 * np.finfo(np.float64).eps
    assert np.array_equal(op.origin, case["pooled_origin"])
    assert np.array_equal(op.receiver, case["pooled_receiver"])
    assert np.array_equal(op.weight, case["pooled_count"] / np.float64(R))
    x = case["probe_x"]
    assert _rel(op.raw_matvec(x), case["probe_raw"]) <= PRODUCT_RTOL
    assert _rel(op.raw_rmatvec(x), case["probe_raw_t"]) <= PRODUCT_RTOL
    assert _rel(op.symmetric_matvec(x), case["probe_sym"]) <= PRODUCT_RTOL
    assert _rel(op.matvec(x), case["probe_matvec"]) <= SCALE_RTOL
    assert _rel(op.rmatvec(x), case["probe_rmatvec"]) <= SCALE_RTOL
    assert op._closure_error(np.log(op.scale)) <= 1e-10


@pytest.mark.parametrize("name", SMALL)
def test_radiosity(name):
    from porerad_b200 import exchange

    case = load_small(name)
    n = case["patches_patch_class"].size
    R = int(case["rays_per_patch"]) * len(case["seeds"])
    area = case["patches_patch_area_m2"]
    op = exchange.ExchangeOperator(case["pooled_origin"], case["pooled_receiver"], case["pooled_count"],
                                   np.full(n, R, np.int64), area)
    plain = exchange.net_patch_power(op, case["T"], case["eps"], area, relative_tolerance=1e-13)
    assert _rel(plain.absorbed_power_W, case["plain_absorbed"]) <= FLUX_RTOL
    assert abs(plain.iterations - int(case["plain_iterations"])) <= 1
    refd = exchange.net_patch_power(op, case["T"], case["eps"], area, relative_tolerance=1e-13,
                                    reference_temperature_K=650.0)
    assert _rel(refd.absorbed_power_W, case["ref_absorbed"]) <= FLUX_RTOL
    assert abs(refd.global_energy_residual_W) <= 1e-9 * float(np.sum(np.abs(refd.emitted_power_W)))
    jvp = exchange.net_patch_power_jvp(op, case["T"], case["dT"], case["eps"], area, relative_tolerance=1e-13)
    assert _rel(jvp, case["jvp"]) <= FLUX_RTOL
    series = exchange.reflection_series(op, plain.emitted_power_W, case["eps"], relative_tolerance=1e-13)
    assert np.array_equal(series.absorbed_power_W, plain.absorbed_power_W)


@pytest.mark.parametrize("name", SMALL)
def test_prescribed_channels(name):
    from porerad_b200 import coupled, exchange

    case = load_small(name)
    p = _patches(case)
    R = int(case["rays_per_patch"])
    table = _vf().first_hit_counts_pooled(p, R, [int(s) for s in case["seeds"]])
    op = exchange.ExchangeOperator(table, None, None, np.full(p.n_patches, R * len(case["seeds"]), np.int64),
                                   p.patch_area_m2)
    for row, coarse in zip(case["channels"], case["coarse"]):
        Tm, dT, eps, qh, qc, qi, _ = row
        ch = coupled.prescribed_field_channels(op, p, Tm, dT, eps)
        scale = max(abs(qh), abs(qc), abs(qi))
        for got, want in ((ch.q_h, qh), (ch.q_c, qc), (ch.q_i, qi)):
            assert abs(got - want) <= FLUX_RTOL * scale
        assert ch.closure_rel <= 1e-10
        assert float(np.sum(np.abs(ch.coarse_source - coarse))) <= FLUX_RTOL * float(np.sum(np.abs(coarse)))
        mixed = coupled.prescribed_field_channels(op, p, Tm, dT, eps, precision="mixed")
        for got, want in ((mixed.q_h, ch.q_h), (mixed.q_c, ch.q_c)):
            assert abs(got - want) <= MIXED_RTOL * abs(want)
        assert abs(mixed.q_i - ch.q_i) <= MIXED_RTOL * scale


def test_stored_count_hashes():
    """Every stored raw_count_sha256_A/B of the committed canonical microstructures (data/cases_coupled.csv)."""

    vf = _vf()
    cache = {}
    for key, c in sorted(count_hash_cases("stored").items()):
        if c["microstructure"] not in cache:
            cache[c["microstructure"]] = load_canonical(c["microstructure"])
        ph = vf.orient_along_x(cache[c["microstructure"]], c["axis"])
        assert hashlib.sha256(ph.tobytes()).hexdigest() == c["phase_sha256_x"]
        p = vf.build_surface_patches(ph, c["H_m"])
        for s in ("A", "B"):
            table = vf.first_hit_counts_pooled(p, c["rays_per_patch"], c["seeds_" + s])
            assert table.sha256() == c["sha256_" + s], f"{key} set {s}"
            table.close()


@pytest.mark.parametrize("key", sorted(count_hash_cases("generated")))
def test_resolution_count_hashes(key):
    """The stored raw_count_sha256_A/B of the N = 160 and 192 resolution cases (data/cases_coupled.csv):
    the canonical arrays rebuilt by the generators (phase hash checked), 2 blocks of 64 rays per
    patch per set, up to 1.4e8 rays per set."""

    vf = _vf()
    c = count_hash_cases("generated")[key]
    ph = vf.orient_along_x(case_phases(c["microstructure"]), c["axis"])
    assert hashlib.sha256(ph.tobytes()).hexdigest() == c["phase_sha256_x"]
    p = vf.build_surface_patches(ph, c["H_m"])
    for s in ("A", "B"):
        table = vf.first_hit_counts_pooled(p, c["rays_per_patch"], c["seeds_" + s])
        assert table.sha256() == c["sha256_" + s], f"{key} set {s}"
        table.close()


def test_archived_prescribed_field_rows():
    """results/prescribed_field.csv rows of one core case, end to end on the GPU."""

    from porerad_b200 import coupled, exchange

    vf = _vf()
    c = prescribed_case()
    ph = vf.orient_along_x(load_canonical(c["microstructure"]), c["axis"])
    assert hashlib.sha256(ph.tobytes()).hexdigest() == c["phase_sha256_x"]
    p = vf.build_surface_patches(ph, c["H_m"])
    table = vf.first_hit_counts_pooled(p, c["rays_per_patch"], c["seeds"])
    rays = np.full(p.n_patches, c["rays_per_patch"] * len(c["seeds"]), np.int64)
    op = exchange.ExchangeOperator(table, None, None, rays, p.patch_area_m2)
    assert op.row_sum_error <= 1e-10
    for row in c["rows"]:
        ch = coupled.prescribed_field_channels(op, p, row["T_mean_K"], c["delta_T_K"], row["epsilon"])
        scale = max(abs(row["q_h"]), abs(row["q_c"]), abs(row["q_i"]))
        assert abs(ch.q_h - row["q_h"]) <= FLUX_RTOL * scale
        assert abs(ch.q_c - row["q_c"]) <= FLUX_RTOL * scale
        assert abs(ch.q_i - row["q_i"]) <= FLUX_RTOL * scale


def test_accounting_error():
    from porerad_b200 import exchange

    case = load_small("box12")
    n = case["patches_patch_class"].size
    count = case["pooled_count"].copy()
    count[0] += 1
    with pytest.raises(ValueError, match="account for every emitted ray"):
        exchange.ExchangeOperator(case["pooled_origin"], case["pooled_receiver"], count,
                                  np.full(n, 32, np.int64), case["patches_patch_area_m2"])


def test_unresolved_ray_error():
    case = load_small("box12")
    p = _patches(case)
    o = case["ray_origins"][:4].copy()
    d = case["ray_directions"][:4].copy()
    d[1] = (0.0, 1.0, 0.0)  # dx == 0 never resolves (view_factors.py:213-215)
    with pytest.raises(RuntimeError, match="1 rays did not resolve a receiving patch"):
        _vf().trace_first_hit(p, o, d)


def test_empty_and_degenerate_inputs():
    vf = _vf()
    case = load_small("box12")
    p = _patches(case)
    o, d = vf.generate_rays(p, 5, 5, 16, 1)
    assert o.shape == (0, 3) and d.shape == (0, 3)
    assert vf.trace_first_hit(p, o, d).shape == (0,)
    # an all-pore slab: only wall patches, every ray crosses to the opposite wall
    ph = np.zeros((6, 5, 4), np.uint8)
    q = vf.build_surface_patches(ph, 0.01)
    assert q.n_patches == 2 * 5 * 4
    o, r, c = vf.first_hit_counts(q, 8, 3)
    assert np.all(q.patch_class[o] != q.patch_class[r])
    assert int(c.sum()) == q.n_patches * 8
    e = vf.pool_counts([], 7)
    assert all(a.size == 0 for a in e)


@pytest.mark.parametrize("name", SMALL)
def test_device_merge_of_count_tables(name):
    vf = _vf()
    case = load_small(name)
    p = _patches(case)
    R = int(case["rays_per_patch"])
    a, b = (vf.first_hit_counts_pooled(p, R, [int(s)]) for s in case["seeds"][:2])
    merged = a.merge(b)
    assert merged.sha256() == case["count_hash"].item().decode()
    assert merged.rays_traced == a.rays_traced + b.rays_traced


def test_operator_general_areas_against_oracle(oracle):
    """Unequal patch areas select the binary64-value storage of S; checked against the oracle."""

    from porerad_b200 import exchange

    case = load_small("box12")
    n = case["patches_patch_class"].size
    R = int(case["rays_per_patch"]) * len(case["seeds"])
    rays = np.full(n, R, np.int64)
    area = case["patches_patch_area_m2"] * (1.0 + 0.5 * np.random.default_rng(4).random(n))
    args = (case["pooled_origin"], case["pooled_receiver"], case["pooled_count"], rays, area)
    op = exchange.ExchangeOperator(*args)
    ref = oracle.ExchangeOperator(*args)
    assert _rel(op.scale, ref.scale) <= SCALE_RTOL
    x = case["probe_x"]
    assert _rel(op.symmetric_matvec(x), ref.symmetric_matvec(x)) <= PRODUCT_RTOL
    assert _rel(op.rmatvec(x), ref.rmatvec(x)) <= SCALE_RTOL
    assert abs(op.reciprocity_error() - ref.reciprocity_error()) <= 1e-12


def test_operator_wide_counts_storage():
    """Counts and rays scaled by 2^16 keep every weight but no longer fit packed 32-bit words."""

    from porerad_b200 import exchange

    case = load_small("cube20")
    n = case["patches_patch_class"].size
    R = int(case["rays_per_patch"]) * len(case["seeds"])
    k = 1 << 16
    op = exchange.ExchangeOperator(case["pooled_origin"], case["pooled_receiver"], case["pooled_count"] * k,
                                   np.full(n, R * k, np.int64), case["patches_patch_area_m2"])
    assert _rel(op.scale, case["scale"]) <= SCALE_RTOL
    assert _rel(op.symmetric_matvec(case["probe_x"]), case["probe_sym"]) <= PRODUCT_RTOL


@pytest.mark.parametrize("name", SMALL)
def test_cell_field_channels_against_oracle(oracle, name):
    """An arbitrary cell field (walls fixed) against the oracle's evaluate_radiation + channel sums."""

    from porerad_b200 import coupled, exchange

    case = load_small(name)
    p = _patches(case)
    R = int(case["rays_per_patch"]) * len(case["seeds"])
    args = (case["pooled_origin"], case["pooled_receiver"], case["pooled_count"],
            np.full(p.n_patches, R, np.int64), case["patches_patch_area_m2"])
    op = exchange.ExchangeOperator(*args)
    ref_op = oracle.ExchangeOperator(*args)
    q = oracle.build_surface_patches(case["phases"], float(case["H_m"]))
    rng = np.random.default_rng(2)
    T_cells = 700.0 + 5.0 * rng.standard_normal(case["phases"].shape)
    for ref_T, prec in ((700.0, "fp64"), (None, "fp64"), (700.0, "mixed")):
        got = coupled.cell_field_channels(op, p, T_cells, 710.0, 690.0, 0.6, reference_temperature_K=ref_T,
                                          precision=prec)
        Tp = oracle.patch_temperature(q, T_cells, 710.0, 690.0)
        rad = oracle.net_patch_power(ref_op, Tp, np.full(q.n_patches, 0.6), q.patch_area_m2,
                                     relative_tolerance=1e-13, reference_temperature_K=ref_T)
        area = oracle.cross_section_area(q)
        want = [-float(np.sum(rad.net_power_W[q.patch_class == k])) / area for k in (0, 1, 2)]
        scale = max(abs(w) for w in want)
        tol = MIXED_RTOL if prec == "mixed" else FLUX_RTOL
        if ref_T is None:
            tol = max(tol, 1e-7)  # absolute emission T^4 without the reference subtraction: q is a small difference
        for g, w in zip((got.q_h, got.q_c, got.q_i), want):
            assert abs(g - w) <= tol * scale


def test_every_traversal_variant_gives_the_same_counts():
    """The autotuner may pick any compiled variant: all must produce the reference's counts."""

    from porerad_b200 import _lib

    vf = _vf()
    case = load_small("cube20")
    p = _patches(case)
    R = int(case["rays_per_patch"])
    n = ctypes_int = None
    import ctypes

    count = ctypes.c_int()
    _lib.check(_lib.load().pr_trace_variant_info(ctypes.byref(count), None, None))
    try:
        for v in range(count.value):
            _lib.check(_lib.load().pr_trace_set_variant(v))
            t = vf.first_hit_counts_pooled(p, R, [int(s) for s in case["seeds"]])
            assert t.sha256() == case["count_hash"].item().decode(), v
            assert _lib.trace_variant()[0] == v
    finally:
        _lib.load().pr_trace_set_variant(-1)


def test_batched_counts_equal_single_case_counts():
    """Cases of different shapes and sizes traced in shared launches give each case's own counts."""

    from porerad_b200 import geometry

    vf = _vf()
    pats, seeds, want = [], [], []
    for k, name in enumerate(SMALL):
        case = load_small(name)
        pats.append(_patches(case))
        seeds.append([int(s) for s in case["seeds"][:2]])
    for k, arch in enumerate(geometry.ARCHETYPES):
        pats.append(vf.build_surface_patches(geometry.make(arch, 24 + 8 * k, 0.15, k), 0.005))
        seeds.append([1000 + k, 2000 + k])
    R = 24
    for p, ss in zip(pats, seeds):
        t = vf.first_hit_counts_pooled(p, R, ss)
        want.append((t.sha256(), t.dda_steps))
        t.close()
    got = vf.first_hit_counts_batch(pats, R, seeds)
    for g, (h, st) in zip(got, want):
        assert g.sha256() == h
        assert g.dda_steps == st


@pytest.mark.parametrize("R,seeds", [(20, [5]), (64, [6]), (100, [7]), (250, [8]), (700, [9]), (1000, [10]),
                                     (300, [11, 12, 13]), (1100, [14])])
def test_per_patch_reduction_against_oracle(oracle, R, seeds):
    """Counts of every per-patch reduction width (32 to 1024 keys, several seeds, beyond 1024)."""

    vf = _vf()
    case = load_small("box12")
    p = _patches(case)
    po = oracle.build_surface_patches(case["phases"], float(case["H_m"]))
    tables = [oracle.first_hit_counts(po, R, s) for s in seeds]
    want = oracle.pool_counts(tables, po.n_patches) if len(seeds) > 1 else tables[0]
    got = vf.first_hit_counts_pooled(p, R, seeds).to_numpy()
    for g, w in zip(got, want):
        assert np.array_equal(np.asarray(g), np.asarray(w))


def test_operators_built_together_equal_operators_built_alone():
    """ExchangeOperator.from_tables (operators assembled one by one, balancing iterations of all of
    them in lockstep with one product launch per iteration) gives each operator bit for bit as
    ExchangeOperator builds it alone: the four canonical 128^3 microstructures (blocked products)
    and a small case (warp-per-row products, balanced on its own)."""

    from porerad_b200 import exchange

    vf = _vf()
    tables, rays, areas = [], [], []
    for name in ("FA", "FI", "OF", "TL"):
        p = vf.build_surface_patches(load_canonical(f"{name}_canonical_phi0.10_N128"), 0.01)
        tables.append(vf.first_hit_counts_pooled(p, 32, [101, 202]))
        rays.append(np.full(p.n_patches, 64, np.int64))
        areas.append(p.patch_area_m2)
    case = load_small("cube20")
    p = _patches(case)
    R = int(case["rays_per_patch"])
    tables.append(vf.first_hit_counts_pooled(p, R, [int(s) for s in case["seeds"]]))
    rays.append(np.full(p.n_patches, R * len(case["seeds"]), np.int64))
    areas.append(p.patch_area_m2)
    together = exchange.ExchangeOperator.from_tables(tables, rays, areas)
    for t, r, a, op in zip(tables, rays, areas, together):
        alone = exchange.ExchangeOperator(t, None, None, r, a)
        assert op.balance_method == alone.balance_method
        assert op.balance_iterations == alone.balance_iterations
        assert np.array_equal(op.scale, alone.scale)
        assert op.row_sum_error == alone.row_sum_error
        x = np.random.default_rng(3).random(op.n_patches)
        assert np.array_equal(op.matvec(x), alone.matvec(x))
        alone.close()
        op.close()
    with pytest.raises(ValueError):
        exchange.ExchangeOperator.from_tables(tables[:2], rays[:1], areas[:2])
    assert exchange.ExchangeOperator.from_tables([], [], []) == []

"""Regenerate the golden fixtures of tests/golden from the reference implementation.

    python tests/golden/make_golden.py --reference <checkout of porerad> [--only part,part,...]

(or set PORERAD_REFERENCE to the checkout instead of passing --reference.)

Runs the unmodified reference package ``porerad`` (moxi000/pore-radiation-ijhmt2026)
on small seeded inputs and stores its outputs, so that the GPU parity tests can run
where the reference is not installed:

* ``small_<name>.npz``: phases, the full SurfacePatches table, the rays of one patch
  range, the receivers of those rays, per-seed and pooled counts, the count hash,
  the balanced operator (scale, method, row-sum error, reciprocity), one radiosity
  solve with and without a reference temperature, one JVP, and the prescribed-field
  channels (q_h, q_c, q_i, closure, coarse source) at two conditions.
* ``canonical_<name>.npz``: the four canonical 128^3 microstructures of the
  reference's data/microstructures (CC-BY 4.0, credited in tests/golden/README.md), bit-packed.
* ``count_hashes.json``: every stored first-hit count hash of data/cases_coupled.csv
  (columns raw_count_sha256_A/B) with its seeds: the canonical 128^3 microstructures
  stored here (``"array": "stored"``) and the N = 160 and 192 resolution microstructures,
  which are not stored and are rebuilt by the generators from their archived phase hash
  (``"array": "generated"``).
* ``prescribed_field.json``: archived prescribed-field rows of
  results/prescribed_field.csv for the committed core microstructure, with its seeds.
* ``coupled_<name>.npz``: the strictly coupled solve of each small case (conduction
  system of K_SOLID/K_GAS, pure-conduction field, solve_coupled at two conditions: final
  field, wall-flux metrics, Newton and GMRES iteration record).
* ``coupled.json``: every archived row of results/coupled.csv with its case parameters
  (groups canonical, thickness, resolution and matched; ``"array"`` says whether the
  microstructure is stored here or rebuilt by the generators).
* ``public_api.json``: the public names of porerad.view_factors, .exchange, .coupled and
  .conduction (kind, call signature, class members, constant values).
* ``fullpath.json``: the two ``first_hit_radiosity`` rows of results/fullpath_crosscheck.csv
  (OF and TL canonical, x, 700 K, 20 K, eps 0.6) with the ray seeds of the coupled cases'
  sets A + B and the reference's own channels recomputed from them, with the file's full-path
  Monte Carlo rows of the same microstructures (channels and standard errors).
* ``prescribed_cases.json``: all 48 cases of data/cases_prescribed_field.csv (seeds, append
  seeds and decision, conditions, phase hash) with their archived rows of
  results/prescribed_field.csv (q_h, q_c, q_i and the A/B wall-channel difference); their
  18 microstructures are stored like the canonical ones (``canonical_<name>.npz``).
* ``multibounce.json``: the archived rows of results/radiative_properties.csv and
  results/penetration_response.csv (and of results/hit_point_restart/, the other restart rule)
  for the microstructures stored here.
* ``ray_set_comparison.json``: the "A vs B" rows of results/coupled_ray_set_comparison.csv
  (one emissivity, N = 128): largest temperature and relative total-flux differences of the
  coupled solves with sets A and B on their own.
* ``microstructures.json``: every row of data/microstructures.csv (id, structure, set, N,
  target solid fraction, seed, archived phase_sha256) for the generator tests.
* ``descriptors.json``: porerad.descriptors run on every microstructure stored here
  (scalar and directional descriptors, chord histograms, lineal paths) with their archived
  columns of data/microstructures.csv, and on seeded small and 128^3 phase arrays
  (``random_phases``; sha256 of each recorded), edge cases included (uniform arrays,
  thin boxes, all-pore lines, a non-cubic box).
"""

from __future__ import annotations

import argparse
import csv
import hashlib
import json
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent

SMALL_CASES = {
    # name: (shape, solid fraction, phase seed, H, seeds, rays per patch)
    "box12": ((12, 10, 9), 0.30, 7, 0.01, [11, 2212], 16),
    "cube20": ((20, 20, 20), 0.12, 3, 0.004, [5, 912345678901234567], 24),
    "slab16": ((16, 24, 8), 0.20, 9, 0.02, [77, 78], 12),
}
CONDITIONS = [(700.0, 20.0, 0.6), (400.0, 100.0, 0.3)]
CANONICAL = ["FA_canonical_phi0.10_N128", "FI_canonical_phi0.10_N128", "OF_canonical_phi0.10_N128",
             "TL_canonical_phi0.10_N128"]
MATCHED = [f"{s}_matched_pair{k}" for s in ("FA", "FI") for k in (1, 2, 3)]
CORE_CASE = "pf_OF_core_phi0.05_s3_x"


def random_phases(shape, phi, seed):
    rng = np.random.default_rng(seed)
    field = rng.random(shape)
    # a little spatial correlation: average with a rolled copy, then threshold at phi
    field = (field + np.roll(field, 1, axis=0) + np.roll(field, 1, axis=2)) / 3.0
    thr = np.quantile(field, phi)
    return (field < thr).astype(np.uint8)


def small_case(vf, ex, cp, name, spec):
    shape, phi, pseed, H, seeds, R = spec
    phases = random_phases(shape, phi, pseed)
    patches = vf.build_surface_patches(phases, H)
    n = patches.n_patches
    p0, p1 = min(3, n), min(40, n)
    o, d = vf.generate_rays(patches, p0, p1, R, seeds[0])
    rec = vf.trace_first_hit(patches, o, d)
    per_seed = [vf.first_hit_counts(patches, R, s, patch_chunk=max(1, n // 3)) for s in seeds]
    pooled = vf.pool_counts(per_seed, n)
    rays = np.full(n, R * len(seeds), np.int64)
    op = ex.ExchangeOperator(*pooled, rays, patches.patch_area_m2)
    rng = np.random.default_rng(pseed + 100)
    T = 600.0 + 100.0 * rng.random(n)
    eps = np.full(n, 0.7)
    plain = ex.net_patch_power(op, T, eps, patches.patch_area_m2, relative_tolerance=1e-13)
    refd = ex.net_patch_power(op, T, eps, patches.patch_area_m2, relative_tolerance=1e-13,
                              reference_temperature_K=650.0)
    dT = rng.standard_normal(n)
    jvp = ex.net_patch_power_jvp(op, T, dT, eps, patches.patch_area_m2, relative_tolerance=1e-13)
    x = rng.random(n)
    out = dict(
        phases=phases, H_m=np.float64(H), seeds=np.asarray(seeds, np.uint64), rays_per_patch=np.int64(R),
        ray_range=np.asarray([p0, p1], np.int64), ray_origins=o, ray_directions=d, ray_receivers=rec,
        pooled_origin=pooled[0], pooled_receiver=pooled[1], pooled_count=pooled[2],
        count_hash=np.bytes_(vf.count_sha256(*pooled, rays)),
        scale=op.scale, row_sum_error=np.float64(op.row_sum_error),
        reciprocity_error=np.float64(op.reciprocity_error()),
        balance_method=np.bytes_(op.balance_method), probe_x=x,
        probe_raw=op.raw_matvec(x), probe_raw_t=op.raw_rmatvec(x), probe_sym=op.symmetric_matvec(x),
        probe_matvec=op.matvec(x), probe_rmatvec=op.rmatvec(x),
        T=T, eps=eps, dT=dT, plain_absorbed=plain.absorbed_power_W, plain_residual=np.float64(plain.residual_power_W),
        plain_iterations=np.int64(plain.iterations), ref_absorbed=refd.absorbed_power_W,
        ref_iterations=np.int64(refd.iterations), jvp=jvp,
    )
    for k, (o_, r_, c_) in enumerate(per_seed):
        out[f"seed{k}_origin"], out[f"seed{k}_receiver"], out[f"seed{k}_count"] = o_, r_, c_
    for field in ("solid", "patch_class", "patch_cell", "patch_face", "patch_origin", "patch_normal",
                  "patch_area_m2", "cell_face_patch", "hot_wall_patch", "cold_wall_patch"):
        out["patches_" + field] = getattr(patches, field)
    ch = []
    coarse = []
    for Tm, dTm, e in CONDITIONS:
        c = cp.prescribed_field_channels(op, patches, Tm, dTm, e)
        ch.append([Tm, dTm, e, c.q_h, c.q_c, c.q_i, c.closure_rel])
        coarse.append(c.coarse_source)
    out["channels"] = np.asarray(ch)
    out["coarse"] = np.asarray(coarse)
    np.savez_compressed(HERE / f"small_{name}.npz", **out)
    print(f"{name}: {n} patches, {pooled[2].size} pairs, {op.balance_method} {op.balance_iterations}")


COUPLED_CONDITIONS = ((700.0, 20.0, 0.6), (500.0, 200.0, 0.3))  # (T_mean, delta_T, eps)


def coupled_small(name, spec):
    from porerad import conduction, coupled as cp, exchange as ex, view_factors as vf
    from porerad.constants import K_GAS, K_SOLID

    shape, phi, pseed, H, seeds, R = spec
    ph = random_phases(shape, phi, pseed)
    p = vf.build_surface_patches(ph, H)
    o, r, c = vf.pool_counts([vf.first_hit_counts(p, R, s) for s in seeds], p.n_patches)
    op = ex.ExchangeOperator(o, r, c, np.full(p.n_patches, R * len(seeds), np.int64), p.patch_area_m2)
    system = conduction.assemble_conduction(np.where(ph == 1, K_SOLID, K_GAS), H)
    out = dict(diag=system.matrix.diagonal(), hot_rhs=system.hot_rhs, cold_rhs=system.cold_rhs,
               conditions=np.asarray(COUPLED_CONDITIONS))
    names = ("q_cond_hot_W_m2", "q_rad_hot_W_m2", "q_total_hot_W_m2", "q_cond_cold_W_m2", "q_rad_cold_W_m2",
             "q_total_cold_W_m2", "radiative_fraction_hot", "k_eff_apparent_W_mK", "wall_flux_mismatch_rel",
             "energy_residual_rel", "T_min_K", "T_max_K")
    out["metric_names"] = np.asarray(names)
    metrics, record = [], []
    for k, (Tm, dT, eps) in enumerate(COUPLED_CONDITIONS):
        Th, Tc = Tm + dT / 2.0, Tm - dT / 2.0
        T0 = conduction.solve_conduction(system, Th, Tc)
        res = cp.solve_coupled(system, op, p, Th, Tc, eps, T0)
        m = cp.wall_flux_metrics(system, p, res, Th, Tc)
        assert not cp.acceptance_failures(res, m)
        out[f"T_initial_{k}"] = T0
        out[f"T_final_{k}"] = res.temperature_K
        out[f"cell_power_{k}"] = res.state.cell_net_power_W
        metrics.append([m[n] for n in names])
        record.append([res.newton_iterations, res.preconditioner_steps, len(res.linear_solves)])
        out[f"gmres_{k}"] = np.asarray([s["gmres_iterations"] for s in res.linear_solves], np.int64)
    out["metrics"] = np.asarray(metrics)
    out["record"] = np.asarray(record, np.int64)
    np.savez_compressed(HERE / f"coupled_{name}.npz", **out)
    print(f"coupled {name}: newton {[r[0] for r in record]}")


def coupled_rows(ref):
    cases = {r["case_id"]: r for r in csv.DictReader(open(ref / "data" / "cases_coupled.csv"))}
    rows = []
    for r in csv.DictReader(open(ref / "results" / "coupled.csv")):
        c = cases[r["case_id"]]
        stored = c["microstructure"] in CANONICAL or c["microstructure"] in MATCHED
        row = dict(case_id=r["case_id"], group=c["group"], microstructure=c["microstructure"],
                   axis=c["transfer_axis"], repeats=int(c["repeats_along_axis"]), H_m=float(c["H_m"]),
                   N_axis=int(c["N_axis"]), T_mean_K=float(c["T_mean_K"]), delta_T_K=float(c["delta_T_K"]),
                   epsilon=float(c["epsilon"]), rays_per_patch=int(c["rays_per_patch_per_block"]),
                   seeds_A=[int(s) for s in c["seeds_A"].split(";")],
                   seeds_B=[int(s) for s in c["seeds_B"].split(";")], phase_sha256_x=c["phase_sha256_x"],
                   newton_updates=int(r["newton_updates"]), array="stored" if stored else "generated")
        for k in ("q_cond_hot_W_m2", "q_rad_hot_W_m2", "q_total_hot_W_m2", "q_cond_cold_W_m2", "q_rad_cold_W_m2",
                  "q_total_cold_W_m2", "radiative_fraction_hot", "k_eff_apparent_W_mK", "wall_flux_mismatch_rel",
                  "energy_residual_rel", "T_min_K", "T_max_K"):
            row[k] = float(r[k]) if r[k] != "" else None  # some archived rows leave the cold side empty
        rows.append(row)
    (HERE / "coupled.json").write_text(json.dumps(dict(rows=rows, source="data/cases_coupled.csv, "
                                                                           "results/coupled.csv"), indent=1))
    print("coupled rows:", len(rows))


def prescribed_cases(ref):
    cases = list(csv.DictReader(open(ref / "data" / "cases_prescribed_field.csv")))
    res = list(csv.DictReader(open(ref / "results" / "prescribed_field.csv")))
    out = []
    for c in cases:
        rows = [r for r in res if r["case_id"] == c["case_id"]]
        out.append(dict(
            case_id=c["case_id"], group=c["group"], structure=c["structure"], microstructure=c["microstructure"],
            axis=c["transfer_axis"], H_m=float(c["H_m"]), rays_per_patch=int(c["rays_per_patch_per_block"]),
            seeds_A=[int(x) for x in c["seeds_A"].split(";")], seeds_B=[int(x) for x in c["seeds_B"].split(";")],
            append_seeds_A=[int(x) for x in c["append_seeds_A"].split(";")],
            append_seeds_B=[int(x) for x in c["append_seeds_B"].split(";")],
            append_used=c["append_used"] == "true",
            conditions=[[float(a) for a in item.split("/")] for item in c["conditions"].split(";")],
            phase_sha256_x=c["phase_sha256_x"], delta_T_K=float(rows[0]["delta_T_K"]),
            ab_wall_channel_rel_difference=float(rows[0]["ab_wall_channel_rel_difference"]),
            rows=[dict(T_mean_K=float(r["T_mean_K"]), epsilon=float(r["epsilon"]), q_h=float(r["q_h_W_m2"]),
                       q_c=float(r["q_c_W_m2"]), q_i=float(r["q_i_W_m2"])) for r in rows]))
    (HERE / "prescribed_cases.json").write_text(json.dumps(dict(
        cases=out, source="data/cases_prescribed_field.csv, results/prescribed_field.csv"), indent=1))
    names = sorted({c["microstructure"] for c in out})
    for name in names:
        ph = np.load(ref / "data" / "microstructures" / f"{name}.npz")["phases"]
        assert ph.dtype == np.uint8 and set(np.unique(ph)) <= {0, 1}
        np.savez_compressed(HERE / f"canonical_{name}.npz", bits=np.packbits(ph.ravel()),
                            shape=np.asarray(ph.shape, np.int64),
                            sha256=np.bytes_(hashlib.sha256(ph.tobytes()).hexdigest()))
    print("prescribed-field cases:", len(out), "microstructures:", len(names))


def multibounce_rows(ref):
    have = {p.name[len("canonical_"):-4] for p in HERE.glob("canonical_*.npz")}
    out = {}
    for key, name in (("properties", "radiative_properties.csv"), ("penetration", "penetration_response.csv"),
                      ("properties_hit_point", "hit_point_restart/radiative_properties.csv"),
                      ("penetration_hit_point", "hit_point_restart/penetration_response.csv")):
        rows = []
        for r in csv.DictReader(open(ref / "results" / name)):
            if r["microstructure"] not in have:
                continue
            row = {k: r[k] for k in ("microstructure", "structure", "transfer_axis")}
            for k, v in r.items():
                if k not in row and k != "retained":
                    row[k] = float(v)
            if "retained" in r:
                row["retained"] = r["retained"] == "True"
            rows.append(row)
        out[key] = rows
    out["source"] = ("results/radiative_properties.csv, results/penetration_response.csv and their "
                     "hit_point_restart/ versions")
    (HERE / "multibounce.json").write_text(json.dumps(out, indent=1))
    print("multibounce rows:", {k: len(v) for k, v in out.items() if k != "source"})


DESCRIPTOR_SMALL = {
    # name: (shape, solid fraction, seed); directional descriptors need every axis >= 128
    "d7x5x6": ((7, 5, 6), 0.40, 1),
    "d9": ((9, 9, 9), 0.20, 2),
    "d1x6x5": ((1, 6, 5), 0.50, 3),
    "d12x3x1": ((12, 3, 1), 0.30, 4),
    "d16": ((16, 16, 16), 0.60, 5),
    "d10": ((10, 10, 10), 0.02, 6),
    "d128_half": ((128, 128, 128), 0.50, 7),
    "d128_sparse": ((128, 128, 128), 0.004, 8),
    "d128_box": ((128, 136, 144), 0.30, 9),
}


def _plain(v):
    if isinstance(v, np.ndarray):
        return v.tolist()
    if isinstance(v, (tuple, list)):
        return [_plain(x) for x in v]
    if isinstance(v, (np.bool_, bool)):
        return bool(v)
    if isinstance(v, (np.integer,)):
        return int(v)
    if isinstance(v, (np.floating,)):
        return float(v)
    return v


def _descriptor_record(dm, ph, directional):
    rec = {"shape": list(ph.shape), "sha256": hashlib.sha256(ph.tobytes()).hexdigest()}
    try:
        rec["scalar"] = {k: _plain(v) for k, v in dm.scalar_descriptors(ph).items()}
    except Exception as e:  # noqa: BLE001 - the reference's own error is the expected outcome
        rec["scalar_error"] = type(e).__name__
    pore = ph == 0
    rec["chords"] = []
    for a in range(3):
        chords, allp, M, N = dm.periodic_chords(pore, a)
        rec["chords"].append({"hist": np.bincount(chords, minlength=N + 1).tolist(), "all_pore": int(allp),
                              "lines": int(M), "N": int(N)})
    rec["interface_face_counts"] = dm.interface_face_counts(~pore).tolist()
    if directional:
        rec["directional"] = [{k: _plain(v) for k, v in row.items()} for row in dm.directional_descriptors(ph)]
    return rec


def descriptor_rows(ref):
    from porerad import descriptors as dm  # noqa: E402

    table = {r["id"]: r for r in csv.DictReader(open(ref / "data" / "microstructures.csv"))}
    stored = {}
    for path in sorted(HERE.glob("canonical_*.npz")):
        name = path.name[len("canonical_"):-4]
        ph = np.load(ref / "data" / "microstructures" / f"{name}.npz")["phases"]
        rec = _descriptor_record(dm, ph, True)
        r = table[name]
        rec["archived"] = {k: (float(r[k]) if k not in ("structure", "set", "medoid") else r[k]) for k in (
            "structure", "set", "N", "target_phi", "realized_phi", "interfacial_area_density_per_cell",
            "mean_beam_length_cells", "mean_pore_chord_x_cells", "mean_pore_chord_y_cells",
            "mean_pore_chord_z_cells", "medoid")}
        stored[name] = rec
    small = {}
    for name, (shape, phi, seed) in DESCRIPTOR_SMALL.items():
        ph = random_phases(shape, phi, seed)
        small[name] = dict(_descriptor_record(dm, ph, min(shape) >= 128), phi=phi, seed=seed)
    for name, value in (("d_solid", 1), ("d_pore", 0)):
        ph = np.full((4, 5, 6), value, np.uint8)
        small[name] = dict(_descriptor_record(dm, ph, False), fill=value)
    (HERE / "descriptors.json").write_text(json.dumps(dict(
        stored=stored, small=small, source="porerad/descriptors.py; data/microstructures.csv"), indent=None))
    print("descriptor records:", len(stored), "stored,", len(small), "small")


def ray_set_comparison_rows(ref):
    rows = []
    for r in csv.DictReader(open(ref / "results" / "coupled_ray_set_comparison.csv")):
        if r["sets_compared"] == "A vs B" and ";" not in r["epsilon"] and r["N_axis"] == "128":
            rows.append(dict(microstructure=r["microstructure"], axis=r["transfer_axis"], T_mean_K=float(r["T_mean_K"]),
                             epsilon=float(r["epsilon"]),
                             max_temperature_difference_K=float(r["max_temperature_difference_K"]),
                             total_flux_rel_difference=float(r["total_flux_rel_difference"])))
    (HERE / "ray_set_comparison.json").write_text(json.dumps(dict(
        rows=rows, source="results/coupled_ray_set_comparison.csv (A vs B, one emissivity, N = 128)"), indent=1))
    print("ray-set comparison rows:", len(rows))


def microstructure_rows(ref):
    rows = []
    for r in csv.DictReader(open(ref / "data" / "microstructures.csv")):
        rows.append(dict(id=r["id"], structure=r["structure"], set=r["set"], N=int(r["N"]),
                         target_phi=float(r["target_phi"]), seed=int(r["seed"]), phase_sha256=r["phase_sha256"]))
    (HERE / "microstructures.json").write_text(json.dumps(dict(rows=rows, source="data/microstructures.csv"),
                                                          indent=1))
    print("microstructure rows:", len(rows))


def count_hash_rows(ref):
    hashes = {}
    for r in csv.DictReader(open(ref / "data" / "cases_coupled.csv")):
        if r["raw_count_sha256_A"]:
            key = f"{r['microstructure']}|{r['transfer_axis']}"
            hashes[key] = dict(microstructure=r["microstructure"], axis=r["transfer_axis"], H_m=float(r["H_m"]),
                               rays_per_patch=int(r["rays_per_patch_per_block"]),
                               seeds_A=[int(s) for s in r["seeds_A"].split(";")],
                               seeds_B=[int(s) for s in r["seeds_B"].split(";")],
                               phase_sha256_x=r["phase_sha256_x"], sha256_A=r["raw_count_sha256_A"],
                               sha256_B=r["raw_count_sha256_B"], source="data/cases_coupled.csv",
                               array="stored" if r["microstructure"] in CANONICAL else "generated")
    (HERE / "count_hashes.json").write_text(json.dumps(hashes, indent=1, sort_keys=True))
    print("hash cases:", len(hashes))


def fullpath_rows(ref):
    """results/fullpath_crosscheck.csv first_hit_radiosity rows, with the reference's recomputation.

    No script of the reference writes these rows and none records their rays.  Stored with them:
    the prescribed-field channels the reference computes from the coupled case's sets A + B (2 + 2
    blocks of 64 rays per patch) on the same microstructure, and the file's full-path Monte Carlo
    rows of that microstructure.
    """

    from porerad import coupled as cp, exchange as ex, view_factors as vf

    cases = {r["case_id"]: r for r in csv.DictReader(open(ref / "data" / "cases_coupled.csv"))}
    rows = []
    table = list(csv.DictReader(open(ref / "results" / "fullpath_crosscheck.csv")))
    for r in table:
        if r["method"] != "first_hit_radiosity":
            continue
        T, dT, eps = float(r["T_mean_K"]), float(r["delta_T_K"]), float(r["epsilon"])
        c = cases[f"coupled_{r['structure']}_{r['transfer_axis']}_T{int(T)}_eps{eps:g}_N128"]
        ph = vf.orient_along_x(np.load(ref / "data" / "microstructures" / f"{r['microstructure']}.npz")["phases"],
                               r["transfer_axis"])
        p = vf.build_surface_patches(ph, float(c["H_m"]))
        seeds = [int(x) for k in ("seeds_A", "seeds_B") for x in c[k].split(";")]
        R = int(c["rays_per_patch_per_block"])
        o, rc, n = vf.pool_counts([vf.first_hit_counts(p, R, sd) for sd in seeds], p.n_patches)
        op = ex.ExchangeOperator(o, rc, n, np.full(p.n_patches, R * len(seeds), np.int64), p.patch_area_m2)
        ch = cp.prescribed_field_channels(op, p, T, dT, eps)
        rows.append(dict(microstructure=r["microstructure"], axis=r["transfer_axis"], H_m=float(c["H_m"]),
                         T_mean_K=T, delta_T_K=dT, epsilon=eps, rays_per_patch=R, seeds=seeds,
                         phase_sha256_x=c["phase_sha256_x"], q_h=float(r["q_h_W_m2"]), q_c=float(r["q_c_W_m2"]),
                         q_i=float(r["q_i_W_m2"]), recomputed=dict(q_h=ch.q_h, q_c=ch.q_c, q_i=ch.q_i),
                         monte_carlo=[{k: float(m[k]) for k in ("q_h_W_m2", "q_c_W_m2", "q_i_W_m2", "q_h_se_W_m2",
                                                                 "q_c_se_W_m2", "q_i_se_W_m2", "histories")}
                                      for m in table if m["method"] == "full_path_monte_carlo"
                                      and m["microstructure"] == r["microstructure"]]))
        print("fullpath", r["microstructure"], ch.q_h, ch.q_c, ch.q_i, "archived", r["q_h_W_m2"], flush=True)
    (HERE / "fullpath.json").write_text(json.dumps(dict(rows=rows, source="results/fullpath_crosscheck.csv, "
                                                                            "data/cases_coupled.csv"), indent=1))


def public_api(ref):
    """Public names of the reference modules on the path, with call signatures.

    A name is public when it does not start with an underscore and is not a module or a helper
    imported from a third-party package or the standard library.
    """

    import importlib
    import inspect
    import types

    out = {}
    for mod_name in ("view_factors", "exchange", "coupled", "conduction"):
        mod = importlib.import_module(f"porerad.{mod_name}")
        names = {}
        for name, obj in sorted(vars(mod).items()):
            if name.startswith("_") or isinstance(obj, types.ModuleType) or name == "annotations":
                continue
            if not getattr(obj, "__module__", "porerad").startswith("porerad"):
                continue  # helpers imported from NumPy, SciPy, Numba or the standard library
            rec = {"kind": "class" if inspect.isclass(obj) else "function" if callable(obj) else "constant"}
            if rec["kind"] == "constant":
                rec["value"] = repr(obj)
            else:
                try:
                    sig = inspect.signature(obj)
                    rec["parameters"] = [[p.name, p.kind.name, None if p.default is p.empty else repr(p.default)]
                                         for p in sig.parameters.values()]
                except (TypeError, ValueError):
                    pass
                if rec["kind"] == "class":
                    rec["members"] = sorted(n for n in vars(obj) if not n.startswith("_"))
            names[name] = rec
        out[mod_name] = names
    (HERE / "public_api.json").write_text(json.dumps(out, indent=1, sort_keys=True))
    print("public api:", {k: len(v) for k, v in out.items()})


PARTS = ("small", "coupled_rows", "prescribed", "multibounce", "descriptors", "microstructures", "ray_sets",
         "count_hashes", "stored_arrays", "fullpath", "public_api")


def main():
    import os

    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("PORERAD_REFERENCE"),
                    help="checkout of moxi000/pore-radiation-ijhmt2026 (default: $PORERAD_REFERENCE)")
    ap.add_argument("--only", default=",".join(PARTS), help="comma-separated parts: " + ", ".join(PARTS))
    args = ap.parse_args()
    if not args.reference:
        ap.error("give --reference or set PORERAD_REFERENCE")
    parts = set(args.only.split(","))
    if parts - set(PARTS):
        ap.error(f"unknown parts {sorted(parts - set(PARTS))}")
    ref = Path(args.reference)
    sys.path.insert(0, str(ref))
    from porerad import coupled as cp, exchange as ex, view_factors as vf  # noqa: E402

    if "small" in parts:
        for name, spec in SMALL_CASES.items():
            small_case(vf, ex, cp, name, spec)
            coupled_small(name, spec)
    steps = dict(coupled_rows=coupled_rows, prescribed=prescribed_cases, multibounce=multibounce_rows,
                 descriptors=descriptor_rows, microstructures=microstructure_rows, ray_sets=ray_set_comparison_rows,
                 count_hashes=count_hash_rows, fullpath=fullpath_rows, public_api=public_api)
    for name, fn in steps.items():
        if name in parts:
            fn(ref)
    if "stored_arrays" not in parts:
        return
    for name in CANONICAL + ["OF_core_phi0.05_s3"]:
        ph = np.load(ref / "data" / "microstructures" / f"{name}.npz")["phases"]
        assert ph.dtype == np.uint8 and set(np.unique(ph)) <= {0, 1}
        np.savez_compressed(HERE / f"canonical_{name}.npz", bits=np.packbits(ph.ravel()),
                            shape=np.asarray(ph.shape, np.int64),
                            sha256=np.bytes_(hashlib.sha256(ph.tobytes()).hexdigest()))

    case = next(r for r in csv.DictReader(open(ref / "data" / "cases_prescribed_field.csv"))
                if r["case_id"] == CORE_CASE)
    res = [r for r in csv.DictReader(open(ref / "results" / "prescribed_field.csv")) if r["case_id"] == CORE_CASE]
    pf = dict(case_id=CORE_CASE, microstructure=case["microstructure"], axis=case["transfer_axis"],
              H_m=float(case["H_m"]), rays_per_patch=int(case["rays_per_patch_per_block"]),
              seeds=[int(s) for k in ("seeds_A", "seeds_B") for s in case[k].split(";")],
              phase_sha256_x=case["phase_sha256_x"], delta_T_K=20.0,
              rows=[dict(T_mean_K=float(r["T_mean_K"]), epsilon=float(r["epsilon"]), q_h=float(r["q_h_W_m2"]),
                         q_c=float(r["q_c_W_m2"]), q_i=float(r["q_i_W_m2"])) for r in res],
              source="data/cases_prescribed_field.csv, results/prescribed_field.csv")
    (HERE / "prescribed_field.json").write_text(json.dumps(pf, indent=1))


if __name__ == "__main__":
    main()

"""The coupled case driver of the reference (scripts/run_coupled.py) on a B200.

``coupled_case`` takes one row of data/cases_coupled.csv and the case's microstructure, and runs
the reference driver's sequence on the device (run_coupled.py:119-158): the phase array
oriented along the transfer axis and repeated, checked against the row's phase hash; surface
patches; every seed block traced once; the counts of sets A and B pooled and compared with the
row's stored count hashes (the comparison is reported, as the reference logs it); the balanced
operator of A + B; the conduction system and its pure-conduction field; the coupled solve, its
wall-flux metrics and the acceptance rules; optionally the solves with sets A and B on their own
and their differences.  The result row has the reference's result columns.
"""

from __future__ import annotations

import hashlib
from dataclasses import dataclass, field

import numpy as np

from . import conduction, coupled, view_factors as vf
from .constants import K_GAS, K_SOLID
from .ray_sets import RaySets

COUPLED_COLUMNS = [
    "case_id", "group", "structure", "microstructure", "transfer_axis", "H_m", "N_axis", "T_mean_K", "delta_T_K",
    "epsilon", "q_cond_hot_W_m2", "q_rad_hot_W_m2", "q_total_hot_W_m2", "q_cond_cold_W_m2", "q_rad_cold_W_m2",
    "q_total_cold_W_m2", "radiative_fraction_hot", "k_eff_apparent_W_mK", "wall_flux_mismatch_rel",
    "energy_residual_rel", "newton_updates", "T_min_K", "T_max_K",
]
"""The columns of results/coupled.csv (run_coupled.py:32-38)."""


@dataclass
class CoupledCase:
    row: dict
    count_hashes: dict                      # set name -> stored hash reproduced (True/False); absent if none stored
    result: coupled.CoupledResult = field(repr=False)
    metrics: dict = field(repr=False)
    ab: dict | None = None                  # largest temperature and relative total-flux differences of A and B


def _seeds(v) -> list[int]:
    return [int(s) for s in v.split(";")] if isinstance(v, str) else [int(s) for s in v]


def _solve(system, operator, patches, T_hot, T_cold, epsilon, T_initial):
    """Coupled solve, metrics and acceptance (run_coupled.py:98-111); RuntimeError when not accepted."""

    result = coupled.solve_coupled(system, operator, patches, T_hot, T_cold, epsilon, T_initial)
    metrics = coupled.wall_flux_metrics(system, patches, result, T_hot, T_cold)
    failures = coupled.acceptance_failures(result, metrics)
    if result.failure:
        failures.insert(0, result.failure)
    if failures:
        raise RuntimeError("solution not accepted: " + "; ".join(failures))
    return result, metrics


def coupled_case(case: dict, phases: np.ndarray, *, ab: bool = False) -> CoupledCase:
    """One coupled case (run_coupled.py:114-158); ``case`` holds the row's columns of
    data/cases_coupled.csv, ``phases`` the microstructure as stored (not yet oriented)."""

    axis, H, eps = case["transfer_axis"], float(case["H_m"]), float(case["epsilon"])
    T_mean, delta_T = float(case["T_mean_K"]), float(case["delta_T_K"])
    T_hot, T_cold = T_mean + delta_T / 2.0, T_mean - delta_T / 2.0
    rpp = int(case["rays_per_patch_per_block"])
    seeds = {name: _seeds(case[f"seeds_{name}"]) for name in ("A", "B")}

    ph = vf.orient_along_x(np.asarray(phases, dtype=np.uint8), axis)
    ph = np.ascontiguousarray(np.concatenate([ph] * int(case.get("repeats_along_axis", 1)), axis=0))
    if ph.shape[0] != int(case["N_axis"]):
        raise ValueError(f"microstructure has {ph.shape[0]} cells along the transfer axis")
    if case.get("phase_sha256_x") and hashlib.sha256(ph.tobytes()).hexdigest() != case["phase_sha256_x"]:
        raise ValueError("phase array differs from the one listed for this case")
    patches = vf.build_surface_patches(ph, H)
    sets = RaySets(patches, rpp)
    ops = []
    try:
        hashes = {}
        for name in ("A", "B"):
            expected = case.get(f"raw_count_sha256_{name}", "")
            if expected:
                hashes[name] = sets.pooled(seeds[name]).sha256() == expected
        final = sets.operator(seeds["A"] + seeds["B"])
        ops.append(final)
        system = conduction.assemble_conduction(np.where(ph == 1, K_SOLID, K_GAS), H)
        try:
            T_initial = conduction.solve_conduction(system, T_hot, T_cold)
            result, metrics = _solve(system, final, patches, T_hot, T_cold, eps, T_initial)
            row = {key: case[key] for key in ("case_id", "group", "structure", "microstructure", "transfer_axis",
                                              "H_m", "N_axis", "T_mean_K", "delta_T_K", "epsilon") if key in case}
            row.update({key: metrics[key] for key in COUPLED_COLUMNS if key in metrics})
            row["newton_updates"] = result.newton_iterations
            out = CoupledCase(row, hashes, result, metrics)
            if ab:
                solved = {}
                for name in ("A", "B"):
                    op = sets.operator(seeds[name])
                    ops.append(op)
                    solved[name] = _solve(system, op, patches, T_hot, T_cold, eps, T_initial)
                (ra, ma), (rb, mb) = solved["A"], solved["B"]
                out.ab = {"max_temperature_difference_K": float(np.max(np.abs(ra.temperature_K - rb.temperature_K))),
                          "total_flux_rel_difference": coupled.relative_difference(ma["q_total_hot_W_m2"],
                                                                                   mb["q_total_hot_W_m2"])}
            return out
        finally:
            system.close()
    finally:
        for op in ops:
            op.close()
        sets.close()

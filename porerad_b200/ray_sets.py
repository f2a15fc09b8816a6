"""Ray sets of a prescribed-field case on a B200: A/B sets, the append rule, pooled operators.

Mirrors the ray-set logic of the reference's case driver
(scripts/run_prescribed_field.py:78-160): each ray block (one PCG64 seed) is traced once
into a device count table; a set is the pool of its blocks (device merges of the tables);
the operator of a set is built from the pooled table without a host round trip.  With the
A/B comparison, both sets are evaluated on their own, their wall-channel and coarse-source
differences decide one symmetric append of a further block to each set
(coupled.py:197-219), and the final operator pools every block used.
"""

from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from . import coupled, exchange, view_factors as vf

DELTA_T_K = 20.0
"""Wall temperature difference of the prescribed-field cases (run_prescribed_field.py:31)."""

CLOSURE_LIMIT = 1.0e-4
"""Largest accepted channel imbalance |q_h + q_c + q_i| / max|q| (run_prescribed_field.py:146-147)."""


class RaySets:
    """Count tables of the ray blocks of one geometry, traced once each, pooled on demand."""

    def __init__(self, patches, rays_per_patch: int):
        self.patches = patches
        self.rays_per_patch = int(rays_per_patch)
        self._blocks: dict[int, vf.CountTable] = {}
        self.traced: list[int] = []

    def block(self, seed: int) -> vf.CountTable:
        seed = int(seed)
        if seed not in self._blocks:
            self._blocks[seed] = vf.first_hit_counts_pooled(self.patches, self.rays_per_patch, [seed])
            self.traced.append(seed)
        return self._blocks[seed]

    def pooled(self, seeds) -> vf.CountTable:
        """Counts of the given blocks pooled (view_factors.py:290-300), on the device."""

        seeds = [int(s) for s in seeds]
        table = self.block(seeds[0])
        owned = False
        for s in seeds[1:]:
            merged = table.merge(self.block(s))
            if owned:
                table.close()
            table, owned = merged, True
        return table

    def operator(self, seeds) -> exchange.ExchangeOperator:
        """Projected operator of the given blocks (run_prescribed_field.py:78-92)."""

        table = self.pooled(seeds)
        n = self.patches.n_patches
        rays = np.full(n, self.rays_per_patch * len(list(seeds)), dtype=np.int64)
        return exchange.ExchangeOperator(table, None, None, rays, np.asarray(self.patches.patch_area_m2))

    def close(self) -> None:
        for t in self._blocks.values():
            t.close()
        self._blocks.clear()


def channels(operator, patches, conditions, delta_T_K: float = DELTA_T_K) -> list[coupled.PrescribedChannels]:
    """Prescribed-field channels at every condition (T_mean, eps) (run_prescribed_field.py:95-96)."""

    return [coupled.prescribed_field_channels(operator, patches, float(T), float(delta_T_K), float(eps))
            for T, eps in conditions]


@dataclass
class CaseResult:
    """Rows of one case (the columns of results/prescribed_field.csv) and its ray-set record."""

    rows: list[dict]
    append: bool
    ab_channel_difference: float | None = None
    ab_source_difference: float | None = None
    append_rule: bool | None = None
    seeds_used: list[int] = field(default_factory=list)


def prescribed_field_case(phases_x, H_m: float, rays_per_patch: int, seeds_A, seeds_B, append_seeds_A,
                          append_seeds_B, append_used: bool, conditions, *, ab: bool = True,
                          delta_T_K: float = DELTA_T_K) -> CaseResult:
    """One prescribed-field case end to end (run_prescribed_field.py:99-160).

    ``ab=True`` evaluates sets A and B on their own and applies the append rule to their
    difference (the rule's decision is used where it differs from ``append_used``, as the
    reference does); the reported A/B difference is that of the appended sets when an
    append is made.  ``RuntimeError`` when a channel balance exceeds 1e-4.
    """

    patches = vf.build_surface_patches(phases_x, H_m)
    sets = RaySets(patches, rays_per_patch)
    seeds_A, seeds_B = [int(s) for s in seeds_A], [int(s) for s in seeds_B]
    app_A, app_B = [int(s) for s in append_seeds_A], [int(s) for s in append_seeds_B]
    append = bool(append_used)
    out = CaseResult([], append)
    ops = []
    try:
        ab_difference = ""
        if ab:
            def set_channels(seeds):
                op = sets.operator(seeds)
                ops.append(op)
                return channels(op, patches, conditions, delta_T_K)

            ch_a, ch_b = set_channels(seeds_A), set_channels(seeds_B)
            channel, source = coupled.ab_differences(ch_a, ch_b)
            rule = coupled.append_required(channel, source)
            out.append_rule = rule
            append = rule
            if append:
                ch_a, ch_b = set_channels(seeds_A + app_A), set_channels(seeds_B + app_B)
                channel, source = coupled.ab_differences(ch_a, ch_b)
            out.ab_channel_difference, out.ab_source_difference = channel, source
            ab_difference = channel
        final_seeds = seeds_A + seeds_B + (app_A + app_B if append else [])
        final = sets.operator(final_seeds)
        ops.append(final)
        for res in channels(final, patches, conditions, delta_T_K):
            if res.closure_rel > CLOSURE_LIMIT:
                raise RuntimeError(f"channel balance not closed: {res.closure_rel:.2e}")
            out.rows.append({"T_mean_K": res.T_mean_K, "delta_T_K": float(delta_T_K), "epsilon": res.epsilon,
                             "q_h_W_m2": res.q_h, "q_c_W_m2": res.q_c, "q_i_W_m2": res.q_i,
                             "ab_wall_channel_rel_difference": ab_difference})
        out.append = append
        out.seeds_used = list(sets.traced)
        return out
    finally:
        for op in ops:
            op.close()
        sets.close()

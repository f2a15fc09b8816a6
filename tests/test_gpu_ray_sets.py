"""GPU parity of the prescribed-field case flow: A/B sets, the append rule and the final operator.

Every case of data/cases_prescribed_field.csv is run through ``ray_sets.prescribed_field_case``
with the A/B comparison (the reference's ``--ab`` flow) and compared with its archived rows of
results/prescribed_field.csv: q_h, q_c and q_i of every condition to 1e-9 of the largest
channel (the operator's scale is pinned only to the balancing tolerance), the recorded A/B
wall-channel difference to 1e-6 relative, and the append decision of the case table (one case,
pf_TL_core_phi0.10_s0_y, appends a block to each set).
"""

from __future__ import annotations

import hashlib

import numpy as np
import pytest

from tests.helpers import load_canonical, prescribed_cases

pytestmark = pytest.mark.gpu

FLUX_RTOL = 1e-9
AB_RTOL = 1e-6


@pytest.mark.parametrize("case_id", [c["case_id"] for c in prescribed_cases()])
def test_archived_prescribed_field_case(case_id):
    from porerad_b200 import ray_sets, view_factors as vf

    case = next(c for c in prescribed_cases() if c["case_id"] == case_id)
    ph = vf.orient_along_x(load_canonical(case["microstructure"]), case["axis"])
    assert hashlib.sha256(np.ascontiguousarray(ph).tobytes()).hexdigest() == case["phase_sha256_x"]
    res = ray_sets.prescribed_field_case(ph, case["H_m"], case["rays_per_patch"], case["seeds_A"], case["seeds_B"],
                                         case["append_seeds_A"], case["append_seeds_B"], case["append_used"],
                                         case["conditions"], ab=True, delta_T_K=case["delta_T_K"])
    assert res.append == case["append_used"] and res.append_rule == case["append_used"]
    want_ab = case["ab_wall_channel_rel_difference"]
    assert abs(res.ab_channel_difference - want_ab) <= AB_RTOL * want_ab
    assert len(res.rows) == len(case["rows"])
    for got, want in zip(res.rows, case["rows"]):
        assert (got["T_mean_K"], got["epsilon"]) == (want["T_mean_K"], want["epsilon"])
        scale = max(abs(want["q_h"]), abs(want["q_c"]), abs(want["q_i"]))
        for k in ("q_h", "q_c", "q_i"):
            assert abs(got[k + "_W_m2"] - want[k]) <= FLUX_RTOL * scale, (k, got[k + "_W_m2"], want[k])
    n_blocks = len(case["seeds_A"]) + len(case["seeds_B"])
    if case["append_used"]:
        n_blocks += len(case["append_seeds_A"]) + len(case["append_seeds_B"])
    assert len(res.seeds_used) == n_blocks  # every block traced once

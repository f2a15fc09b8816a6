"""The generator oracle (oracle/generators.py) against the archived phase_sha256 column of
data/microstructures.csv, on a sample covering every structure and set (CPU)."""

from __future__ import annotations

import hashlib
import json

import pytest

from oracle import generators as og
from tests.helpers import GOLDEN

ROWS = {r["id"]: r for r in json.loads((GOLDEN / "microstructures.json").read_text())["rows"]}
SAMPLE = ["FI_core_phi0.10_s0", "FA_core_phi0.05_s2", "TL_core_phi0.15_s1", "FA_matched_pair3", "FI_matched_pair1",
          "TL_canonical_phi0.10_N128", "FI_canonical_phi0.10_N160", "OF_core_phi0.05_s0"]


@pytest.mark.parametrize("mid", SAMPLE)
def test_oracle_generator(mid):
    r = ROWS[mid]
    if r["set"] == "core":
        ph = og.build(r["structure"], r["N"], r["target_phi"], r["seed"])
    elif r["set"] == "canonical":
        ph = og.canonical(r["structure"], r["N"])
    else:
        ph = og.matched(r["structure"], int(mid[-1]))
    assert hashlib.sha256(ph.tobytes()).hexdigest() == r["phase_sha256"]

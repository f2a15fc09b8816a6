"""Fixture loaders shared by the tests (golden vectors made by tests/golden/make_golden.py)."""

from __future__ import annotations

import hashlib
import json
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[1]
GOLDEN = ROOT / "tests" / "golden"

SMALL = ["box12", "cube20", "slab16"]


def load_small(name: str) -> dict:
    with np.load(GOLDEN / f"small_{name}.npz") as z:
        return {k: z[k] for k in z.files}


def load_canonical(name: str) -> np.ndarray:
    with np.load(GOLDEN / f"canonical_{name}.npz") as z:
        shape = tuple(int(s) for s in z["shape"])
        ph = np.unpackbits(z["bits"])[: int(np.prod(shape))].reshape(shape).astype(np.uint8)
        assert hashlib.sha256(ph.tobytes()).hexdigest() == z["sha256"].item().decode()
    return ph


def count_hash_cases(array: str | None = None) -> dict:
    """Stored count hashes of data/cases_coupled.csv; ``array`` selects "stored" or "generated" rows."""

    rows = json.loads((GOLDEN / "count_hashes.json").read_text())
    return {k: v for k, v in rows.items() if array is None or v.get("array", "stored") == array}


def case_phases(name: str) -> np.ndarray:
    """Phases of an archived microstructure: the stored fixture, or (N = 160 and 192 canonical arrays,
    which are not stored) the device generators' rebuild; callers check the archived phase hash."""

    if (GOLDEN / f"canonical_{name}.npz").is_file():
        return load_canonical(name)
    structure, kind, _, n = name.split("_")
    if kind != "canonical" or not n.startswith("N"):
        raise FileNotFoundError(f"no stored array and no generator rule for {name}")
    from porerad_b200 import geometry

    return geometry.canonical(structure, int(n[1:]))


def prescribed_case() -> dict:
    return json.loads((GOLDEN / "prescribed_field.json").read_text())


def load_coupled(name: str) -> dict:
    """Coupled-solve golden of a small case (tests/golden/make_golden.py)."""

    with np.load(GOLDEN / f"coupled_{name}.npz") as z:
        return {k: z[k] for k in z.files}


def coupled_rows() -> list[dict]:
    """Archived results/coupled.csv rows of the canonical microstructures with their case parameters."""

    return json.loads((GOLDEN / "coupled.json").read_text())["rows"]


def prescribed_cases() -> list[dict]:
    """All 48 prescribed-field cases with their archived rows (tests/golden/make_golden.py)."""

    return json.loads((GOLDEN / "prescribed_cases.json").read_text())["cases"]


def multibounce_rows() -> dict:
    """Archived properties and penetration rows of the stored microstructures (tests/golden/make_golden.py)."""

    return json.loads((GOLDEN / "multibounce.json").read_text())


def descriptor_records() -> dict:
    """porerad.descriptors outputs stored by make_golden.descriptor_rows."""

    return json.loads((GOLDEN / "descriptors.json").read_text())


def random_phases(shape, phi, seed) -> np.ndarray:
    """The seeded phase arrays of make_golden.random_phases (same generator and threshold)."""

    rng = np.random.default_rng(seed)
    field = rng.random(shape)
    field = (field + np.roll(field, 1, axis=0) + np.roll(field, 1, axis=2)) / 3.0
    thr = np.quantile(field, phi)
    return (field < thr).astype(np.uint8)


def descriptor_phases(name: str, rec: dict) -> np.ndarray:
    """Phase array of a descriptor record: a stored microstructure, a seeded array or a uniform one."""

    if "fill" in rec:
        ph = np.full(tuple(rec["shape"]), rec["fill"], np.uint8)
    elif "seed" in rec:
        ph = random_phases(tuple(rec["shape"]), rec["phi"], rec["seed"])
    else:
        ph = load_canonical(name)
    assert hashlib.sha256(ph.tobytes()).hexdigest() == rec["sha256"]
    return ph

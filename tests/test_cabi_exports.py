"""The C-ABI library loads and exports every entry point include/porerad.h declares (no GPU needed)."""

from __future__ import annotations

import ctypes
import re

from tests.helpers import ROOT


def _declared() -> list[str]:
    text = (ROOT / "include" / "porerad.h").read_text()
    return re.findall(r"^PR_API\s+[\w\s\*]*?\b(pr_\w+)\(", text, flags=re.M)


def test_library_exports_every_declared_symbol():
    from porerad_b200 import _lib, build

    build.build()
    names = _declared()
    assert len(names) >= 20
    lib = ctypes.CDLL(str(_lib.LIB_PATH))
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert set(_lib._SIGNATURES) <= set(names)


def test_binding_loads_and_reports_version():
    from porerad_b200 import _lib

    assert _lib.load().pr_version() == 1


def test_null_arguments_are_errors_not_crashes():
    from porerad_b200 import _lib

    lib = _lib.load()
    out = ctypes.c_void_p()
    assert lib.pr_case_create(None, 4, 4, 4, 0.01, None, ctypes.byref(out)) == _lib.PR_ERR_ARG
    assert "phases_x" in _lib.last_error()
    assert lib.pr_counts_from_edges(None, None, None, 5, 3, None, ctypes.byref(out)) == _lib.PR_ERR_ARG
    assert lib.pr_operator_apply(None, 0, None, None, None) == _lib.PR_ERR_ARG


def test_widened_entry_points_reject_bad_arguments():
    """Descriptors, generators, archetypes and multi-bounce entry points: invalid arguments give
    PR_ERR_ARG and a message, before any device work (no GPU needed)."""

    from porerad_b200 import _lib

    lib = _lib.load()
    ERR = _lib.PR_ERR_ARG
    m = _lib.Morphology()
    ph = (ctypes.c_uint8 * 8)()
    assert lib.pr_morphology_counts(None, 2, 2, 2, 0, ctypes.byref(m), None, None, None, None) == ERR
    assert lib.pr_morphology_counts(ph, 2, 0, 2, 0, ctypes.byref(m), None, None, None, None) == ERR
    assert "empty" in _lib.last_error()
    assert lib.pr_morphology_counts(ph, 2, 2, 2, 8, ctypes.byref(m), None, None, None, None) == ERR
    assert "flags" in _lib.last_error()
    solid = ctypes.c_int64()
    assert lib.pr_render_shapes(0, None, 0, ph, ctypes.byref(solid), None) == ERR
    assert lib.pr_render_shapes(2000, None, 0, ph, ctypes.byref(solid), None) == ERR
    assert "1..1290" in _lib.last_error()
    assert lib.pr_render_shapes(8, None, -1, ph, ctypes.byref(solid), None) == ERR
    starts = (ctypes.c_int64 * 2)(0, 0)
    assert lib.pr_stamp_cells(8, None, starts, None, starts, 1, 0, 300, ph, None, None) == ERR
    assert "byte" in _lib.last_error()
    assert lib.pr_stamp_fibers(8, None, None, None, None, 1, 0, ph, None, None) == ERR
    seeds = (ctypes.c_double * 6)()
    assert lib.pr_voronoi_edge_field(8, seeds, 2, seeds, None) == ERR
    assert "n_seeds" in _lib.last_error()
    assert lib.pr_quantile_threshold(seeds, 6, 1.5, 1, ph, None, None, None) == ERR
    assert "quantile" in _lib.last_error()
    assert lib.pr_lamellar_field(8, None, seeds, seeds, 1.0, 1.0, seeds, seeds, None) == ERR
    new = (ctypes.c_int64 * 2)()
    assert lib.pr_stamp_first(8, None, starts, None, 0, 2000, 0, ph, None, new, None) == ERR
    assert "n_fibers" in _lib.last_error()
    assert lib.pr_first_threshold(ph, 8, 0, 2, ph, None) == ERR
    assert "mode" in _lib.last_error()
    tally = _lib.PropertiesTally()
    assert lib.pr_radiative_properties(None, 0.5, 10, 1, 0, 10, ctypes.byref(tally), None) == ERR
    counts = (ctypes.c_int64 * 4)()
    assert lib.pr_penetration(None, 0.5, 10, 1, 0, 10, counts, None) == ERR

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

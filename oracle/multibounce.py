"""ORACLE — test infrastructure only.

Python side of oracle/multibounce.c (the CPU restatement of porerad's property and
penetration ray kernels): one run of n rays of one seed on a solid-along-x grid, returning the
tallies of ``trace_properties`` (properties.py:56-279) or the counts of ``trace_penetration``
(penetration.py:281-305).
"""

from __future__ import annotations

import ctypes

import numpy as np

from . import build as _build

_LIB = None


def _lib():
    global _LIB
    if _LIB is None:
        _build.build()
        lib = ctypes.CDLL(str(_build.HERE / "liboracle_mb.so"))
        lib.oracle_multibounce.restype = None
        lib.oracle_multibounce.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                           ctypes.c_longlong, ctypes.c_uint32, ctypes.c_double, ctypes.c_int,
                                           ctypes.c_int, ctypes.c_int, ctypes.c_void_p]
        _LIB = lib
    return _LIB


def run(solid_x: np.ndarray, epsilon: float, n_rays: int, seed: int, *, penetration: bool,
        restart: str = "article", max_bounces: int = 1000) -> np.ndarray:
    """The 8 tallies (properties) or the 4 counts R, T, A, stopped (penetration)."""

    s = np.ascontiguousarray(np.asarray(solid_x) != 0, dtype=np.uint8)
    out = np.zeros(8)
    _lib().oracle_multibounce(s.ctypes.data, s.shape[0], s.shape[1], s.shape[2], int(n_rays),
                              int(seed) & 0xFFFFFFFF, float(epsilon), int(max_bounces),
                              int(restart == "hit_point"), int(penetration), out.ctypes.data)
    return out[:4].astype(np.int64) if penetration else out

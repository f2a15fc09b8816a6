"""The radius bisection of porerad_b200.generators (geometry.py:124-145) against the oracle's, on a
CPU stand-in for the device renderer: the same radii visited, the same one kept (no GPU needed)."""

from __future__ import annotations

import numpy as np
import pytest

from oracle import generators as og
from porerad_b200 import generators as gen


class _Phases:
    """What the device renderer hands back: an array with numel() and clone()."""

    def __init__(self, a):
        self.a = a

    def numel(self):
        return self.a.size

    def clone(self):
        return _Phases(self.a.copy())


@pytest.mark.parametrize("target,lo,hi,tol,max_iter", [(0.10, 0.1, 4.0, 3e-3, 24), (0.1, 0.12, 7.0, 5e-4, 32),
                                                        (0.05, 0.2, 4.0, 3e-3, 24), (0.999, 0.1, 4.0, 1e-9, 10)])
def test_bisection_matches_oracle(target, lo, hi, tol, max_iter):
    field = np.random.default_rng(7).random((24, 24, 24))
    buf = np.zeros(field.shape, np.uint8)
    seen_ours, seen_oracle = [], []

    def render_ours(r):  # in-place like the device renderer (one reused array)
        seen_ours.append(r)
        buf[...] = field < r / 4.0
        return _Phases(buf), int(buf.sum())

    def render_oracle(r):
        seen_oracle.append(r)
        return (field < r / 4.0).astype(np.uint8)

    r, ph = gen.bisect_radius(render_ours, target, lo, hi, tol=tol, max_iter=max_iter)
    want = og.bisect(render_oracle, target, lo, hi, tol=tol, max_iter=max_iter)
    assert seen_ours == seen_oracle
    assert np.array_equal(ph.a, want)

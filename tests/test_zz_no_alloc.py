"""pr_reflection_series_noalloc: the reflection series for callers that cannot allocate device memory.

Some hosts cannot call cudaMalloc while they run the radiosity solve, for example a
process whose device memory is reserved by another framework's allocator, or a caller
that must not take the allocator's implicit synchronisation mid-stream.  This entry
point keeps its scratch in a static device array of the library (at most 262144
patches) and must give the same absorbed power as pr_reflection_series.  The file
sorts last so that a run stopping at the first failure has run every other test.
"""

from __future__ import annotations

import ctypes

import numpy as np
import pytest

from tests.helpers import load_small

pytestmark = pytest.mark.gpu

RTOL = 1e-12  # same kernels as pr_reflection_series; only the scratch location differs


def _entry(lib):
    fn = lib.pr_reflection_series_noalloc
    fn.restype = ctypes.c_int
    fn.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_double, ctypes.c_int64,
                   ctypes.c_void_p, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int64),
                   ctypes.c_void_p]
    return fn


def test_noalloc_series_matches_allocating_entry_point_twice():
    import torch

    from porerad_b200 import _lib, exchange

    case = load_small("cube20")
    n = case["patches_patch_class"].size
    R = int(case["rays_per_patch"]) * len(case["seeds"])
    area = case["patches_patch_area_m2"]
    op = exchange.ExchangeOperator(case["pooled_origin"], case["pooled_receiver"], case["pooled_count"],
                                   np.full(n, R, np.int64), area)
    fn = _entry(_lib.load())
    rng = np.random.default_rng(11)
    dev = torch.cuda.current_device()
    for call in range(2):
        emitted = rng.standard_normal(n) * 1e-6
        eps = 0.3 + 0.6 * rng.random(n)
        want = exchange.reflection_series(op, emitted, eps, relative_tolerance=1e-13)
        d_e = torch.tensor(emitted, dtype=torch.float64, device="cuda")
        d_eps = torch.tensor(eps, dtype=torch.float64, device="cuda")
        d_out = torch.full((n,), float("nan"), dtype=torch.float64, device="cuda")
        res, it = ctypes.c_double(), ctypes.c_int64()
        torch.cuda.synchronize()
        before = (_lib.memory_stats(dev), torch.cuda.memory_allocated(dev))
        status = fn(op.handle, d_e.data_ptr(), d_eps.data_ptr(), 1e-13, 10000, d_out.data_ptr(), ctypes.byref(res),
                    ctypes.byref(it), None)
        assert status == _lib.PR_OK, _lib.last_error()
        torch.cuda.synchronize()
        after = (_lib.memory_stats(dev), torch.cuda.memory_allocated(dev))
        # nothing allocated: no driver allocation, no block taken from the library's cache, no
        # torch allocation, and the library's live and cached bytes unchanged
        assert after == before, (before, after)
        got = d_out.cpu().numpy()
        scale = float(np.max(np.abs(want.absorbed_power_W)))
        assert float(np.max(np.abs(got - want.absorbed_power_W))) <= RTOL * scale, f"call {call}"
        assert int(it.value) == want.iterations
        assert abs(res.value - want.residual_power_W) <= RTOL * float(np.sum(np.abs(emitted)))


def test_noalloc_series_rejects_oversized_operator_and_host_memory():
    import torch

    from porerad_b200 import _lib, exchange

    # 300000 patches that each see only themselves: F = I balances at once
    n = 300_000
    ids = np.arange(n, dtype=np.int32)
    op = exchange.ExchangeOperator(ids, ids, np.ones(n, np.int64), np.ones(n, np.int64), np.full(n, 1e-8))
    fn = _entry(_lib.load())
    d = torch.zeros(n, dtype=torch.float64, device="cuda")
    res, it = ctypes.c_double(), ctypes.c_int64()
    status = fn(op.handle, d.data_ptr(), d.data_ptr(), 1e-13, 100, d.data_ptr(), ctypes.byref(res),
                ctypes.byref(it), None)
    assert status == _lib.PR_ERR_LIMIT
    assert "262144" in _lib.last_error()

    case = load_small("box12")
    m = case["patches_patch_class"].size
    small = exchange.ExchangeOperator(case["pooled_origin"], case["pooled_receiver"], case["pooled_count"],
                                      np.full(m, int(case["rays_per_patch"]) * 2, np.int64),
                                      case["patches_patch_area_m2"])
    host = np.zeros(m)
    status = fn(small.handle, host.ctypes.data, host.ctypes.data, 1e-13, 100, host.ctypes.data, ctypes.byref(res),
                ctypes.byref(it), None)
    assert status == _lib.PR_ERR_ARG
    assert "device memory" in _lib.last_error()

"""Served path on the GPU: concurrent cases give the same results as the same cases alone."""

from __future__ import annotations

import numpy as np
import pytest

from tests.helpers import SMALL, load_small

pytestmark = pytest.mark.gpu


def _requests():
    from porerad_b200 import geometry, serving

    reqs = []
    for k, name in enumerate(SMALL):
        case = load_small(name)
        reqs.append(serving.CaseRequest(case["phases"], float(case["H_m"]), int(case["rays_per_patch"]),
                                        [int(s) for s in case["seeds"]], 700.0, 20.0, 0.6, tag=name))
    for k, arch in enumerate(geometry.ARCHETYPES):
        ph = geometry.make(arch, 32, 0.12, k)
        reqs.append(serving.CaseRequest(ph, 0.005, 48, [k + 1, k + 101], 600.0 + 50 * k, 100.0, 0.3 + 0.15 * k,
                                        precision="mixed" if k % 2 else "fp64", tag=arch))
    return reqs


def test_results_same_alone_and_in_the_mix():
    from porerad_b200 import serving

    reqs = _requests()
    alone = {}
    with serving.Server(slots=1) as srv:
        for r in reqs:
            res = srv.submit(r).result(timeout=300)
            alone[res.tag] = res
    with serving.Server(slots=4) as srv:
        futs = [srv.submit(r) for r in reqs]
        mixed = {f.result(timeout=300).tag: f.result() for f in futs}
    assert set(mixed) == set(alone)
    for tag, a in alone.items():
        m = mixed[tag]
        assert (m.q_h, m.q_c, m.q_i) == (a.q_h, a.q_c, a.q_i), tag
        assert np.array_equal(m.coarse_source, a.coarse_source), tag
        assert m.pairs == a.pairs and m.n_patches == a.n_patches
        assert m.closure_rel <= 1e-8
    slots_used = {f.result().slot for f in futs}
    assert len(slots_used) > 1


def test_repeated_case_reuses_cached_device_memory():
    """A repeated case takes every buffer from the library's cache and gives the same bits."""

    import torch

    from porerad_b200 import _lib, serving

    req = _requests()[-1]
    adm = serving.Admission(1 << 40)
    first = serving.run_case(req, adm)
    torch.cuda.synchronize()
    before = _lib.memory_stats(torch.cuda.current_device())
    again = serving.run_case(req, adm)
    torch.cuda.synchronize()
    after = _lib.memory_stats(torch.cuda.current_device())
    assert after["device_mallocs"] == before["device_mallocs"]
    assert after["cache_hits"] > before["cache_hits"]
    assert after["live_bytes"] == before["live_bytes"]
    assert (again.q_h, again.q_c, again.q_i) == (first.q_h, first.q_c, first.q_i)
    assert np.array_equal(again.coarse_source, first.coarse_source)
    _lib.release_cached_memory(torch.cuda.current_device())
    assert _lib.memory_stats(torch.cuda.current_device())["cached_bytes"] == 0

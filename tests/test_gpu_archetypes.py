"""Benchmark archetypes generated on the device (geometry.make_device) equal their host
definitions (geometry.make) bit for bit, and serving requests may carry a generator spec."""

from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CASES = [("OF", 48, 0.10, 1), ("OF", 128, 0.10, 1), ("OF", 64, 0.20, 7), ("FI", 64, 0.10, 0), ("FI", 96, 0.15, 3),
         ("FA", 64, 0.10, 2), ("FA", 48, 0.05, 5), ("TL", 64, 0.10, 4), ("TL", 96, 0.20, 9), ("FI", 16, 0.0, 1)]


@pytest.mark.parametrize("arch,n,phi,seed", CASES)
def test_device_archetype_equals_host(arch, n, phi, seed):
    from porerad_b200 import geometry

    dev = geometry.make_device(arch, n, phi, seed)
    assert dev.is_cuda and tuple(dev.shape) == (n, n, n)
    assert np.array_equal(dev.cpu().numpy(), geometry.make(arch, n, phi, seed))


def test_serving_from_spec():
    from porerad_b200 import geometry, serving

    spec = serving.GeometrySpec("FA", 48, 0.10, 2, axis="z")
    host = np.ascontiguousarray(np.moveaxis(geometry.make("FA", 48, 0.10, 2), 2, 0))
    reqs = [serving.CaseRequest(p, 0.01, 16, [5], 700.0, 20.0, 0.6, precision="fp64", tag=k)
            for k, p in enumerate((spec, host))]
    with serving.Server(slots=2) as srv:
        a, b = [f.result() for f in [srv.submit(r) for r in reqs]]
    assert (a.q_h, a.q_c, a.q_i, a.n_patches) == (b.q_h, b.q_c, b.q_i, b.n_patches)

"""GPU parity on the benchmark workloads themselves, against the oracle on the same seeded inputs.

* FI 64^3, phi 0.10, 64 rays per patch, one set (the small plain case): the whole case.  The
  count hash equals the oracle's; the binary64 channels agree with the oracle's binary64
  channels to 1e-9 and the mixed-precision channels (binary32 sweeps in binary64 refinement)
  to 1e-8 relative.
* OF 128^3, 1000 rays per patch, sets A and B (the headline case), and TL and FA 192^3, 1000
  rays per patch, sets A, B and C (the coupled-size stress case): the full count tables of every
  set are made on the device (up to 1.1e9 rays per set); the rows of three origin-patch slices
  (first, middle and last patches) equal the oracle's counts of the same slices bit for bit.
  The oracle draws the rays of a slice from the same PCG64 stream position as a full pass
  (view_factors.py:149-151), so a slice checks the full-size tables without tracing them on the
  CPU.  The slices of each workload hold 2-3 x 10^4 rays whose azimuth sine or cosine differs by
  one ulp from glibc's; an equal count table shows that none of them changed a receiver.
"""

from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FLUX_RTOL = 1e-9    # binary64 channels: both sides balance d to 1e-11 (d agrees to about 1e-8 relative)
MIXED_RTOL = 1e-8   # mixed-precision channels against the oracle's binary64 channels

C1 = dict(arch="FI", n=64, phi=0.10, seed=0, rays=64, sets=1, eps=0.9, T_m=650.0, dT=100.0, H=0.01)
SLICED = {
    "OF128-c2": (dict(arch="OF", n=128, phi=0.10, seed=1, rays=1000, sets=2, H=0.01), 4096),
    "TL192-c5": (dict(arch="TL", n=192, phi=0.10, seed=0, rays=1000, sets=3, H=0.01), 2048),
    "FA192-c5": (dict(arch="FA", n=192, phi=0.10, seed=0, ray_seed=7919, rays=1000, sets=3, H=0.01), 2048),
}


def _seeds(spec):
    """The ray-set seeds the benchmark draws for a case (SplitMix64 of its case seed and set index)."""

    from porerad_b200.geometry import ray_set_seed

    return [ray_set_seed(spec.get("ray_seed", spec["seed"]), s) for s in range(spec["sets"])]


def test_small_plain_case_whole_path_against_oracle(oracle):
    from porerad_b200 import coupled, exchange, geometry, view_factors as vf

    s = C1
    ph = geometry.make(s["arch"], s["n"], s["phi"], s["seed"])
    seeds = _seeds(s)
    p = vf.build_surface_patches(ph, s["H"])
    q = oracle.build_surface_patches(ph, s["H"])
    assert p.n_patches == q.n_patches
    table = vf.first_hit_counts_pooled(p, s["rays"], seeds)
    pooled = oracle.pool_counts([oracle.first_hit_counts(q, s["rays"], sd) for sd in seeds], q.n_patches)
    rays = np.full(q.n_patches, s["rays"] * len(seeds), np.int64)
    assert table.rays_traced == int(rays.sum())
    assert table.sha256() == oracle.count_sha256(*pooled, rays)

    op = exchange.ExchangeOperator(table, None, None, rays, p.patch_area_m2)
    ref_op = oracle.ExchangeOperator(*pooled, rays, q.patch_area_m2)
    want = oracle.prescribed_field_channels(ref_op, q, s["T_m"], s["dT"], s["eps"])
    got = coupled.prescribed_field_channels(op, p, s["T_m"], s["dT"], s["eps"])
    mixed = coupled.prescribed_field_channels(op, p, s["T_m"], s["dT"], s["eps"], precision="mixed")
    scale = max(abs(want.q_h), abs(want.q_c), abs(want.q_i))
    for name in ("q_h", "q_c", "q_i"):
        assert abs(getattr(got, name) - getattr(want, name)) <= FLUX_RTOL * scale, name
    for name in ("q_h", "q_c"):
        assert abs(getattr(mixed, name) - getattr(want, name)) <= MIXED_RTOL * abs(getattr(want, name)), name
    assert abs(mixed.q_i - want.q_i) <= MIXED_RTOL * scale
    assert float(np.sum(np.abs(got.coarse_source - want.coarse_source))) <= \
        FLUX_RTOL * float(np.sum(np.abs(want.coarse_source)))
    op.close()
    table.close()


@pytest.mark.parametrize("name", sorted(SLICED))
def test_full_size_count_rows_on_patch_slices(oracle, name):
    from porerad_b200 import geometry, view_factors as vf

    s, width = SLICED[name]
    ph = geometry.make(s["arch"], s["n"], s["phi"], s["seed"])
    p = vf.build_surface_patches(ph, s["H"])
    q = oracle.build_surface_patches(ph, s["H"])
    P = p.n_patches
    assert P == q.n_patches and P >= 3 * width
    slices = [(0, width), (P // 2, P // 2 + width), (P - width, P)]
    for sd in _seeds(s):
        table = vf.first_hit_counts_pooled(p, s["rays"], [sd])
        assert table.rays_traced == P * s["rays"]
        for b, e in slices:
            got = table.rows(b, e)
            want = oracle.first_hit_counts(q, s["rays"], sd, patch_start=b, patch_end=e)
            assert int(got[2].sum()) == (e - b) * s["rays"]
            for g, w, field in zip(got, want, ("origin", "receiver", "count")):
                assert g.dtype == w.dtype and np.array_equal(g, w), (name, sd, b, field)
        table.close()


def test_count_rows_edges_and_errors():
    """Row ranges: empty, a single row, the whole table (equal to the full copy), out of range."""

    from porerad_b200 import view_factors as vf
    from tests.helpers import load_small

    case = load_small("cube20")
    p = vf.build_surface_patches(case["phases"], float(case["H_m"]))
    table = vf.first_hit_counts_pooled(p, int(case["rays_per_patch"]), [int(x) for x in case["seeds"]])
    full = table.to_numpy()
    n = table.n_patches
    for got, want in zip(table.rows(0, n), full):
        assert np.array_equal(got, want)
    assert all(a.size == 0 for a in table.rows(5, 5))
    o, r, c = table.rows(7, 8)
    sel = full[0] == 7
    assert np.array_equal(o, full[0][sel]) and np.array_equal(r, full[1][sel]) and np.array_equal(c, full[2][sel])
    for b, e in ((-1, 3), (3, n + 1), (4, 3)):
        with pytest.raises(ValueError, match="row range"):
            table.rows(b, e)
    table.close()


def test_large_count_copies_to_pageable_and_pinned_memory_agree():
    """Count arrays above 16 MB copied into pageable NumPy memory (pinned staging buffers, host
    threads), into the library's pinned host blocks (to_numpy) and into pinned torch memory are
    equal; so are the row ranges."""

    import torch

    from porerad_b200 import _lib, view_factors as vf
    from tests.helpers import load_canonical

    p = vf.build_surface_patches(load_canonical("FA_canonical_phi0.10_N128"), 0.01)
    table = vf.first_hit_counts_pooled(p, 64, [11, 12])
    m = table.nnz
    assert m * 4 > (16 << 20)
    import gc

    gc.collect()  # arrays of earlier tests give their blocks back; the cache is then emptied
    vf.release_host_blocks(0)
    o, r, c = table.to_numpy()  # views of a newly pinned block
    assert o.base is not None and vf.host_blocks_stats()["live_bytes"] >= 16 * m
    assert o.size == m and o.dtype == np.int32 and r.dtype == np.int32 and c.dtype == np.int64
    assert o.flags.writeable and o.flags.c_contiguous and c.flags.aligned
    lib = _lib.load()
    pageable = [np.empty(m, np.int32), np.empty(m, np.int32), np.empty(m, np.int64)]
    _lib.check(lib.pr_counts_copy(table.handle, *[a.ctypes.data for a in pageable], None, _lib.stream()))
    pinned = [torch.empty(m, dtype=dt).pin_memory() for dt in (torch.int32, torch.int32, torch.int64)]
    _lib.check(lib.pr_counts_copy(table.handle, *[t.data_ptr() for t in pinned], None, _lib.stream()))
    for got, a, t in zip((o, r, c), pageable, pinned):
        assert np.array_equal(got, a) and np.array_equal(got, t.numpy())
    b = table.n_patches // 3
    sel = o >= b
    for got, want in zip(table.rows(b, table.n_patches), (o, r, c)):
        assert np.array_equal(got, want[sel])
    rows_pageable = [np.empty(int(sel.sum()), dt) for dt in (np.int32, np.int32, np.int64)]
    n = _lib.ctypes.c_int64()
    _lib.check(lib.pr_counts_rows(table.handle, b, table.n_patches, _lib.ctypes.byref(n),
                                  *[a.ctypes.data for a in rows_pageable], _lib.stream()))
    for got, want in zip(rows_pageable, (o, r, c)):
        assert np.array_equal(got, want[sel])
    table.close()


def test_host_blocks_are_reused_and_checked():
    """Released pinned blocks are cached and handed out again; foreign or released pointers are
    refused; trimming frees the cache."""

    import gc

    from porerad_b200 import _lib, view_factors as vf

    lib = _lib.load()
    gc.collect()  # arrays of earlier tests give their blocks back before the baseline is read
    vf.release_host_blocks(0)
    s0 = vf.host_blocks_stats()
    o, r, c = vf._edge_arrays(3 << 20)  # 48 MiB: a newly pinned block
    o[:] = 1
    c[:] = -5
    r[-1] = 7
    assert int(o.sum()) == 3 << 20 and int(c[0]) == -5 and int(r[-1]) == 7
    s1 = vf.host_blocks_stats()
    assert s1["allocations"] == s0["allocations"] + 1 and s1["live_bytes"] >= 48 << 20
    del o, r, c
    gc.collect()
    s2 = vf.host_blocks_stats()
    assert s2["live_bytes"] == s0["live_bytes"] and s2["cached_bytes"] >= 48 << 20
    o, r, c = vf._edge_arrays((3 << 20) - 1000)  # fits the cached block: reused, no new allocation
    s3 = vf.host_blocks_stats()
    assert s3["allocations"] == s1["allocations"] and s3["reuses"] == s2["reuses"] + 1
    x = np.empty(16, np.int64)
    assert lib.pr_host_block_release(_lib.ctypes.c_void_p(x.ctypes.data)) == _lib.PR_ERR_ARG
    blk = _lib.ctypes.c_void_p()
    _lib.check(lib.pr_host_block(1 << 20, _lib.ctypes.byref(blk)))
    _lib.check(lib.pr_host_block_release(blk))
    assert lib.pr_host_block_release(blk) == _lib.PR_ERR_ARG  # released twice
    del o, r, c
    gc.collect()
    vf.release_host_blocks(0)
    assert vf.host_blocks_stats()["cached_bytes"] == 0
    small = vf._edge_arrays(1000)  # small edge lists stay ordinary NumPy memory
    assert all(a.base is None for a in small)


def test_pool_counts_of_large_tables_from_pinned_pageable_and_int64_inputs():
    """pool_counts over per-set tables above 16 MB equals the device-pooled table whether the
    tables sit in the library's pinned blocks (first_hit_counts' results), in pageable NumPy
    memory (staged copies) or hold int64 ids; ids outside the patches raise IndexError."""

    from porerad_b200 import view_factors as vf
    from tests.helpers import load_canonical

    p = vf.build_surface_patches(load_canonical("FA_canonical_phi0.10_N128"), 0.01)
    P = p.n_patches
    a0 = vf.first_hit_counts(p, 64, 11)
    b = vf.first_hit_counts(p, 64, 12)
    a = vf.first_hit_counts(p, 64, 11)  # pinned block views
    assert a[0].nbytes > (16 << 20) and a[0].base is not None
    assert all(np.array_equal(x, y) for x, y in zip(a, a0))
    want = vf.first_hit_counts_pooled(p, 64, [11, 12])
    w = want.to_numpy()
    want.close()
    pageable = [tuple(np.array(x, copy=True) for x in t) for t in (a, b)]
    wide = [(t[0].astype(np.int64), t[1].astype(np.int64), t[2]) for t in (a, b)]
    for tables in ([a, b], pageable, wide, [pageable[0], b]):
        got = vf.pool_counts(tables, P)
        for g, x in zip(got, w):
            assert g.dtype == x.dtype and np.array_equal(g, x)
    for dt in (np.int32, np.int64):
        bad = (pageable[0][0].astype(dt), pageable[0][1].astype(dt), pageable[0][2])
        bad[1][12345] = P
        with pytest.raises(IndexError):
            vf.pool_counts([bad, b], P)
    assert all(x.size == 0 for x in vf.pool_counts([], P))


def test_first_hit_counts_host_pass_equals_the_device_table():
    """Above 16 MB first_hit_counts writes the sorted list into a pinned host block chunk by
    chunk (64 M rays each) while later chunks trace; the arrays equal the device table's copy,
    with one chunk (64 rays per patch) and with three (1000 rays per patch: 1.96e8 rays)."""

    from porerad_b200 import view_factors as vf
    from tests.helpers import load_canonical

    p = vf.build_surface_patches(load_canonical("FA_canonical_phi0.10_N128"), 0.01)
    P = p.n_patches
    for R in (64, 1000):
        got = vf.first_hit_counts(p, R, 11)
        assert got[0].base is not None  # views of the pass's pinned block
        t = vf.first_hit_counts_pooled(p, R, [11])
        want = t.to_numpy()
        t.close()
        for g, w in zip(got, want):
            assert g.dtype == w.dtype and g.flags.c_contiguous and np.array_equal(g, w)
        assert int(got[2].sum()) == P * R
        if R == 1000:
            assert P * R > 2 * (1 << 26)  # three chunks of at most 2^26 rays

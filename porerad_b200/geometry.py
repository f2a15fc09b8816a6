"""Seeded synthetic voxel microstructures of the four benchmark archetypes (uint8, 1 = solid).

These are the workload inputs of the benchmark and tests, defined on the host with
NumPy from an integer seed (``make``) and generated bit for bit on the device for
serving (``make_device``).  They follow the archetype definitions of the benchmark
configurations; the reference's own generators (porerad/geometry.py) are re-exported
at the end of this module from ``porerad_b200.generators``:

* FI: isotropic random-axis solid cylinders of radius r placed until the solid
  fraction reaches phi;
* FA: cylinders of radius r aligned with z, placed until phi;
* OF: open-cell foam, struts along the edges of the periodic Voronoi tessellation of
  64 Poisson seed points, dilated until phi;
* TL: tortuous layers, 4-voxel-thick sheets normal to z perforated by random
  8-voxel holes, holes added until phi.

Every field is periodic in y and z (and x) so any axis can be the transfer axis.
"""

from __future__ import annotations

import numpy as np

ARCHETYPES = ("OF", "FI", "FA", "TL")


def _ball(radius: float) -> np.ndarray:
    r = int(np.ceil(radius))
    g = np.arange(-r, r + 1)
    dx, dy, dz = np.meshgrid(g, g, g, indexing="ij")
    keep = dx * dx + dy * dy + dz * dz <= radius * radius
    return np.stack((dx[keep], dy[keep], dz[keep]), axis=1)


def _segment_points(p0: np.ndarray, direction: np.ndarray, length: float) -> np.ndarray:
    """Lattice points along a segment every quarter cell (with repeats)."""

    t = np.arange(-length / 2.0, length / 2.0 + 0.25, 0.25)
    return np.rint(p0[None, :] + t[:, None] * direction[None, :]).astype(np.int64)


def _segment_centres(p0: np.ndarray, direction: np.ndarray, length: float) -> np.ndarray:
    return np.unique(_segment_points(p0, direction, length), axis=0)


def _stamp_segment(solid: np.ndarray, p0: np.ndarray, direction: np.ndarray, length: float, ball: np.ndarray) -> None:
    n = np.asarray(solid.shape)
    centres = _segment_centres(p0, direction, length)
    pts = (centres[:, None, :] + ball[None, :, :]).reshape(-1, 3) % n
    solid[pts[:, 0], pts[:, 1], pts[:, 2]] = 1


def fibers(n: int, phi: float, seed: int, *, radius: float = 2.0, aligned: bool = False) -> np.ndarray:
    """FI (isotropic axes) or FA (axes along z) cylinders of the given radius until phi is reached."""

    rng = np.random.default_rng(seed)
    solid = np.zeros((n, n, n), np.uint8)
    ball = _ball(radius)
    target = phi * solid.size
    count = 0
    while count < target:
        p0, d, length = _fiber_draws(n, rng, aligned)
        _stamp_segment(solid, p0, d, length, ball)
        count = int(solid.sum())
    return solid


def foam(n: int, phi: float, seed: int, *, n_seeds: int = 64) -> np.ndarray:
    """OF: struts on the edges of a periodic Voronoi tessellation, thickened until phi.

    A voxel belongs to a Voronoi edge where its three nearest seeds are nearly
    equidistant; the strut field d3 - d1 (distance to the third minus the first
    nearest seed) is thresholded at the phi-quantile.
    """

    from scipy.spatial import cKDTree

    rng = np.random.default_rng(seed)
    pts = rng.random((n_seeds, 3)) * n
    tree = cKDTree(pts, boxsize=n)
    g = np.arange(n) + 0.5
    cx, cy, cz = np.meshgrid(g, g, g, indexing="ij")
    centres = np.stack((cx.ravel(), cy.ravel(), cz.ravel()), axis=1)
    dist, _ = tree.query(centres, k=3)
    field = (dist[:, 2] - dist[:, 0]).reshape(n, n, n)
    thr = np.quantile(field, phi)
    return (field <= thr).astype(np.uint8)


def layers(n: int, phi: float, seed: int, *, thickness: int = 4, hole: int = 8) -> np.ndarray:
    """TL: sheets normal to z, evenly spaced from a random offset, perforated by random holes until phi."""

    rng = np.random.default_rng(seed)
    solid = np.zeros((n, n, n), np.uint8)
    m = max(1, int(np.ceil(phi * n / thickness)))
    offset = int(rng.integers(0, n))
    for s in range(m):
        z0 = (offset + (s * n) // m) % n
        for dz in range(thickness):
            solid[:, :, (z0 + dz) % n] = 1
    target = phi * solid.size
    r = hole / 2.0
    g = np.arange(-hole, hole + 1)
    dx, dy = np.meshgrid(g, g, indexing="ij")
    disk = np.stack((dx[dx * dx + dy * dy <= r * r], dy[dx * dx + dy * dy <= r * r]), axis=1)
    sheet_z = [(offset + (s * n) // m) % n for s in range(m)]
    while solid.sum() > target:
        z0 = sheet_z[int(rng.integers(0, m))]
        c = rng.integers(0, n, size=2)
        xy = (c[None, :] + disk) % n
        for dz in range(thickness):
            solid[xy[:, 0], xy[:, 1], (z0 + dz) % n] = 0
    return solid


def _fiber_draws(n: int, rng, aligned: bool):
    p0 = rng.random(3) * n
    if aligned:
        return p0, np.array([0.0, 0.0, 1.0]), float(n)
    v = rng.standard_normal(3)
    return p0, v / np.linalg.norm(v), float(n) * np.sqrt(3.0)


def _layer_sheets(n: int, phi: float, thickness: int, offset: int):
    m = max(1, int(np.ceil(phi * n / thickness)))
    return m, [(offset + (s * n) // m) % n for s in range(m)]


def _hole_disk(hole: int) -> np.ndarray:
    r = hole / 2.0
    g = np.arange(-hole, hole + 1)
    dx, dy = np.meshgrid(g, g, indexing="ij")
    keep = dx * dx + dy * dy <= r * r
    return np.stack((dx[keep], dy[keep]), axis=1)


def make_device(archetype: str, n: int, phi: float, seed: int, *, stream=None):
    """``make(archetype, n, phi, seed)`` generated on the device: a uint8 CUDA tensor equal to the
    host array bit for bit.  The random draws stay on the host (the same NumPy generator calls);
    the grid work runs in libporerad: fiber segments in batches, each cell keeping the first fiber
    that covers it (``pr_stamp_first``, ``pr_first_threshold``), hole stamping with solid counts
    (``pr_stamp_cells``), the foam's nearest-seed field (``pr_voronoi_edge_field``) and its quantile
    threshold (``pr_quantile_threshold``)."""

    import ctypes

    import torch

    from . import _lib

    lib = _lib.load()
    st = _lib.stream() if stream is None else _lib.stream_arg(stream)
    n = int(n)
    out = torch.empty((n, n, n), dtype=torch.uint8, device="cuda")
    solid = ctypes.c_int64()
    start = np.array([0, 1], np.int64)

    def count_below(count, target):  # the host loop's condition `while count < target`
        return count < target

    def stamp(nodes, offsets, value, clear):
        nd = np.ascontiguousarray(nodes, dtype=np.int32)
        od = np.ascontiguousarray(offsets, dtype=np.int32)
        ns = np.array([0, len(nd)], np.int64)
        os_ = np.array([0, len(od)], np.int64)
        _lib.check(lib.pr_stamp_cells(n, nd.ctypes.data, ns.ctypes.data, od.ctypes.data, os_.ctypes.data, 1,
                                      int(clear), int(value), out.data_ptr(), ctypes.byref(solid), st))
        return int(solid.value)

    if archetype in ("FI", "FA"):
        # the host loop adds one fiber until the solid reaches phi n^3; here batches of fibers are
        # stamped at once, every cell keeping the first fiber that covers it, and the cells each
        # fiber adds tell where the loop stops (the same union; draws past it are discarded)
        rng = np.random.default_rng(seed)
        ball = np.ascontiguousarray(_ball(2.0), dtype=np.int32)
        target = phi * n ** 3
        if not count_below(0, target):
            out.zero_()
            torch.cuda.current_stream().synchronize()
            return out
        first = torch.full((n, n, n), np.iinfo(np.int32).max, dtype=torch.int32, device="cuda")
        torch.cuda.current_stream().synchronize()
        batch, base, count, last = 64, 0, 0, -1
        while last < 0:
            # stamping is idempotent: the segment's lattice points need no deduplication here
            nodes = [_segment_points(*_fiber_draws(n, rng, archetype == "FA")) % n for _ in range(batch)]
            node_start = np.zeros(batch + 1, np.int64)
            node_start[1:] = np.cumsum([len(a) for a in nodes])
            nd = np.ascontiguousarray(np.concatenate(nodes), dtype=np.int32)
            new = np.zeros(batch, np.int64)
            _lib.check(lib.pr_stamp_first(n, nd.ctypes.data, node_start.ctypes.data, ball.ctypes.data, len(ball),
                                          batch, base, first.data_ptr(), None, new.ctypes.data, st))
            for f in range(batch):
                count += int(new[f])
                if not count_below(count, target):
                    last = base + f
                    break
            base += batch
        _lib.check(lib.pr_first_threshold(first.data_ptr(), n ** 3, last, 0, out.data_ptr(), st))
        return out
    if archetype == "OF":
        rng = np.random.default_rng(seed)
        pts = np.ascontiguousarray(rng.random((64, 3)) * n)
        field = torch.empty((n, n, n), dtype=torch.float64, device="cuda")
        _lib.check(lib.pr_voronoi_edge_field(n, pts.ctypes.data, 64, field.data_ptr(), st))
        _lib.check(lib.pr_quantile_threshold(field.data_ptr(), n ** 3, float(phi), 1, out.data_ptr(), None, None, st))
        return out
    if archetype == "TL":
        thickness, hole = 4, 8
        rng = np.random.default_rng(seed)
        offset = int(rng.integers(0, n))
        m, sheet_z = _layer_sheets(n, phi, thickness, offset)
        planes = np.array([(0, 0, (z0 + dz) % n) for z0 in sheet_z for dz in range(thickness)], np.int64)
        g = np.arange(n)
        plane_offsets = np.stack([a.ravel() for a in np.meshgrid(g, g, [0], indexing="ij")], axis=1)
        count = stamp(planes, plane_offsets, 1, True)
        disk = _hole_disk(hole)
        hole_offsets = np.ascontiguousarray([(dx, dy, dz) for dz in range(thickness) for dx, dy in disk],
                                            dtype=np.int32)
        target = phi * n ** 3
        if not count > target:  # the host loop's condition `while solid.sum() > target`
            return out
        # holes in batches: each cell keeps the first hole covering it, the solid cells each hole
        # removes tell where the host loop stops, and the cells up to that hole are cleared
        first = torch.full((n, n, n), np.iinfo(np.int32).max, dtype=torch.int32, device="cuda")
        torch.cuda.current_stream().synchronize()
        batch, base, last = 64, 0, -1
        node_start = np.arange(batch + 1, dtype=np.int64)
        while last < 0:
            centres = []
            for _ in range(batch):
                z0 = sheet_z[int(rng.integers(0, m))]
                c = rng.integers(0, n, size=2)
                centres.append((c[0], c[1], z0))
            nd = np.ascontiguousarray(centres, dtype=np.int32)
            removed = np.zeros(batch, np.int64)
            _lib.check(lib.pr_stamp_first(n, nd.ctypes.data, node_start.ctypes.data, hole_offsets.ctypes.data,
                                          len(hole_offsets), batch, base, first.data_ptr(), out.data_ptr(),
                                          removed.ctypes.data, st))
            for f in range(batch):
                count -= int(removed[f])
                if not count > target:
                    last = base + f
                    break
            base += batch
        _lib.check(lib.pr_first_threshold(first.data_ptr(), n ** 3, last, 1, out.data_ptr(), st))
        return out
    raise ValueError(f"unknown archetype {archetype!r}; expected one of {ARCHETYPES}")


def make(archetype: str, n: int, phi: float, seed: int) -> np.ndarray:
    """One archetype microstructure of size n^3 (uint8, 1 = solid)."""

    if archetype == "FI":
        return fibers(n, phi, seed)
    if archetype == "FA":
        return fibers(n, phi, seed, aligned=True)
    if archetype == "OF":
        return foam(n, phi, seed)
    if archetype == "TL":
        return layers(n, phi, seed)
    raise ValueError(f"unknown archetype {archetype!r}; expected one of {ARCHETYPES}")


def splitmix64(x: int) -> int:
    """SplitMix64 finaliser: 64-bit ray-set seeds derived from a case seed."""

    x = (x + 0x9E3779B97F4A7C15) & 0xFFFFFFFFFFFFFFFF
    x = ((x ^ (x >> 30)) * 0xBF58476D1CE4E5B9) & 0xFFFFFFFFFFFFFFFF
    x = ((x ^ (x >> 27)) * 0x94D049BB133111EB) & 0xFFFFFFFFFFFFFFFF
    return x ^ (x >> 31)


def ray_set_seed(case_seed: int, set_index: int, block: int = 0) -> int:
    """Seed of ray block ``block`` of ray set ``set_index`` (0 = A, 1 = B, ...) of a case (below 2^63)."""

    return splitmix64(splitmix64(splitmix64(int(case_seed)) ^ int(set_index)) ^ int(block)) >> 1


# The reference's own generators (porerad/geometry.py), rendered on the device: the module is a
# drop-in for porerad.geometry as well as the home of the benchmark archetypes above.
from .generators import (  # noqa: E402,F401
    CORE_N, CORE_PHIS, FA_THETA_SIGMA, FIBER_LENGTH, FIBER_LINES, FOAM_NEIGHBOURS, FOAM_NODES, MATCHED_PAIRS,
    MIN_PORE_CLUSTER, NODE_TO_STRUT, PHI_TOL, STRUCTURES, TL_BASE_N, TL_LAYERS, TL_NOISE, accepted, build, canonical,
    core_library, core_realizations, fiber_lines, foam_graph, lamellar_field, matched, render_fibers, render_foam, shape_mask,
    threshold)

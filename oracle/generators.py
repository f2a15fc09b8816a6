"""ORACLE — test infrastructure only.

CPU restatement of porerad's microstructure generators (porerad/geometry.py), the checker of
``porerad_b200.generators`` and the CPU leg of ``bench.py``'s generators workload.  Every
shape is evaluated over the whole periodic grid with NumPy, as the reference does; the foam
graph uses ``scipy.spatial.cKDTree`` and the TL resampling ``scipy.ndimage.zoom``, the
libraries the reference calls.  Pinned by tests/test_oracle_generators.py to the
``phase_sha256`` column of data/microstructures.csv (tests/golden/microstructures.json).
"""

from __future__ import annotations

import math

import numpy as np

PHI_TOL = 3e-3  # geometry.py:23
FIBERS = {"FI": {0.05: 6, 0.10: 10, 0.15: 14}, "FA": {0.05: 6, 0.10: 12, 0.15: 18}}  # geometry.py:26
LENGTH = {"FI": 9.0, "FA": 10.0}  # geometry.py:27
NODES = {0.05: 24, 0.10: 32, 0.15: 42}  # geometry.py:29
LAYERS = {0.05: 9, 0.10: 7, 0.15: 9}  # geometry.py:32
PAIRS = {1: {"FA": (7, 40), "FI": (0, 12)}, 2: {"FA": (6, 52), "FI": (8, 14)}, 3: {"FA": (2, 32), "FI": (4, 6)}}
E = np.eye(3)


def _mm(a, b):
    with np.errstate(all="ignore"):
        return a @ b


def frame(z, helper):  # geometry.py:49-56
    if abs(float(np.dot(helper, z))) > 0.9:
        helper = E[1]
    x = np.cross(helper, z)
    x /= np.linalg.norm(x)
    return np.stack([x, np.cross(z, x), z], axis=1)


def local_coordinates(N, center, R):
    """R^T times the minimum-image offsets of every cell from center (geometry.py:108-114)."""
    half = float(N) / 2.0
    g = [(np.arange(N).reshape([-1 if a == b else 1 for b in range(3)]) - center[a] + half) % float(N) - half
         for a in range(3)]
    g = np.broadcast_arrays(*g)
    return [v.reshape((N,) * 3) for v in _mm(R.T, np.stack([v.ravel() for v in g], axis=0))]


def long_cylinder(N, r, half_length, R, center=(0.0, 0.0, 0.0)):  # geometry.py:59-82
    axis = _mm(R, E[2])
    axis /= float(np.linalg.norm(axis))
    steps = max(1, int(math.ceil(2.0 * half_length)))
    t = np.arange(steps, dtype=float) - steps / 2.0
    nodes = np.unique(np.rint(t[:, None] * axis[None, :] + np.asarray(center, float)[None, :]).astype(np.int64) % N,
                      axis=0)
    Rq = frame(axis / float(np.linalg.norm(axis)), E[0])
    pad = int(math.ceil(r)) + 2
    g = np.arange(-pad, pad + 1, dtype=np.int64)
    off = np.stack([a.ravel() for a in np.meshgrid(g, g, g, indexing="ij")], axis=1)
    loc = _mm(Rq.T, off.T.astype(float)).T
    disk = ((loc[:, 0] / r) ** 2 + (loc[:, 1] / r) ** 2 <= 1.0 + 1e-12) & (np.abs(loc[:, 2]) <= 0.5 + 1e-12)
    idx = (nodes[:, None, :] + off[disk][None, :, :]) % N
    m = np.zeros(N ** 3, bool)
    m[((idx[..., 0] * N + idx[..., 1]) * N + idx[..., 2]).ravel()] = True
    return m.reshape((N,) * 3)


def shape_mask(N, center, radii, kind, R):  # geometry.py:85-121
    rx, ry, rz = radii
    if kind == "cylinder" and float(2.0 * rz) > float(N):
        ci = tuple(int(round(c)) % N for c in center)
        if any(abs(c - float(i)) > 1e-9 for c, i in zip(center, ci)):
            return long_cylinder(N, rx, rz, R, center)
        return np.roll(long_cylinder(N, rx, rz, R), shift=ci, axis=(0, 1, 2))
    xl, yl, zl = local_coordinates(N, center, R)
    if kind == "ellipsoid":
        return (xl / rx) ** 2 + (yl / ry) ** 2 + (zl / rz) ** 2 <= 1.0
    return ((xl / rx) ** 2 + (yl / ry) ** 2 <= 1.0) & (np.abs(zl) <= rz)


def bisect(render, target, lo, hi, tol=PHI_TOL, max_iter=24):  # geometry.py:124-145
    best = None
    for _ in range(max_iter):
        mid = 0.5 * (lo + hi)
        ph = render(mid)
        phi = float(np.mean(ph == 1))
        err = abs(phi - float(target))
        if best is None or err < best[0]:
            best = (err, ph)
        if err <= tol:
            break
        lo, hi = (mid, hi) if phi < float(target) else (lo, mid)
    return best[1]


def fiber_axis(rng, aligned):  # geometry.py:150-156
    if aligned:
        theta = rng.normal(0.0, 0.05)
        az = rng.uniform(0.0, 2.0 * math.pi)
        return np.array([math.cos(theta), math.sin(theta) * math.cos(az), math.sin(theta) * math.sin(az)])
    return rng.normal(size=3)


def fibers(N, centers, rotations, r, length_factor):  # geometry.py:178-184
    ph = np.zeros((N,) * 3, np.uint8)
    for c, R in zip(centers, rotations):
        ph[shape_mask(N, c, (r, r, 0.5 * float(length_factor) * N), "cylinder", R)] = 1
    return ph


def fiber_params(N, seed, n, aligned, continuous):  # geometry.py:159-175
    rng = np.random.default_rng(int(seed))
    centers, rots = [], []
    for _ in range(n):
        c = rng.random(3) * float(N) if continuous else rng.integers(0, N, size=3)
        centers.append(tuple(float(v) for v in c))
        v = fiber_axis(rng, aligned)
        if not aligned:
            v = v / np.linalg.norm(v)
        rots.append(frame(v / np.linalg.norm(v), E[2]))
    return centers, rots


def foam(N, seed, n_nodes, r):  # geometry.py:189-218
    from scipy.spatial import cKDTree

    rng = np.random.default_rng(int(seed))
    pts = rng.uniform(0, N, size=(n_nodes, 3))
    _, nn = cKDTree(pts, boxsize=N).query(pts, k=4)
    edges = sorted({tuple(sorted((int(i), int(j)))) for i, row in enumerate(nn) for j in row[1:] if int(i) != int(j)})
    ph = np.zeros((N,) * 3, np.uint8)
    for p in pts:
        ph[shape_mask(N, tuple(p.tolist()), (1.2 * r,) * 3, "ellipsoid", E)] = 1
    for a, b in edges:
        vec = pts[b] - pts[a]
        for d in range(3):
            if vec[d] > N / 2:
                vec[d] -= N
            elif vec[d] < -N / 2:
                vec[d] += N
        L = float(np.linalg.norm(vec))
        ph[shape_mask(N, tuple((pts[a] + 0.5 * vec) % N), (r, r, 0.5 * L), "cylinder", frame(vec / L, E[2]))] = 1
    return ph


def layered_field(N, seed, n_layers, waviness, noise=0.12):  # geometry.py:223-239
    rng = np.random.default_rng(int(seed))
    x = np.arange(N, dtype=float)[:, None, None]
    y = np.arange(N, dtype=float)[None, :, None]
    z = np.arange(N, dtype=float)[None, None, :]
    base = np.cos(2.0 * np.pi * n_layers * x / float(N))
    p1, p2 = rng.uniform(0.0, 2 * np.pi), rng.uniform(0.0, 2 * np.pi)
    wav = float(waviness) * (0.65 * np.sin(2 * np.pi * y / float(N) + p1) + 0.35 * np.cos(4 * np.pi * z / float(N) + p2))
    field = base + 0.35 * np.sin(2 * np.pi * n_layers * (x + wav) / float(N))
    w = rng.normal(scale=float(noise), size=(N, N, N))
    w = (w + np.roll(w, 1, 0) + np.roll(w, -1, 0) + np.roll(w, 1, 1) + np.roll(w, -1, 1) + np.roll(w, 1, 2)
         + np.roll(w, -1, 2)) / 7.0
    return field + w


def threshold(field, phi):  # geometry.py:242-245
    return (field >= np.quantile(field.ravel(), 1.0 - float(phi))).astype(np.uint8)


def build(structure, N, target_phi, seed, continuous=False):  # geometry.py:250-258
    phi = round(float(target_phi), 2)
    if structure in ("FI", "FA"):
        c, R = fiber_params(N, seed, FIBERS[structure][phi], structure == "FA", continuous)
        return bisect(lambda r: fibers(N, c, R, r, LENGTH[structure]), target_phi, 0.1, 4.0)
    if structure == "OF":
        s = max(1.0, float(N) / 48.0)
        return bisect(lambda r: foam(N, seed, NODES[phi], r), target_phi, 0.2 * s, 4.0 * s)
    if structure == "TL":
        return threshold(layered_field(N, seed, LAYERS[phi], 1.4 + 3.0 * float(target_phi)), target_phi)
    raise ValueError(structure)


def canonical(structure, N):  # geometry.py:299-314
    if structure == "TL":
        from scipy.ndimage import zoom

        f = layered_field(192, 0, LAYERS[0.10], 1.4 + 3.0 * 0.10)
        if N != 192:
            f = zoom(f, float(N) / 192.0, order=3, mode="grid-wrap", grid_mode=True, prefilter=True)
        return threshold(f, 0.10)
    return build(structure, N, 0.10, 0, continuous=True)


def matched(structure, pair, N=128):  # geometry.py:317-333
    seed, n = PAIRS[pair][structure]
    aligned = structure == "FA"
    centers = [tuple(float(v) for v in c) for c in (np.random.default_rng(seed + 1000003).random((64, 3)) * N)[:n]]
    rng = np.random.default_rng(seed + (3000003 if aligned else 2000003))
    rots = []
    for _ in range(n):
        v = fiber_axis(rng, aligned)
        rots.append(frame(v / np.linalg.norm(v), E[2]))
    return bisect(lambda r: fibers(N, centers, rots, r, 9.0), 0.1, 0.12, 7.0, tol=5e-4, max_iter=32)

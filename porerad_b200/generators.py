"""The reference's digital microstructures (porerad/geometry.py), rendered on a B200.

OF open-cell foam, FI random fibers, FA fibers aligned with x, TL tortuous layered, on a
periodic N x N x N grid (axis 0 = x; uint8, 1 = solid).  The solid fraction is set by bisection
on the strut or fiber radius (OF, FI, FA) or by a quantile threshold of a continuous field (TL).

Where the work is:

* the random parameters (fiber centres and axes, foam nodes), the foam graph (periodic
  k-nearest neighbours) and each shape's frame are drawn on the host exactly as the reference
  draws them: the same NumPy generator calls and the same float operations;
* every rendering of a trial radius runs on the device: foam nodes and struts by
  ``pr_render_shapes`` (cell for cell as the reference's shape test evaluates), fibers by
  ``pr_stamp_fibers`` (lattice nodes along the axis thickened by a one-cell disk); the solid
  count of each trial comes back for the bisection; acceptance uses the device descriptors;
* TL's normal draws and its per-axis sines and cosines are host NumPy calls as in the
  reference; the N^3 field (the wavy layers with a correctly rounded sine, the 7-point smoothing
  of the noise) and its quantile threshold are device work (``pr_lamellar_field``,
  ``pr_quantile_threshold``).  Where the canonical TL is resampled to N = 128 or 160 by SciPy's
  periodic cubic splines, the field stays a host array.

The arithmetic that must equal the reference's to reproduce its arrays bit for bit (frames,
strut vectors, node rounding, disk offsets) follows geometry.py operation for operation.
"""

from __future__ import annotations

import ctypes
import math

import numpy as np

from . import _lib

STRUCTURES = ("OF", "FI", "FA", "TL")
CORE_N = 128
CORE_PHIS = (0.05, 0.10, 0.15)
PHI_TOL = 3e-3
MIN_PORE_CLUSTER = 0.99

FIBER_LINES = {"FI": {0.05: 6, 0.10: 10, 0.15: 14}, "FA": {0.05: 6, 0.10: 12, 0.15: 18}}
FIBER_LENGTH = {"FI": 9.0, "FA": 10.0}
FA_THETA_SIGMA = 0.05
FOAM_NODES = {0.05: 24, 0.10: 32, 0.15: 42}
FOAM_NEIGHBOURS = 3
NODE_TO_STRUT = 1.2
TL_LAYERS = {0.05: 9, 0.10: 7, 0.15: 9}
TL_NOISE = 0.12
TL_BASE_N = 192

MATCHED_PAIRS = {1: {"FA": (7, 40), "FI": (0, 12)},
                 2: {"FA": (6, 52), "FI": (8, 14)},
                 3: {"FA": (2, 32), "FI": (4, 6)}}
"""(seed, number of fibers) of the FA and FI member of matched pair k (geometry.py:36-38)."""

_EX = np.array([1.0, 0.0, 0.0])
_EY = np.array([0.0, 1.0, 0.0])
_EZ = np.array([0.0, 0.0, 1.0])


def _matmul(a, b):
    with np.errstate(all="ignore"):  # some BLAS builds raise spurious flags on large products
        return a @ b


def _frame(z, helper):
    """Rotation with columns (x, y, z) for the unit axis z (geometry.py:49-56)."""

    if abs(float(np.dot(helper, z))) > 0.9:
        helper = _EY
    x = np.cross(helper, z)
    x /= np.linalg.norm(x)
    return np.stack([x, np.cross(z, x), z], axis=1)


# ---------------------------------------------------------------------------- device rendering

def _torch():
    import torch

    return torch


def _device_array(N: int):
    torch = _torch()
    return torch.empty((N, N, N), dtype=torch.uint8, device="cuda")


_OFFSET_GRIDS: dict = {}


def _offset_grid(pad: int):
    """The lattice offsets -pad..pad per axis (ij order) and their float transpose, built once per pad."""

    got = _OFFSET_GRIDS.get(pad)
    if got is None:
        g = np.arange(-pad, pad + 1, dtype=np.int64)
        off = np.stack([a.ravel() for a in np.meshgrid(g, g, g, indexing="ij")], axis=1)
        got = _OFFSET_GRIDS[pad] = (off, off.T.astype(float))  # the reference's layout for the product
    return got


class _Long:
    """A cylinder longer than the cell: its lattice nodes and, per radius, its disk offsets."""

    def __init__(self, N, half_length, R, center):
        self.N = int(N)
        axis = _matmul(R, _EZ)
        axis /= float(np.linalg.norm(axis))
        n_steps = max(1, int(math.ceil(2.0 * half_length)))
        t = np.arange(n_steps, dtype=float) - n_steps / 2.0
        pts = t[:, None] * axis[None, :] + np.asarray(center, dtype=float)[None, :]
        self.nodes = np.unique(np.rint(pts).astype(np.int64) % self.N, axis=0)
        self.Rq = _frame(axis / float(np.linalg.norm(axis)), _EX)

    def disk(self, r):
        """Lattice offsets of the one-cell-thick disk of radius r normal to the axis (geometry.py:73-78)."""

        off, off_t = _offset_grid(int(math.ceil(r)) + 2)
        local = _matmul(self.Rq.T, off_t).T
        keep = (((local[:, 0] / r) ** 2 + (local[:, 1] / r) ** 2 <= 1.0 + 1e-12)
                & (np.abs(local[:, 2]) <= 0.5 + 1e-12))
        return off[keep]


def _long_fiber(N, center, half_length, R):
    """shape_mask's long-cylinder branch (geometry.py:100-106): an integer centre builds at the
    origin and shifts by whole cells."""

    ci = tuple(int(round(c)) % N for c in center)
    if any(abs(c - float(i)) > 1e-9 for c, i in zip(center, ci)):
        return _Long(N, half_length, R, center)
    f = _Long(N, half_length, R, (0.0, 0.0, 0.0))
    if ci != (0, 0, 0):
        f.nodes = (f.nodes + np.asarray(ci, np.int64)) % N
    return f


def _stamp(N, fibers, r, out):
    """Union of the fibers at radius r into the device array ``out``; returns the solid cells."""

    nodes = [f.nodes for f in fibers]
    disks = [f.disk(r) for f in fibers]
    node_start = np.zeros(len(fibers) + 1, np.int64)
    off_start = np.zeros(len(fibers) + 1, np.int64)
    node_start[1:] = np.cumsum([len(a) for a in nodes])
    off_start[1:] = np.cumsum([len(a) for a in disks])
    nd = np.ascontiguousarray(np.concatenate(nodes) if nodes else np.zeros((0, 3)), dtype=np.int32)
    od = np.ascontiguousarray(np.concatenate(disks) if disks else np.zeros((0, 3)), dtype=np.int32)
    solid = ctypes.c_int64()
    _lib.check(_lib.load().pr_stamp_fibers(N, nd.ctypes.data, node_start.ctypes.data, od.ctypes.data,
                                           off_start.ctypes.data, len(fibers), 1, out.data_ptr(),
                                           ctypes.byref(solid), _lib.stream()))
    return int(solid.value)


def _shape(kind, center, radii, R):
    s = _lib.Shape()
    s.kind = 0 if kind == "ellipsoid" else 1
    s.center[:] = [float(c) for c in center]
    s.R[:] = [float(v) for v in np.asarray(R, dtype=float).ravel()]
    s.radii[:] = [float(v) for v in radii]
    return s


def _render_shapes(N, shapes, out):
    arr = (_lib.Shape * max(1, len(shapes)))(*shapes)
    solid = ctypes.c_int64()
    _lib.check(_lib.load().pr_render_shapes(N, arr, len(shapes), out.data_ptr(), ctypes.byref(solid),
                                            _lib.stream()))
    return int(solid.value)


def _host(out) -> np.ndarray:
    return out.cpu().numpy()


def shape_mask(N, center, radii, kind, R):
    """Cells whose centres lie inside a rotated ellipsoid or cylinder on the periodic grid
    (geometry.py:85-121), as a boolean array."""

    if kind not in ("ellipsoid", "cylinder"):
        raise ValueError(kind)
    N = int(N)
    out = _device_array(N)
    rx, ry, rz = radii
    if kind == "cylinder" and float(2.0 * rz) > float(N):
        _stamp(N, [_long_fiber(N, center, rz, R)], rx, out)
    else:
        _render_shapes(N, [_shape(kind, center, radii, R)], out)
    return _host(out).astype(bool)


def _bisect_radius(render, target_phi, r_lo, r_hi, tol=PHI_TOL, max_iter=24):
    """Bisection on a radius until |phi_s(r) - target| <= tol (geometry.py:124-145); render(r)
    fills a device array and returns its solid cells.  Returns (r, device phases)."""

    lo, hi, best = float(r_lo), float(r_hi), None
    for _ in range(int(max_iter)):
        mid = 0.5 * (lo + hi)
        phases, solid = render(mid)
        phi = float(solid / phases.numel())
        err = abs(phi - float(target_phi))
        if best is None or err < best[0]:
            best = (err, mid, phases.clone())  # the renderer reuses its array
        if err <= tol:
            break
        if phi < float(target_phi):
            lo = mid
        else:
            hi = mid
    return best[1], best[2]


# ---------------------------------------------------------------------------- fibers (FI, FA)

def _fiber_axis(rng, aligned):
    """Unnormalized fiber axis: isotropic, or tilted from x by theta ~ N(0, 0.05) with a uniform
    azimuth (geometry.py:150-156)."""

    if aligned:
        theta = rng.normal(0.0, FA_THETA_SIGMA)
        az = rng.uniform(0.0, 2.0 * math.pi)
        return np.array([math.cos(theta), math.sin(theta) * math.cos(az), math.sin(theta) * math.sin(az)])
    return rng.normal(size=3)


def fiber_lines(N, seed, n_lines, aligned, continuous_centers=False):
    """Centres and rotations of n_lines straight fibers from one random stream (geometry.py:159-175)."""

    rng = np.random.default_rng(int(seed))
    centers, rotations = [], []
    for _ in range(int(n_lines)):
        c = rng.random(3) * float(N) if continuous_centers else rng.integers(0, N, size=3)
        centers.append(tuple(float(v) for v in c))
        v = _fiber_axis(rng, aligned)
        if not aligned:
            v = v / np.linalg.norm(v)
        rotations.append(_frame(v / np.linalg.norm(v), _EZ))
    return centers, rotations


def _fiber_renderer(N, centers, rotations, length_factor):
    half = 0.5 * float(length_factor) * N
    fibers = [_long_fiber(N, c, half, R) for c, R in zip(centers, rotations)]
    if float(2.0 * half) <= float(N):
        raise ValueError("fibers shorter than the cell are not rendered by this path")
    out = _device_array(N)

    def render(r):
        return out, _stamp(N, fibers, r, out)

    return render


def render_fibers(N, centers, rotations, radius, length_factor):
    """Solid phase of periodic fibers of radius r and length length_factor * N (geometry.py:178-184)."""

    out, _ = _fiber_renderer(int(N), centers, rotations, length_factor)(float(radius))
    return _host(out)


# ---------------------------------------------------------------------------- open-cell foam (OF)

def foam_graph(N, seed, n_nodes, k=FOAM_NEIGHBOURS):
    """Uniform random nodes joined to their k nearest periodic neighbours (geometry.py:189-195)."""

    from scipy.spatial import cKDTree

    rng = np.random.default_rng(int(seed))
    points = rng.uniform(0, N, size=(int(n_nodes), 3))
    _, nn = cKDTree(points, boxsize=N).query(points, k=int(k) + 1)
    edges = {tuple(sorted((int(i), int(j)))) for i, row in enumerate(nn) for j in row[1:] if int(i) != int(j)}
    return points, sorted(edges)


def _strut_params(N, p0, p1):
    """Centre, half length and frame of the strut between two nodes along the minimum-image
    vector (geometry.py:198-208)."""

    vec = np.asarray(p1, dtype=float) - np.asarray(p0, dtype=float)
    for a in range(3):
        if vec[a] > N / 2:
            vec[a] -= N
        elif vec[a] < -N / 2:
            vec[a] += N
    L = float(np.linalg.norm(vec))
    center = tuple((np.asarray(p0, dtype=float) + 0.5 * vec) % N)
    return center, 0.5 * L, _frame(vec / L, _EZ)


# pr_shape as a NumPy record (int32 kind, int32 pad, f64 centre[3], f64 R[9], f64 radii[3]: 128 bytes)
SHAPE_DTYPE = np.dtype([("kind", "<i4"), ("pad", "<i4"), ("center", "<f8", (3,)), ("R", "<f8", (9,)),
                        ("radii", "<f8", (3,))])


def _foam_renderer(N, points, edges):
    struts = [_strut_params(N, points[a], points[b]) for a, b in edges]
    out = _device_array(N)
    short = [(c, h, R) for c, h, R in struts if not float(2.0 * h) > float(N)]
    longs = [_long_fiber(N, c, h, R) for c, h, R in struts if float(2.0 * h) > float(N)]
    # the shape table once (nodes, then the struts no longer than the cell); a trial sets radii only
    table = np.zeros(len(points) + len(short), dtype=SHAPE_DTYPE)
    n_nodes = len(points)
    table["kind"][:n_nodes] = 0
    table["center"][:n_nodes] = np.asarray([tuple(p.tolist()) for p in points], dtype=float).reshape(-1, 3)
    table["R"][:n_nodes] = np.eye(3).ravel()
    table["kind"][n_nodes:] = 1
    for q, (center, half, R) in enumerate(short):
        table["center"][n_nodes + q] = center
        table["R"][n_nodes + q] = np.asarray(R, dtype=float).ravel()
        table["radii"][n_nodes + q, 2] = half
    lib = _lib.load()

    def render(strut_radius, node_radius):
        table["radii"][:n_nodes] = float(node_radius)
        table["radii"][n_nodes:, 0] = float(strut_radius)
        table["radii"][n_nodes:, 1] = float(strut_radius)
        solid = ctypes.c_int64()
        _lib.check(lib.pr_render_shapes(N, table.ctypes.data, len(table), out.data_ptr(), ctypes.byref(solid),
                                        _lib.stream()))
        solid = int(solid.value)
        if longs:  # not reached for foams (struts are shorter than the cell); kept for generality
            extra = _device_array(N)
            _stamp(N, longs, strut_radius, extra)
            out.bitwise_or_(extra)
            solid = int((out == 1).sum().item())
        return out, solid

    return render


def render_foam(N, points, edges, strut_radius, node_radius):
    """Solid phase of spherical nodes and cylindrical struts (geometry.py:211-218)."""

    out, _ = _foam_renderer(int(N), np.asarray(points, dtype=float), edges)(float(strut_radius), float(node_radius))
    return _host(out)


# ---------------------------------------------------------------------------- tortuous layered (TL)

def lamellar_field(N, seed, n_layers, waviness, noise_amp=TL_NOISE):
    """Layered field of n_layers wavy layers normal to x plus smoothed Gaussian noise
    (geometry.py:223-239); host NumPy, as the reference."""

    rng = np.random.default_rng(int(seed))
    x = np.arange(N, dtype=float)[:, None, None]
    y = np.arange(N, dtype=float)[None, :, None]
    z = np.arange(N, dtype=float)[None, None, :]
    base = np.cos(2.0 * np.pi * n_layers * x / float(N))
    ph1 = rng.uniform(0.0, 2 * np.pi)
    ph2 = rng.uniform(0.0, 2 * np.pi)
    wav = float(waviness) * (0.65 * np.sin(2 * np.pi * y / float(N) + ph1)
                             + 0.35 * np.cos(4 * np.pi * z / float(N) + ph2))
    field = base + 0.35 * np.sin(2 * np.pi * n_layers * (x + wav) / float(N))
    noise = rng.normal(scale=float(noise_amp), size=(N, N, N))
    noise = (noise + np.roll(noise, 1, 0) + np.roll(noise, -1, 0) + np.roll(noise, 1, 1)
             + np.roll(noise, -1, 1) + np.roll(noise, 1, 2) + np.roll(noise, -1, 2)) / 7.0
    return field + noise


def _lamellar_device(N, seed, n_layers, waviness, noise_amp=TL_NOISE):
    """lamellar_field's values in a device array: the draws and the per-axis sines and cosines on
    the host as the reference makes them, the N^3 field on the device (``pr_lamellar_field``)."""

    torch = _torch()
    rng = np.random.default_rng(int(seed))
    x = np.arange(N, dtype=float)
    base = np.ascontiguousarray(np.cos(2.0 * np.pi * n_layers * x / float(N)))
    ph1 = rng.uniform(0.0, 2 * np.pi)
    ph2 = rng.uniform(0.0, 2 * np.pi)
    sin_y = np.ascontiguousarray(np.sin(2 * np.pi * x / float(N) + ph1))
    cos_z = np.ascontiguousarray(np.cos(4 * np.pi * x / float(N) + ph2))
    noise = np.ascontiguousarray(rng.normal(scale=float(noise_amp), size=(N, N, N)))
    field = torch.empty((N, N, N), dtype=torch.float64, device="cuda")
    _lib.check(_lib.load().pr_lamellar_field(N, base.ctypes.data, sin_y.ctypes.data, cos_z.ctypes.data,
                                             float(waviness), 2 * np.pi * n_layers, noise.ctypes.data,
                                             field.data_ptr(), _lib.stream()))
    return field


def _threshold_device(field, target_phi):
    out = _torch().empty(field.shape, dtype=_torch().uint8, device="cuda")
    _lib.check(_lib.load().pr_quantile_threshold(field.data_ptr(), field.numel(), 1.0 - float(target_phi), 0,
                                                 out.data_ptr(), None, None, _lib.stream()))
    return out


def threshold(field, target_phi):
    """Solid where the field reaches its (1 - phi_s) quantile (geometry.py:242-245)."""

    q = np.quantile(field.ravel(), 1.0 - float(target_phi))
    return (field >= q).astype(np.uint8)


# ---------------------------------------------------------------------------- builders

def _build_device(structure, N, target_phi, seed, continuous_centers=False):
    phi = round(float(target_phi), 2)
    if structure in ("FI", "FA"):
        centers, rotations = fiber_lines(N, seed, FIBER_LINES[structure][phi], structure == "FA", continuous_centers)
        render = _fiber_renderer(N, centers, rotations, FIBER_LENGTH[structure])
        return _bisect_radius(render, target_phi, 0.1, 4.0)[1]
    if structure == "OF":
        points, edges = foam_graph(N, seed, FOAM_NODES[phi])
        s = max(1.0, float(N) / 48.0)
        render = _foam_renderer(N, points, edges)
        return _bisect_radius(lambda r: render(r, float(NODE_TO_STRUT * r)), target_phi, 0.2 * s, 4.0 * s)[1]
    if structure == "TL":
        return _threshold_device(_lamellar_device(N, seed, TL_LAYERS[phi], 1.4 + 3.0 * float(target_phi)),
                                 target_phi)
    raise ValueError(structure)


def build(structure, N, target_phi, seed, continuous_centers=False, *, device=False):
    """Digital microstructure of one structure at a target solid fraction (geometry.py:250-258).
    ``device=True`` returns the uint8 CUDA tensor instead of a NumPy array."""

    out = _build_device(structure, int(N), target_phi, seed, continuous_centers)
    return out if device else _host(out)


def accepted(structure, d, target_phi):
    """Acceptance rules of the core library (geometry.py:261-281)."""

    if abs(float(d["phi_solid"]) - float(target_phi)) > PHI_TOL:
        return False
    c = d["mean_pore_chord"]
    if structure == "OF":
        return all(d["pore_percolates"]) and d["pore_largest_cluster_fraction"] >= MIN_PORE_CLUSTER
    if structure == "TL":
        return max(c) / max(min(c), 1e-12) >= 2.0
    if structure == "FA":
        return c[0] / max(0.5 * (c[1] + c[2]), 1e-12) >= 2.0
    if structure == "FI":
        return max(c) / max(min(c), 1e-12) < 2.0
    raise ValueError(structure)


def core_realizations(structure, target_phi, n_accept=4, max_trials=80, *, device=False):
    """One cell of the core library at N = 128 from seeds 0, 1, 2, ... until n_accept are accepted
    (geometry.py:284-296); the scalar descriptors of each trial come from the device."""

    from .descriptors import scalar_descriptors

    out = []
    for seed in range(int(max_trials)):
        phases = _build_device(structure, CORE_N, target_phi, seed)
        if accepted(structure, scalar_descriptors(phases), target_phi):
            out.append((seed, phases if device else _host(phases)))
            if len(out) == int(n_accept):
                break
    return out


def core_library(structures=STRUCTURES, phis=CORE_PHIS, n_accept=4, max_trials=80, *, device=False):
    """Every cell of the core library, {(structure, phi): [(seed, phases), ...]}, as
    ``core_realizations`` builds each; the cells run at once on worker threads with their own
    streams, so TL's host fields overlap the device renderings of the other structures."""

    from .streams import run_concurrently

    cells = [(s, phi) for s in structures for phi in phis]
    out = run_concurrently([(core_realizations, (s, phi, n_accept, max_trials), dict(device=device))
                            for s, phi in cells])
    return dict(zip(cells, out))


def canonical(structure, N, *, device=False):
    """Canonical microstructure at phi_s = 0.10 and seed 0 on an N^3 grid (geometry.py:299-314);
    TL's field is drawn at N = 192 and resampled by periodic cubic splines on the host."""

    if structure == "TL":
        from scipy.ndimage import zoom

        if N == TL_BASE_N:
            out = _threshold_device(_lamellar_device(TL_BASE_N, 0, TL_LAYERS[0.10], 1.4 + 3.0 * 0.10), 0.10)
            return out if device else _host(out)
        field = lamellar_field(TL_BASE_N, 0, TL_LAYERS[0.10], 1.4 + 3.0 * 0.10)
        if N != TL_BASE_N:
            field = zoom(field, float(N) / float(TL_BASE_N), order=3, mode="grid-wrap", grid_mode=True,
                         prefilter=True)
        ph = threshold(field, 0.10)
        return _torch().from_numpy(ph).cuda() if device else ph
    return build(structure, N, 0.10, 0, continuous_centers=True, device=device)


def matched(structure, pair, N=CORE_N, *, device=False):
    """Member FA or FI of matched fiber pair k = 1, 2, 3 at phi_s = 0.10 (geometry.py:317-333)."""

    seed, n_lines = MATCHED_PAIRS[pair][structure]
    aligned = structure == "FA"
    centers = [tuple(float(v) for v in c)
               for c in (np.random.default_rng(seed + 1000003).random((64, 3)) * N)[:n_lines]]
    rng = np.random.default_rng(seed + (3000003 if aligned else 2000003))
    rotations = []
    for _ in range(n_lines):
        v = _fiber_axis(rng, aligned)
        rotations.append(_frame(v / np.linalg.norm(v), _EZ))
    render = _fiber_renderer(int(N), centers, rotations, 9.0)
    out = _bisect_radius(render, 0.1, 0.12, 7.0, tol=5e-4, max_iter=32)[1]
    return out if device else _host(out)

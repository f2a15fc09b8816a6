"""The reference's digital microstructures (porerad/geometry.py), generated on a B200.

Four structures on a periodic N x N x N grid (axis 0 = x; uint8, 1 = solid): OF open-cell foam,
FI random fibers, FA fibers aligned with x, TL tortuous layers.  The archived arrays of the
reference (data/microstructures.csv, ``phase_sha256``) are reproduced bit for bit.

Generation is split in three parts:

1. **Draws.**  Everything random is drawn on the host with the reference's NumPy calls in the
   reference's order and recorded as plain arrays: :class:`CylinderDraws` (fiber centres and
   frames), :class:`FoamDraws` (node positions and the periodic k-nearest-neighbour edges) and
   :class:`LayerDraws` (the two layer phases and the Gaussian noise of TL).
2. **Geometry records.**  The draws become the inputs of the device kernels: for each cylinder
   longer than the cell, its lattice nodes and, per radius, the offsets of a one-cell-thick disk
   (:class:`LatticeCylinder`); for shorter shapes, a table of ``pr_shape`` records (kind, centre,
   frame, radii) in which a trial radius rewrites only the radii (:class:`ShapeTable`).
3. **Device work.**  ``pr_stamp_fibers`` and ``pr_render_shapes`` fill a device array and count
   its solid cells for each trial radius of the bisection; TL's N^3 field and its quantile
   threshold are ``pr_lamellar_field`` and ``pr_quantile_threshold``; acceptance of a core-library
   trial reads the device descriptors.

The floating-point steps that decide a cell are the reference's, operation for operation (frame
construction, repeated normalisations, the 3 x M product of a disk's offsets, the minimum-image
strut vector, rounding of lattice nodes, the field's evaluation order), because a different
rounding anywhere would move a cell.  TL's field stays a host array only where SciPy resamples
it (the canonical TL at N = 128 and 160).
"""

from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass

import numpy as np

from . import _lib

# Parameter tables of the reference's library (porerad/geometry.py:19-38).  These values define
# the archived microstructures, so they are the reference's.
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
"""(seed, number of fibers) of the FA and FI member of matched pair k."""

_BASIS = np.eye(3)  # rows: unit vectors along x, y, z
_MATCHED_CENTRE_STREAM, _MATCHED_AXIS_STREAM = 1000003, {True: 3000003, False: 2000003}
_MATCHED_LENGTH = 9.0


def _blas(a, b):
    """a @ b with floating-point warnings off (some BLAS builds flag large products spuriously)."""

    with np.errstate(all="ignore"):
        return a @ b


def axis_frame(axis: np.ndarray, helper: int) -> np.ndarray:
    """Rotation whose columns are (u, axis x u, axis) for a unit ``axis``.

    u is the normalised cross product of a helper basis vector (x: 0, z: 2) with the axis; the
    helper becomes y where it lies within acos(0.9) of the axis.
    """

    h = _BASIS[1] if abs(float(np.dot(_BASIS[helper], axis))) > 0.9 else _BASIS[helper]
    u = np.cross(h, axis)
    u /= np.linalg.norm(u)
    return np.stack([u, np.cross(axis, u), axis], axis=1)


# ---------------------------------------------------------------------------- draws

@dataclass
class CylinderDraws:
    """Straight cylinders as drawn: centres (n, 3) in cells and frames (n, 3, 3) whose third
    column is the cylinder axis."""

    centres: np.ndarray
    frames: np.ndarray

    def __len__(self) -> int:
        return len(self.centres)


def _direction(rng, tilted: bool) -> np.ndarray:
    """One fiber direction, not yet normalised: three standard normals (isotropic), or a tilt
    theta ~ N(0, FA_THETA_SIGMA) away from x at a uniform azimuth (aligned)."""

    if not tilted:
        return rng.normal(size=3)
    theta = rng.normal(0.0, FA_THETA_SIGMA)
    azimuth = rng.uniform(0.0, 2.0 * math.pi)
    return np.array([math.cos(theta), math.sin(theta) * math.cos(azimuth), math.sin(theta) * math.sin(azimuth)])


def _unit(v: np.ndarray) -> np.ndarray:
    return v / np.linalg.norm(v)


def draw_library_fibers(N: int, seed: int, count: int, tilted: bool, uniform_centres: bool) -> CylinderDraws:
    """Fibers of a core or canonical microstructure: one stream; per fiber its centre (a lattice
    node, or a uniform point when ``uniform_centres``) and then its direction."""

    rng = np.random.default_rng(int(seed))
    centres = np.empty((int(count), 3))
    frames = np.empty((int(count), 3, 3))
    for i in range(int(count)):
        centres[i] = rng.random(3) * float(N) if uniform_centres else rng.integers(0, N, size=3)
        d = _direction(rng, tilted)
        if not tilted:
            d = _unit(d)  # isotropic directions are normalised once more below, as drawn
        frames[i] = axis_frame(_unit(d), 2)
    return CylinderDraws(centres, frames)


def draw_matched_fibers(N: int, pair: int, structure: str) -> CylinderDraws:
    """Fibers of a member of a matched pair: the centres from the first rows of a 64-point
    uniform stream, the directions from a second stream."""

    seed, count = MATCHED_PAIRS[int(pair)][structure]
    tilted = structure == "FA"
    points = np.random.default_rng(seed + _MATCHED_CENTRE_STREAM).random((64, 3)) * N
    rng = np.random.default_rng(seed + _MATCHED_AXIS_STREAM[tilted])
    frames = np.stack([axis_frame(_unit(_direction(rng, tilted)), 2) for _ in range(count)]) if count else \
        np.empty((0, 3, 3))
    return CylinderDraws(np.array(points[:count]), frames)


@dataclass
class FoamDraws:
    """Foam nodes (m, 3) uniform in the cell and the edges (i < j) joining each node to its
    k nearest periodic neighbours, sorted."""

    nodes: np.ndarray
    edges: np.ndarray  # (k, 2) int64

    def struts(self, N: int):
        """Centre (k, 3), half length (k,) and frame (k, 3, 3) of each strut, along the
        minimum-image vector between its nodes."""

        p0, p1 = self.nodes[self.edges[:, 0]], self.nodes[self.edges[:, 1]]
        v = p1 - p0
        half_cell = N / 2
        v = np.where(v > half_cell, v - N, np.where(v < -half_cell, v + N, v))
        lengths = np.array([float(np.linalg.norm(row)) for row in v])
        centres = (p0 + 0.5 * v) % N
        frames = np.stack([axis_frame(row / L, 2) for row, L in zip(v, lengths)]) if len(v) else \
            np.empty((0, 3, 3))
        return centres, 0.5 * lengths, frames


def draw_foam(N: int, seed: int, n_nodes: int, k: int = FOAM_NEIGHBOURS) -> FoamDraws:
    from scipy.spatial import cKDTree

    nodes = np.random.default_rng(int(seed)).uniform(0, N, size=(int(n_nodes), 3))
    _, near = cKDTree(nodes, boxsize=N).query(nodes, k=int(k) + 1)
    own = np.repeat(np.arange(len(nodes)), int(k))
    other = near[:, 1:].ravel().astype(np.int64)
    keep = other != own
    pairs = np.sort(np.stack([own[keep], other[keep]], axis=1), axis=1)
    edges = np.unique(pairs, axis=0) if len(pairs) else np.empty((0, 2), np.int64)
    return FoamDraws(nodes, edges.astype(np.int64))


@dataclass
class LayerDraws:
    """TL's draws: the phases of the y and z waviness and the Gaussian noise (N, N, N)."""

    phase_y: float
    phase_z: float
    noise: np.ndarray


def draw_layers(N: int, seed: int, noise_amp: float = TL_NOISE) -> LayerDraws:
    rng = np.random.default_rng(int(seed))
    py = rng.uniform(0.0, 2 * np.pi)
    pz = rng.uniform(0.0, 2 * np.pi)
    return LayerDraws(py, pz, rng.normal(scale=float(noise_amp), size=(N, N, N)))


def _layer_profiles(N: int, n_layers: int, draws: LayerDraws):
    """Per-axis factors of the layered field: cos of the layer index along x, the y waviness
    sine and the z waviness cosine."""

    g = np.arange(N, dtype=float)
    across = np.cos(2.0 * np.pi * n_layers * g / float(N))
    wave_y = np.sin(2 * np.pi * g / float(N) + draws.phase_y)
    wave_z = np.cos(4 * np.pi * g / float(N) + draws.phase_z)
    return across, wave_y, wave_z


def layer_field_host(N: int, n_layers: int, waviness: float, draws: LayerDraws) -> np.ndarray:
    """The layered field on the host: layers plus a sine displaced by the y/z waviness, plus the
    noise averaged over each cell and its six neighbours."""

    across, wave_y, wave_z = _layer_profiles(N, n_layers, draws)
    shift = float(waviness) * (0.65 * wave_y[None, :, None] + 0.35 * wave_z[None, None, :])
    x = np.arange(N, dtype=float)[:, None, None]
    field = across[:, None, None] + 0.35 * np.sin(2 * np.pi * n_layers * (x + shift) / float(N))
    smooth = draws.noise.copy()
    for axis in range(3):
        for step in (1, -1):
            smooth += np.roll(draws.noise, step, axis)
    smooth /= 7.0
    return field + smooth


def layer_field_device(N: int, n_layers: int, waviness: float, draws: LayerDraws):
    """The layered field as a device array (``pr_lamellar_field``, with a correctly rounded sine)."""

    torch = _torch()
    across, wave_y, wave_z = (np.ascontiguousarray(a) for a in _layer_profiles(N, n_layers, draws))
    noise = np.ascontiguousarray(draws.noise)
    field = torch.empty((N, N, N), dtype=torch.float64, device="cuda")
    _lib.check(_lib.load().pr_lamellar_field(N, across.ctypes.data, wave_y.ctypes.data, wave_z.ctypes.data,
                                             float(waviness), 2 * np.pi * n_layers, noise.ctypes.data,
                                             field.data_ptr(), _lib.stream()))
    return field


# ---------------------------------------------------------------------------- geometry records

def _torch():
    import torch

    return torch


def _device_array(N: int):
    torch = _torch()
    return torch.empty((N, N, N), dtype=torch.uint8, device="cuda")


_OFFSETS: dict = {}


def _offsets(pad: int):
    """Integer offsets -pad..pad per axis in C order, and their transpose as floats (3, M)."""

    got = _OFFSETS.get(pad)
    if got is None:
        g = np.arange(-pad, pad + 1, dtype=np.int64)
        off = np.stack([a.ravel() for a in np.meshgrid(g, g, g, indexing="ij")], axis=1)
        got = _OFFSETS[pad] = (off, off.T.astype(float))
    return got


class LatticeCylinder:
    """A cylinder longer than the cell: the lattice nodes nearest to unit steps along its axis
    (rounded half to even, wrapped) and, per radius, the cells of a one-cell-thick disk of that
    radius normal to the axis.  The cylinder is the union of the disks placed on the nodes.

    A centre on a lattice node builds the nodes about the origin and shifts them by whole cells.
    """

    def __init__(self, N: int, centre, half_length: float, frame: np.ndarray):
        self.N = int(N)
        c = np.asarray(centre, dtype=float)
        node = np.array([int(round(float(v))) % self.N for v in c], dtype=np.int64)
        on_node = all(abs(float(v) - float(i)) <= 1e-9 for v, i in zip(c, node))
        axis = _blas(frame, _BASIS[2])
        axis /= float(np.linalg.norm(axis))
        steps = max(1, int(math.ceil(2.0 * half_length)))
        t = np.arange(steps, dtype=float) - steps / 2.0
        origin = np.zeros(3) if on_node else c
        nodes = np.unique(np.rint(t[:, None] * axis[None, :] + origin[None, :]).astype(np.int64) % self.N, axis=0)
        if on_node and node.any():
            nodes = (nodes + node) % self.N
        self.nodes = nodes
        self.disk_frame = axis_frame(axis / float(np.linalg.norm(axis)), 0)

    def disk(self, r: float) -> np.ndarray:
        off, off_t = _offsets(int(math.ceil(r)) + 2)
        local = _blas(self.disk_frame.T, off_t).T
        inside = ((local[:, 0] / r) ** 2 + (local[:, 1] / r) ** 2 <= 1.0 + 1e-12) & (np.abs(local[:, 2]) <= 0.5 + 1e-12)
        return off[inside]


def stamp_cylinders(N: int, cylinders, r: float, out) -> int:
    """Union of the cylinders at radius r written into the device array ``out``; returns its solid cells."""

    nodes = [c.nodes for c in cylinders]
    disks = [c.disk(r) for c in cylinders]
    node_start = np.concatenate([[0], np.cumsum([len(a) for a in nodes], dtype=np.int64)]).astype(np.int64)
    disk_start = np.concatenate([[0], np.cumsum([len(a) for a in disks], dtype=np.int64)]).astype(np.int64)
    nd = np.ascontiguousarray(np.concatenate(nodes) if nodes else np.zeros((0, 3)), dtype=np.int32)
    dd = np.ascontiguousarray(np.concatenate(disks) if disks else np.zeros((0, 3)), dtype=np.int32)
    solid = ctypes.c_int64()
    _lib.check(_lib.load().pr_stamp_fibers(N, nd.ctypes.data, node_start.ctypes.data, dd.ctypes.data,
                                           disk_start.ctypes.data, len(cylinders), 1, out.data_ptr(),
                                           ctypes.byref(solid), _lib.stream()))
    return int(solid.value)


SHAPE_DTYPE = np.dtype([("kind", "<i4"), ("pad", "<i4"), ("center", "<f8", (3,)), ("R", "<f8", (9,)),
                        ("radii", "<f8", (3,))])
"""``pr_shape`` as a NumPy record: kind (0 ellipsoid, 1 cylinder), centre, frame, radii (128 bytes)."""


class ShapeTable:
    """Ellipsoids and cylinders no longer than the cell as ``pr_shape`` records.  ``pr_render_shapes``
    tests every cell centre against each shape in its frame with minimum-image offsets."""

    def __init__(self, centres, frames, kinds, half_lengths=None):
        n = len(centres)
        self.table = np.zeros(n, dtype=SHAPE_DTYPE)
        self.table["kind"] = kinds
        self.table["center"] = np.asarray(centres, dtype=float).reshape(n, 3)
        self.table["R"] = np.asarray(frames, dtype=float).reshape(n, 9)
        if half_lengths is not None:
            self.table["radii"][:, 2] = half_lengths

    def render(self, N: int, out) -> int:
        solid = ctypes.c_int64()
        _lib.check(_lib.load().pr_render_shapes(N, self.table.ctypes.data, len(self.table), out.data_ptr(),
                                                ctypes.byref(solid), _lib.stream()))
        return int(solid.value)


def shape_mask(N, center, radii, kind, R):
    """Cells whose centres lie inside a rotated ellipsoid or cylinder on the periodic grid, as a
    boolean array (geometry.py:85-121).  A cylinder longer than the cell is stamped on the lattice."""

    if kind not in ("ellipsoid", "cylinder"):
        raise ValueError(kind)
    N = int(N)
    out = _device_array(N)
    if kind == "cylinder" and float(2.0 * radii[2]) > float(N):
        stamp_cylinders(N, [LatticeCylinder(N, center, radii[2], np.asarray(R, dtype=float))], radii[0], out)
    else:
        shapes = ShapeTable([center], [R], [0 if kind == "ellipsoid" else 1])
        shapes.table["radii"][0] = [float(v) for v in radii]
        shapes.render(N, out)
    return out.cpu().numpy().astype(bool)


# ---------------------------------------------------------------------------- renderers

class FiberRenderer:
    """Fibers of length ``length_factor`` x N from their draws; ``render(r)`` stamps them at radius r
    into one reused device array and returns (array, solid cells)."""

    def __init__(self, N: int, draws: CylinderDraws, length_factor: float):
        self.N = int(N)
        half = 0.5 * float(length_factor) * self.N
        if float(2.0 * half) <= float(self.N):
            raise ValueError("fibers shorter than the cell are not rendered by this path")
        self.cylinders = [LatticeCylinder(self.N, c, half, f) for c, f in zip(draws.centres, draws.frames)]
        self.out = _device_array(self.N)

    def __call__(self, r: float):
        return self.out, stamp_cylinders(self.N, self.cylinders, r, self.out)


class FoamRenderer:
    """Spherical nodes of radius 1.2 r and cylindrical struts of radius r from the foam draws."""

    def __init__(self, N: int, foam: FoamDraws):
        self.N = int(N)
        centres, half, frames = foam.struts(self.N)
        long = 2.0 * half > float(self.N)
        m = len(foam.nodes)
        self.shapes = ShapeTable(np.concatenate([foam.nodes, centres[~long]]),
                                 np.concatenate([np.broadcast_to(np.eye(3), (m, 3, 3)), frames[~long]]),
                                 [0] * m + [1] * int((~long).sum()),
                                 np.concatenate([np.zeros(m), half[~long]]))
        self.n_nodes = m
        # struts longer than the cell (not met by the reference's foams, kept for generality)
        self.long = [LatticeCylinder(self.N, c, h, f) for c, h, f in zip(centres[long], half[long], frames[long])]
        self.out = _device_array(self.N)

    def __call__(self, strut_radius: float, node_radius: float):
        radii = self.shapes.table["radii"]
        radii[: self.n_nodes] = float(node_radius)
        radii[self.n_nodes:, :2] = float(strut_radius)
        solid = self.shapes.render(self.N, self.out)
        if self.long:
            extra = _device_array(self.N)
            stamp_cylinders(self.N, self.long, strut_radius, extra)
            self.out.bitwise_or_(extra)
            solid = int((self.out == 1).sum().item())
        return self.out, solid


def bisect_radius(render, target_phi, r_lo, r_hi, tol=PHI_TOL, max_iter=24):
    """Radius bisection until |phi_s(r) - target| <= tol, keeping the first closest trial
    (geometry.py:124-145).  ``render(r)`` returns (device array, solid cells); the array may be
    reused by the next trial.  Returns (r, device phases)."""

    lo, hi = float(r_lo), float(r_hi)
    best_err, best = math.inf, None
    for _ in range(int(max_iter)):
        r = 0.5 * (lo + hi)
        phases, solid = render(r)
        phi = float(solid / phases.numel())
        err = abs(phi - float(target_phi))
        if best is None or err < best_err:
            best_err, best = err, (r, phases.clone())
        if err <= tol:
            break
        lo, hi = (r, hi) if phi < float(target_phi) else (lo, r)
    return best


# ---------------------------------------------------------------------------- the reference's API

def fiber_lines(N, seed, n_lines, aligned, continuous_centers=False):
    """Centres (tuples) and frames of n_lines straight fibers drawn from one stream (geometry.py:159-175)."""

    d = draw_library_fibers(N, seed, n_lines, bool(aligned), bool(continuous_centers))
    return [tuple(float(v) for v in c) for c in d.centres], list(d.frames)


def render_fibers(N, centers, rotations, radius, length_factor):
    """Solid phase of periodic fibers of radius r and length length_factor x N (geometry.py:178-184)."""

    draws = CylinderDraws(np.asarray(centers, dtype=float).reshape(-1, 3), np.asarray(rotations, dtype=float))
    out, _ = FiberRenderer(int(N), draws, length_factor)(float(radius))
    return out.cpu().numpy()


def foam_graph(N, seed, n_nodes, k=FOAM_NEIGHBOURS):
    """Random nodes and the sorted edges (i, j), i < j, to each node's k nearest periodic neighbours
    (geometry.py:189-195)."""

    foam = draw_foam(N, seed, n_nodes, k)
    return foam.nodes, [tuple(int(v) for v in e) for e in foam.edges]


def render_foam(N, points, edges, strut_radius, node_radius):
    """Solid phase of spherical nodes and cylindrical struts (geometry.py:211-218)."""

    foam = FoamDraws(np.asarray(points, dtype=float), np.asarray(edges, dtype=np.int64).reshape(-1, 2))
    out, _ = FoamRenderer(int(N), foam)(float(strut_radius), float(node_radius))
    return out.cpu().numpy()


def lamellar_field(N, seed, n_layers, waviness, noise_amp=TL_NOISE):
    """TL's continuous field of n_layers wavy layers normal to x plus smoothed noise, as a host
    array (geometry.py:223-239)."""

    return layer_field_host(int(N), n_layers, waviness, draw_layers(int(N), seed, noise_amp))


def threshold(field, target_phi):
    """Solid where the field reaches its (1 - phi_s) quantile (geometry.py:242-245)."""

    level = np.quantile(np.ravel(field), 1.0 - float(target_phi))
    return (field >= level).astype(np.uint8)


def _threshold_device(field, target_phi):
    torch = _torch()
    out = torch.empty(field.shape, dtype=torch.uint8, device="cuda")
    _lib.check(_lib.load().pr_quantile_threshold(field.data_ptr(), field.numel(), 1.0 - float(target_phi), 0,
                                                 out.data_ptr(), None, None, _lib.stream()))
    return out


def _fibers(structure, N, phi, seed, uniform_centres):
    draws = draw_library_fibers(N, seed, FIBER_LINES[structure][round(float(phi), 2)], structure == "FA",
                                uniform_centres)
    return bisect_radius(FiberRenderer(N, draws, FIBER_LENGTH[structure]), phi, 0.1, 4.0)[1]


def _foam(N, phi, seed):
    render = FoamRenderer(N, draw_foam(N, seed, FOAM_NODES[round(float(phi), 2)]))
    scale = max(1.0, float(N) / 48.0)
    return bisect_radius(lambda r: render(r, float(NODE_TO_STRUT * r)), phi, 0.2 * scale, 4.0 * scale)[1]


def _layers(N, phi, seed):
    field = layer_field_device(N, TL_LAYERS[round(float(phi), 2)], 1.4 + 3.0 * float(phi), draw_layers(N, seed))
    return _threshold_device(field, phi)


_RECIPES = {
    "FI": lambda N, phi, seed, uniform: _fibers("FI", N, phi, seed, uniform),
    "FA": lambda N, phi, seed, uniform: _fibers("FA", N, phi, seed, uniform),
    "OF": lambda N, phi, seed, uniform: _foam(N, phi, seed),
    "TL": lambda N, phi, seed, uniform: _layers(N, phi, seed),
}


def _on_device(structure, N, target_phi, seed, continuous_centers=False):
    if structure not in _RECIPES:
        raise ValueError(structure)
    return _RECIPES[structure](int(N), target_phi, seed, bool(continuous_centers))


def build(structure, N, target_phi, seed, continuous_centers=False, *, device=False):
    """Digital microstructure of one structure at a target solid fraction (geometry.py:250-258).
    ``device=True`` returns the uint8 CUDA tensor instead of a NumPy array."""

    out = _on_device(structure, N, target_phi, seed, continuous_centers)
    return out if device else out.cpu().numpy()


def _anisotropy(chords) -> float:
    return max(chords) / max(min(chords), 1e-12)


# structure signature of an accepted core-library trial, over its scalar descriptor record
_SIGNATURES = {
    "OF": lambda d: all(d["pore_percolates"]) and d["pore_largest_cluster_fraction"] >= MIN_PORE_CLUSTER,
    "TL": lambda d: _anisotropy(d["mean_pore_chord"]) >= 2.0,
    "FA": lambda d: d["mean_pore_chord"][0] / max(0.5 * (d["mean_pore_chord"][1] + d["mean_pore_chord"][2]),
                                                  1e-12) >= 2.0,
    "FI": lambda d: _anisotropy(d["mean_pore_chord"]) < 2.0,
}


def accepted(structure, d, target_phi):
    """Acceptance of a core-library trial from its descriptor record (geometry.py:261-281): solid
    fraction within PHI_TOL of the target and the structure's signature (OF: pore phase
    percolating along x, y and z with its largest 26-connected cluster >= 99 % of the pores; TL:
    max/min mean pore chord >= 2; FA: chord along x >= 2 x the mean of y and z; FI: max/min < 2)."""

    if abs(float(d["phi_solid"]) - float(target_phi)) > PHI_TOL:
        return False
    if structure not in _SIGNATURES:
        raise ValueError(structure)
    return bool(_SIGNATURES[structure](d))


def core_realizations(structure, target_phi, n_accept=4, max_trials=80, *, device=False):
    """One cell of the core library at N = 128: seeds 0, 1, 2, ... until n_accept trials are
    accepted (geometry.py:284-296); each trial's scalar descriptors come from the device."""

    from .descriptors import scalar_descriptors

    kept = []
    for seed in range(int(max_trials)):
        phases = _on_device(structure, CORE_N, target_phi, seed)
        if accepted(structure, scalar_descriptors(phases), target_phi):
            kept.append((seed, phases if device else phases.cpu().numpy()))
            if len(kept) == int(n_accept):
                break
    return kept


def core_library(structures=STRUCTURES, phis=CORE_PHIS, n_accept=4, max_trials=80, *, device=False):
    """Every cell of the core library, {(structure, phi): [(seed, phases), ...]}, each as
    ``core_realizations`` builds it; the cells run at once on worker threads with their own
    streams, so TL's host draws overlap the device renderings of the other structures."""

    from .streams import run_concurrently

    cells = [(s, phi) for s in structures for phi in phis]
    out = run_concurrently([(core_realizations, (s, phi, n_accept, max_trials), dict(device=device))
                            for s, phi in cells])
    return dict(zip(cells, out))


def canonical(structure, N, *, device=False):
    """Canonical microstructure at phi_s = 0.10, seed 0, on an N^3 grid (geometry.py:299-314).

    FI and FA use uniform fiber centres (the same fibers at every N).  TL's field is drawn at
    N = 192; at other N it is resampled by SciPy's periodic cubic splines on the host before the
    threshold."""

    if structure != "TL":
        return build(structure, N, 0.10, 0, continuous_centers=True, device=device)
    draws = draw_layers(TL_BASE_N, 0)
    waviness = 1.4 + 3.0 * 0.10
    if int(N) == TL_BASE_N:
        out = _threshold_device(layer_field_device(TL_BASE_N, TL_LAYERS[0.10], waviness, draws), 0.10)
        return out if device else out.cpu().numpy()
    from scipy.ndimage import zoom

    field = zoom(layer_field_host(TL_BASE_N, TL_LAYERS[0.10], waviness, draws), float(N) / float(TL_BASE_N),
                 order=3, mode="grid-wrap", grid_mode=True, prefilter=True)
    ph = threshold(field, 0.10)
    return _torch().from_numpy(ph).cuda() if device else ph


def matched(structure, pair, N=CORE_N, *, device=False):
    """Member FA or FI of matched fiber pair k = 1, 2, 3 at phi_s = 0.10: fibers of length 9 N,
    radius bisected to |phi_s - 0.10| <= 5e-4 (geometry.py:317-333)."""

    render = FiberRenderer(int(N), draw_matched_fibers(int(N), pair, structure), _MATCHED_LENGTH)
    out = bisect_radius(render, 0.1, 0.12, 7.0, tol=5e-4, max_iter=32)[1]
    return out if device else out.cpu().numpy()

"""ORACLE — test infrastructure only.

CPU restatement of porerad's surface-radiation path (moxi000/pore-radiation-ijhmt2026),
used as the checker by ``tests/``, by ``__graft_entry__.smoke()`` and by the CPU-baseline
leg of ``bench.py``.  The product (``porerad_b200``) never imports this module: its path
runs on the GPU and fails loudly when the CUDA library is missing.

Every function names the reference lines it restates (porerad/view_factors.py,
porerad/exchange.py, porerad/coupled.py, porerad/conduction.py).  The traversal itself is the C
file ``oracle/dda.c`` (an OpenMP loop over rays, like the reference's Numba ``prange``);
the rest is NumPy/SciPy.  Third-party arithmetic on the path is used exactly as the
reference uses it: ``numpy.random.PCG64`` + ``Generator.random`` for the ray stream,
NumPy's ``cos``/``sin`` (glibc) for the azimuth, and ``scipy.optimize.anderson`` for
the diagonal balancing.

Pinning: the integer first-hit counts of this oracle reproduce the SHA-256 hashes the
reference stores in data/cases_coupled.csv (columns raw_count_sha256_A/B), and its
outputs equal those of the reference module on the seeded fixtures under tests/golden
(see tests/test_oracle_golden.py).
"""

from __future__ import annotations

import ctypes
import hashlib
import os
import types
from pathlib import Path

import numpy as np
from scipy.optimize import NoConvergence, anderson

HOT, COLD, INTERNAL = 0, 1, 2
SIGMA = 5.670374419e-8  # porerad/constants.py:3
SUPPORT_DIAGONAL_FRACTION = 1.0e-15  # porerad/exchange.py:30
CLOSURE_TOLERANCE = 1.0e-10  # porerad/exchange.py:31
RADIOSITY_RTOL_FINAL = 1.0e-13  # porerad/coupled.py:38

_EDGE = 1.0e-12  # view_factors.py:30, face-edge inset of ray origins
_WALL_INSET = 1.0e-9  # view_factors.py:88, 106-107
_TINY = np.finfo(np.float64).tiny
_LOG_MAX = float(np.log(np.finfo(np.float64).max))
_LOG_MIN = float(np.log(np.nextafter(0.0, 1.0)))
# tangent axes (first, second) of a face whose normal lies along axis 0, 1, 2 (view_factors.py:159-164, 174)
_TANGENT = np.array([[1, 2], [0, 2], [0, 1]], dtype=np.int64)

_HERE = Path(__file__).resolve().parent
_LIB = None


def library_path() -> Path:
    return _HERE / "liboracle_dda.so"


def _lib():
    global _LIB
    if _LIB is None:
        path = library_path()
        if not path.is_file():
            raise RuntimeError(f"oracle traversal library missing: build it with `python {_HERE / 'build.py'}`")
        lib = ctypes.CDLL(str(path))
        lib.oracle_trace.restype = None
        lib.oracle_trace.argtypes = [ctypes.c_void_p, ctypes.c_long, ctypes.c_long, ctypes.c_long,
                                     ctypes.c_void_p, ctypes.c_void_p, ctypes.c_long, ctypes.c_void_p,
                                     ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                     ctypes.c_void_p]
        _LIB = lib
    return _LIB


# --------------------------------------------------------------------------- patches

def orient_along_x(array: np.ndarray, axis: str) -> np.ndarray:
    """view_factors.py:37-40: transfer axis moved to index 0, C-contiguous."""

    return np.ascontiguousarray(np.moveaxis(np.asarray(array), "xyz".index(axis), 0))


def build_surface_patches(phases_x: np.ndarray, H_m: float):
    """view_factors.py:70-132.

    Walls first in (j, k, hot-before-cold) order where the boundary cell is pore; then
    the exposed faces of solid cells in (i, j, k, face) order, lateral neighbours
    periodic, no internal patch on the x boundary faces.
    """

    solid = np.ascontiguousarray((np.asarray(phases_x) == 1).astype(np.uint8))
    nx, ny, nz = solid.shape
    s = solid.astype(bool)
    area = (float(H_m) / nx) ** 2

    open_wall = np.stack((~s[0], ~s[-1]), axis=-1)  # (ny, nz, 2): hot, cold
    flat = np.flatnonzero(open_wall.ravel())
    wj, rem = np.divmod(flat, nz * 2)
    wk, wc = np.divmod(rem, 2)
    n_wall = flat.size
    w_origin = np.column_stack((
        np.where(wc == 0, _WALL_INSET, float(nx) - _WALL_INSET),
        wj.astype(np.float64) + 0.5,
        wk.astype(np.float64) + 0.5,
    ))
    w_normal = np.zeros((n_wall, 3))
    w_normal[:, 0] = np.where(wc == 0, 1.0, -1.0)

    mask = np.zeros(solid.shape + (6,), dtype=bool)
    mask[:-1, ..., 0] = s[:-1] & ~s[1:]
    mask[1:, ..., 1] = s[1:] & ~s[:-1]
    mask[..., 2] = s & ~np.roll(s, -1, axis=1)
    mask[..., 3] = s & ~np.roll(s, 1, axis=1)
    mask[..., 4] = s & ~np.roll(s, -1, axis=2)
    mask[..., 5] = s & ~np.roll(s, 1, axis=2)
    flat = np.flatnonzero(mask.ravel())
    cell, face = np.divmod(flat, 6)
    ci, rem = np.divmod(cell, ny * nz)
    cj, ck = np.divmod(rem, nz)
    n_int = face.size
    axis = face // 2
    sign = np.where(face % 2 == 0, 1.0, -1.0)
    i_normal = np.zeros((n_int, 3))
    i_normal[np.arange(n_int), axis] = sign
    i_origin = np.column_stack((ci, cj, ck)).astype(np.float64) + 0.5
    offset = 0.5 + _WALL_INSET
    rows = np.arange(n_int)
    i_origin[rows, axis] = np.where(sign > 0, i_origin[rows, axis] + offset, i_origin[rows, axis] - offset)
    i_origin[:, 1] = np.remainder(i_origin[:, 1], ny)
    i_origin[:, 2] = np.remainder(i_origin[:, 2], nz)

    P = n_wall + n_int
    cell_face_patch = np.full((nx * ny * nz, 6), -1, dtype=np.int32)
    cell_face_patch[cell, face] = np.arange(n_wall, P, dtype=np.int32)
    hot_map = np.full((ny, nz), -1, dtype=np.int32)
    cold_map = np.full((ny, nz), -1, dtype=np.int32)
    ids = np.arange(n_wall, dtype=np.int32)
    hot_map[wj[wc == 0], wk[wc == 0]] = ids[wc == 0]
    cold_map[wj[wc == 1], wk[wc == 1]] = ids[wc == 1]
    return types.SimpleNamespace(
        solid=solid,
        patch_class=np.concatenate((wc.astype(np.int8), np.full(n_int, INTERNAL, np.int8))),
        patch_cell=np.concatenate((np.full(n_wall, -1, np.int32), cell.astype(np.int32))),
        patch_face=np.concatenate((np.full(n_wall, -1, np.int8), face.astype(np.int8))),
        patch_origin=np.ascontiguousarray(np.vstack((w_origin, i_origin))),
        patch_normal=np.ascontiguousarray(np.vstack((w_normal, i_normal))),
        patch_area_m2=np.full(P, area),
        cell_face_patch=cell_face_patch,
        hot_wall_patch=hot_map,
        cold_wall_patch=cold_map,
        H_m=float(H_m),
        n_patches=P,
    )


# --------------------------------------------------------------------------- rays

def generate_rays(patches, patch_start: int, patch_end: int, rays_per_patch: int, seed: int):
    """view_factors.py:135-182.

    Ray (p, r) takes draws (p*R + r)*4 + c, c = 0..3, of PCG64(seed): c = 0, 1 place
    the origin on the face (clipped 1e-12 from its edges), c = 2, 3 give the
    cosine-weighted direction; y, z origins wrap periodically; directions are
    divided by their Euclidean norm.
    """

    p0, p1, R = int(patch_start), int(patch_end), int(rays_per_patch)
    bitgen = np.random.PCG64(int(seed))
    bitgen.advance(p0 * R * 4)
    u = np.random.Generator(bitgen).random((p1 - p0) * R * 4, dtype=np.float64).reshape(-1, 4)
    normal = patches.patch_normal[p0:p1]
    axis = np.argmax(normal != 0.0, axis=1)
    sign = normal[np.arange(p1 - p0), axis]
    axis = np.repeat(axis, R)
    sign = np.repeat(sign, R)
    n = axis.size
    rows = np.arange(n)
    first, second = _TANGENT[axis, 0], _TANGENT[axis, 1]

    origin = np.repeat(patches.patch_origin[p0:p1], R, axis=0)
    origin[rows, first] += np.clip(u[:, 0], _EDGE, 1.0 - _EDGE) - 0.5
    origin[rows, second] += np.clip(u[:, 1], _EDGE, 1.0 - _EDGE) - 0.5
    ny, nz = patches.solid.shape[1], patches.solid.shape[2]
    origin[:, 1] = np.remainder(origin[:, 1], ny)
    origin[:, 2] = np.remainder(origin[:, 2], nz)

    radius = np.sqrt(u[:, 2])
    azimuth = (2.0 * np.pi) * u[:, 3]
    lat_a = radius * np.cos(azimuth)
    lat_b = radius * np.sin(azimuth)
    polar = np.sqrt(1.0 - u[:, 2])
    d = np.empty((n, 3))
    d[rows, axis] = sign * polar
    d[rows, first] = lat_a
    d[rows, second] = sign * lat_b
    length = np.sqrt((d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1]) + d[:, 2] * d[:, 2])
    d = d / length[:, None]
    return np.ascontiguousarray(origin), np.ascontiguousarray(d)


def trace_first_hit(patches, origins, directions, *, return_steps: bool = False):
    """view_factors.py:261-270 over the C traversal of oracle/dda.c (view_factors.py:185-258)."""

    solid = np.ascontiguousarray(patches.solid, dtype=np.uint8)
    nx, ny, nz = solid.shape
    o = np.ascontiguousarray(origins, dtype=np.float64)
    d = np.ascontiguousarray(directions, dtype=np.float64)
    n = o.shape[0]
    hot = np.ascontiguousarray(patches.hot_wall_patch, dtype=np.int32)
    cold = np.ascontiguousarray(patches.cold_wall_patch, dtype=np.int32)
    cfp = np.ascontiguousarray(patches.cell_face_patch, dtype=np.int32)
    receiver = np.empty(n, dtype=np.int32)
    failed = np.empty(n, dtype=np.uint8)
    steps = np.empty(n, dtype=np.int64) if return_steps else None
    _lib().oracle_trace(solid.ctypes.data, nx, ny, nz, o.ctypes.data, d.ctypes.data, n,
                        hot.ctypes.data, cold.ctypes.data, cfp.ctypes.data, receiver.ctypes.data,
                        failed.ctypes.data, steps.ctypes.data if steps is not None else None)
    bad = int(np.count_nonzero(failed))
    if bad:
        raise RuntimeError(f"{bad} rays did not resolve a receiving patch")
    return (receiver, steps) if return_steps else receiver


def first_hit_counts(patches, rays_per_patch: int, seed: int, *, patch_chunk: int = 16384, stats=None,
                     patch_start: int = 0, patch_end: int | None = None):
    """view_factors.py:273-287: per chunk of patches, unique (origin, receiver) pairs and counts.

    ``patch_start`` and ``patch_end`` (not in the reference) restrict the origins to
    ``[patch_start, patch_end)``, for parity on a slice and for timing a bounded sample;
    the rays of those origins are the ones a full pass draws (the stream is advanced by
    ``start * R * 4``) and the pair keys still span all patches.
    """

    n = patches.n_patches
    R = int(rays_per_patch)
    last = n if patch_end is None else min(int(patch_end), n)
    parts = []
    for start in range(max(0, int(patch_start)), last, int(patch_chunk)):
        end = min(start + int(patch_chunk), last)
        o, d = generate_rays(patches, start, end, R, seed)
        if stats is not None:
            rec, steps = trace_first_hit(patches, o, d, return_steps=True)
            stats["steps"] = stats.get("steps", 0) + int(steps.sum())
            stats["rays"] = stats.get("rays", 0) + int(steps.size)
        else:
            rec = trace_first_hit(patches, o, d)
        key = np.repeat(np.arange(start, end, dtype=np.int64), R) * n + rec.astype(np.int64)
        key, cnt = np.unique(key, return_counts=True)
        parts.append(((key // n).astype(np.int32), (key % n).astype(np.int32), cnt.astype(np.int64)))
    return pool_counts(parts, n)


def pool_counts(tables, n_patches: int):
    """view_factors.py:290-300: sum the counts of equal (origin, receiver) pairs, sorted by pair."""

    n = int(n_patches)
    key = np.concatenate([np.asarray(o, np.int64) * n + np.asarray(r, np.int64) for o, r, _ in tables])
    cnt = np.concatenate([np.asarray(c, np.int64) for _, _, c in tables])
    order = np.argsort(key, kind="stable")
    key, cnt = key[order], cnt[order]
    head = np.flatnonzero(np.r_[True, key[1:] != key[:-1]])
    uk = key[head]
    return (uk // n).astype(np.int32), (uk % n).astype(np.int32), np.add.reduceat(cnt, head)


def count_sha256(origin, receiver, count, rays_per_origin) -> str:
    """view_factors.py:303-323: name, dtype string, int64 shape and C-order bytes of each array."""

    h = hashlib.sha256()
    for name, arr in (("origin_patch_id", np.asarray(origin, np.int32)),
                      ("receiver_patch_id", np.asarray(receiver, np.int32)),
                      ("count", np.asarray(count, np.int64)),
                      ("rays_per_origin", np.asarray(rays_per_origin, np.int64))):
        h.update(name.encode("ascii"))
        h.update(arr.dtype.str.encode("ascii"))
        h.update(np.asarray(arr.shape, np.int64).tobytes())
        h.update(np.ascontiguousarray(arr).tobytes())
    return h.hexdigest()


# --------------------------------------------------------------------------- operator

class ExchangeOperator:
    """exchange.py:37-197: S = 0.5 (A F + F^T A) + delta A, d * (S d) = A by Anderson on log d.

    F x and F^T x are bincount scatters over the pooled edge list (exchange.py:82-106).
    """

    def __init__(self, origin, receiver, count, rays_per_origin, patch_area_m2, *,
                 support_diagonal_fraction=SUPPORT_DIAGONAL_FRACTION, balance_tolerance=1.0e-11,
                 event_chunk_size=4_000_000):
        rays = np.asarray(rays_per_origin, dtype=np.int64)
        n = rays.size
        o, r, c = pool_counts([(origin, receiver, count)], n)  # exchange.py:59-67
        observed = np.zeros(n, dtype=np.int64)
        np.add.at(observed, o, c)
        if not np.array_equal(observed, rays):  # exchange.py:68-71
            raise ValueError("first-hit counts do not account for every emitted ray")
        self.origin, self.receiver = o, r
        self.weight = c.astype(np.float64) / rays[o]
        self.patch_area_m2 = np.asarray(patch_area_m2, dtype=np.float64).copy()
        self.support_diagonal_fraction = float(support_diagonal_fraction)
        self.event_chunk_size = int(event_chunk_size)
        self.n_patches = n
        self.spmv_count = 0
        self.scale, self.balance_method, self.balance_iterations = self._balance(float(balance_tolerance))
        self.row_sum_error = float(np.max(np.abs(self.matvec(np.ones(n)) - 1.0)))  # exchange.py:78-80
        if self.row_sum_error > CLOSURE_TOLERANCE:
            raise RuntimeError(f"projected rows do not close: {self.row_sum_error:.3e}")

    def _scatter(self, rows, cols, x):
        out = np.zeros(self.n_patches)
        step = self.event_chunk_size
        for a in range(0, self.weight.size, step):
            b = min(a + step, self.weight.size)
            out += np.bincount(rows[a:b], weights=self.weight[a:b] * x[cols[a:b]], minlength=self.n_patches)
        return out

    def raw_matvec(self, x):  # exchange.py:82-93
        return self._scatter(self.origin, self.receiver, x)

    def raw_rmatvec(self, x):  # exchange.py:95-106
        return self._scatter(self.receiver, self.origin, x)

    def symmetric_matvec(self, x):  # exchange.py:108-112
        self.spmv_count += 1
        a = self.patch_area_m2
        return 0.5 * (a * self.raw_matvec(x) + self.raw_rmatvec(a * x)) + self.support_diagonal_fraction * a * x

    def matvec(self, x):  # exchange.py:114-117
        return (self.scale / self.patch_area_m2) * self.symmetric_matvec(self.scale * x)

    def rmatvec(self, x):  # exchange.py:119-122
        return self.scale * self.symmetric_matvec(self.scale * (x / self.patch_area_m2))

    def reciprocity_error(self):  # exchange.py:124-140
        n, d, a = self.n_patches, self.scale, self.patch_area_m2
        fwd = self.origin.astype(np.int64) * n + self.receiver
        rev = self.receiver.astype(np.int64) * n + self.origin
        pos = np.minimum(np.searchsorted(fwd, rev), fwd.size - 1)
        w_rev = np.where(fwd[pos] == rev, self.weight[pos], 0.0)
        i, j = self.origin, self.receiver
        s_ij = 0.5 * (a[i] * self.weight + a[j] * w_rev)
        s_ji = 0.5 * (a[j] * w_rev + a[i] * self.weight)
        diag = i == j
        s_ij[diag] += self.support_diagonal_fraction * a[i[diag]]
        s_ji[diag] += self.support_diagonal_fraction * a[j[diag]]
        jij = a[i] * ((d[i] / a[i]) * s_ij * d[j])
        jji = a[j] * ((d[j] / a[j]) * s_ji * d[i])
        return float(np.max(np.abs(jij - jji)) / max(float(np.max(np.abs(jij))), _TINY))

    def _finite_log(self, y):
        return np.all(np.isfinite(y)) and np.max(y) < _LOG_MAX and np.min(y) > _LOG_MIN

    def _closure_error(self, y):  # exchange.py:142-151
        if not self._finite_log(y):
            return float("inf")
        d = np.exp(y)
        row = d * self.symmetric_matvec(d)
        if not np.all(np.isfinite(row)) or np.any(row <= 0.0):
            return float("inf")
        return float(np.max(np.abs(row / self.patch_area_m2 - 1.0)))

    def _balance(self, tol):  # exchange.py:153-197
        n = self.n_patches
        log_a = np.log(self.patch_area_m2)
        y0 = np.zeros(n)
        if self._closure_error(y0) <= tol:
            return np.exp(y0), "none", 0
        count = [0]

        def residual(y):
            y = np.asarray(y, dtype=np.float64)
            if not self._finite_log(y):
                return np.full(n, np.inf)
            prod = self.symmetric_matvec(np.exp(y))
            if not np.all(np.isfinite(prod)) or np.any(prod <= 0.0):
                return np.full(n, np.inf)
            return y + np.log(prod) - log_a

        def tick(_x, _f):
            count[0] += 1

        try:
            y = np.asarray(anderson(residual, y0, M=10, w0=0.01, maxiter=500, f_tol=tol, callback=tick),
                           dtype=np.float64)
            if self._closure_error(y) <= min(max(10.0 * tol, 10.0 * np.finfo(float).eps), CLOSURE_TOLERANCE):
                return np.exp(y), "anderson", count[0]
        except (NoConvergence, ValueError, FloatingPointError, np.linalg.LinAlgError):
            pass
        y = y0.copy()
        for it in range(1, 20_001):
            d = np.exp(y)
            row = d * self.symmetric_matvec(d)
            if not np.all(np.isfinite(row)) or np.any(row <= 0.0):
                break
            y = y + 0.5 * (log_a - np.log(row))
            err = self._closure_error(y)
            if not np.isfinite(err):
                break
            if err <= min(tol, CLOSURE_TOLERANCE):
                return np.exp(y), "multiplicative", it
        raise RuntimeError("diagonal balancing of the exchange matrix did not converge")


# --------------------------------------------------------------------------- radiosity

def reflection_series(operator, emitted_W, emissivity, *, relative_tolerance, max_reflections=10000):
    """exchange.py:217-245: flight <- (1 - eps) F_p^T flight, absorbed += eps F_p^T flight."""

    e = np.asarray(emitted_W, dtype=np.float64)
    absorbed = np.zeros_like(e)
    flight = e.copy()
    ref = max(float(np.sum(np.abs(e))), _TINY)
    for it in range(1, int(max_reflections) + 1):
        inc = operator.rmatvec(flight)
        absorbed += emissivity * inc
        flight = (1.0 - emissivity) * inc
        if float(np.sum(np.abs(flight))) <= float(relative_tolerance) * ref:
            break
    else:
        raise RuntimeError("radiosity reflection series did not converge")
    return types.SimpleNamespace(emitted_power_W=e, absorbed_power_W=absorbed, net_power_W=absorbed - e,
                                 residual_power_W=float(np.sum(flight)), iterations=it)


def net_patch_power(operator, temperature_K, emissivity, area_m2, *, relative_tolerance,
                    reference_temperature_K=None):
    """exchange.py:248-271: signed emission eps sigma A (T^4 - T_ref^4) in factored form."""

    T = np.asarray(temperature_K, dtype=np.float64)
    if reference_temperature_K is None:
        e = emissivity * SIGMA * area_m2 * T**4
    else:
        t0 = float(reference_temperature_K)
        e = emissivity * SIGMA * area_m2 * ((T - t0) * (T + t0) * (T * T + t0 * t0))
    return reflection_series(operator, e, emissivity, relative_tolerance=relative_tolerance)


def net_patch_power_jvp(operator, temperature_K, delta_temperature_K, emissivity, area_m2, *, relative_tolerance):
    """exchange.py:274-287."""

    de = 4.0 * emissivity * SIGMA * area_m2 * temperature_K**3 * delta_temperature_K
    res = reflection_series(operator, de, emissivity, relative_tolerance=relative_tolerance)
    return res.absorbed_power_W - de


# --------------------------------------------------------------------------- channels (callers)

def patch_temperature(patches, T_cells, T_hot_K, T_cold_K):  # coupled.py:45-53
    T = np.empty(patches.n_patches)
    cls = patches.patch_class
    T[cls == HOT] = float(T_hot_K)
    T[cls == COLD] = float(T_cold_K)
    inner = cls == INTERNAL
    T[inner] = np.asarray(T_cells, dtype=np.float64).ravel()[patches.patch_cell[inner]]
    return T


def cell_power(patches, patch_power_W):  # coupled.py:56-62
    inner = patches.patch_class == INTERNAL
    out = np.zeros(patches.solid.size)
    np.add.at(out, patches.patch_cell[inner], patch_power_W[inner])
    return out.reshape(patches.solid.shape)


def linear_cell_temperature(shape, T_mean_K, delta_T_K):  # coupled.py:138-143
    nx = int(shape[0])
    axial = (T_mean_K + delta_T_K / 2.0) - (np.arange(nx, dtype=np.float64) + 0.5) * delta_T_K / nx
    return np.broadcast_to(axial[:, None, None], tuple(int(s) for s in shape)).copy()


def coarse_source(cell_power_W, bins=8):  # coupled.py:146-153
    arr = np.asarray(cell_power_W, dtype=np.float64)
    parts = [np.array_split(np.arange(n), min(bins, n)) for n in arr.shape]
    return np.asarray([float(np.sum(arr[np.ix_(a, b, c)])) for a in parts[0] for b in parts[1] for c in parts[2]]
                      ).reshape(tuple(len(p) for p in parts))


def cross_section_area(patches):  # coupled.py:129-133
    nx, ny, nz = patches.solid.shape
    return float(ny * nz) * (patches.H_m / float(nx)) ** 2


def prescribed_field_channels(operator, patches, T_mean_K, delta_T_K, epsilon):  # coupled.py:170-194
    T_cells = linear_cell_temperature(patches.solid.shape, T_mean_K, delta_T_K)
    Tp = patch_temperature(patches, T_cells, T_mean_K + delta_T_K / 2.0, T_mean_K - delta_T_K / 2.0)
    eps = np.full(patches.n_patches, float(epsilon))
    rad = net_patch_power(operator, Tp, eps, patches.patch_area_m2, relative_tolerance=RADIOSITY_RTOL_FINAL,
                          reference_temperature_K=T_mean_K)
    area = cross_section_area(patches)
    net = rad.net_power_W
    cls = patches.patch_class
    q_h = -float(np.sum(net[cls == HOT])) / area
    q_c = -float(np.sum(net[cls == COLD])) / area
    q_i = -float(np.sum(net[cls == INTERNAL])) / area
    closure = abs(q_h + q_c + q_i) / max(abs(q_h), abs(q_c), abs(q_i), 1.0e-30)
    return types.SimpleNamespace(T_mean_K=float(T_mean_K), delta_T_K=float(delta_T_K), epsilon=float(epsilon),
                                 q_h=q_h, q_c=q_c, q_i=q_i, closure_rel=closure,
                                 coarse_source=coarse_source(cell_power(patches, net)) / area,
                                 radiosity=rad)


def relative_difference(a, b):  # coupled.py:197-198
    return abs(float(a) - float(b)) / max(abs(float(a)), abs(float(b)), _TINY)


def ab_differences(set_a, set_b):  # coupled.py:201-213
    channel = max(relative_difference(getattr(a, k), getattr(b, k)) for a, b in zip(set_a, set_b) for k in ("q_h", "q_c"))
    source = max(float(np.sum(np.abs(a.coarse_source - b.coarse_source)))
                 / max(float(np.sum(np.abs(a.coarse_source))), float(np.sum(np.abs(b.coarse_source))), _TINY)
                 for a, b in zip(set_a, set_b))
    return channel, source


def append_required(channel_difference, source_difference):  # coupled.py:216-219
    return channel_difference > 0.01 or source_difference > 0.05


# --------------------------------------------------------------------------- conduction (conduction.py)

K_SOLID = 0.20  # porerad/constants.py:8
K_GAS = 0.026   # porerad/constants.py:11


def assemble_conduction(conductivity_x, H_m):
    """conduction.py:53-92: face conductance 2 k1 k2 / (k1 + k2 + 1e-30) * dx^2 / dx between
    neighbours (x open, y and z periodic), 2 k dx to the walls; A as a SciPy CSR matrix."""

    from scipy.sparse import coo_matrix

    k = np.ascontiguousarray(conductivity_x, dtype=np.float64)
    nx, ny, nz = k.shape
    dx = float(H_m) / nx
    idx = np.arange(k.size, dtype=np.int64).reshape(k.shape)
    diag = np.zeros(k.size)
    rows, cols, vals = [], [], []
    faces = [(idx[:-1], idx[1:], k[:-1], k[1:]),
             (idx[:, :-1], idx[:, 1:], k[:, :-1], k[:, 1:]), (idx[:, -1], idx[:, 0], k[:, -1], k[:, 0]),
             (idx[:, :, :-1], idx[:, :, 1:], k[:, :, :-1], k[:, :, 1:]),
             (idx[:, :, -1], idx[:, :, 0], k[:, :, -1], k[:, :, 0])]
    for lo, hi, klo, khi in faces:
        g = (2.0 * klo * khi / (klo + khi + 1.0e-30) * (dx * dx) / dx).ravel()
        lo, hi = lo.ravel(), hi.ravel()
        diag[lo] += g
        diag[hi] += g
        rows += [lo, hi]
        cols += [hi, lo]
        vals += [-g, -g]
    hot = np.zeros(k.size)
    cold = np.zeros(k.size)
    hot.reshape(k.shape)[0] = 2.0 * k[0] * (dx * dx / dx)
    cold.reshape(k.shape)[-1] = 2.0 * k[-1] * (dx * dx / dx)
    diag += hot + cold
    rows.append(idx.ravel())
    cols.append(idx.ravel())
    vals.append(diag)
    A = coo_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))),
                   shape=(k.size, k.size)).tocsc().tocsr()
    A.sum_duplicates()
    A.sort_indices()
    return types.SimpleNamespace(matrix=A, hot_rhs=hot, cold_rhs=cold, conductivity=k, H_m=float(H_m),
                                 shape=k.shape)


def boundary_rhs(system, T_hot_K, T_cold_K):  # conduction.py:37-40
    return system.hot_rhs * float(T_hot_K) + system.cold_rhs * float(T_cold_K)


def solve_conduction(system, T_hot_K, T_cold_K, *, rtol=1.0e-11):
    """conduction.py:95-120: Jacobi-PCG (SciPy cg) from the linear wall-to-wall profile."""

    from scipy.sparse.linalg import LinearOperator, cg

    A = system.matrix
    b = boundary_rhs(system, T_hot_K, T_cold_K)
    nx = system.shape[0]
    line = float(T_hot_K) + (float(T_cold_K) - float(T_hot_K)) * ((np.arange(nx) + 0.5) / nx)
    x0 = np.broadcast_to(line[:, None, None], system.shape).reshape(-1).copy()
    inv = 1.0 / A.diagonal()
    M = LinearOperator(A.shape, matvec=lambda v: inv * v, dtype=np.float64)
    T, info = cg(A, b, x0=x0, rtol=float(rtol), atol=0.0, maxiter=max(50000, 20 * nx), M=M)
    rel = float(np.linalg.norm(A @ T - b) / np.linalg.norm(b))
    if info != 0 or rel > 1.0e-9:
        raise RuntimeError(f"conduction solve did not converge: info={info}, residual={rel:.3e}")
    return T.reshape(system.shape)


def wall_fluxes(system, T, T_hot_K, T_cold_K):  # conduction.py:43-50
    k = system.conductivity
    T = np.asarray(T, dtype=np.float64).reshape(system.shape)
    dx = system.H_m / k.shape[0]
    return (float(np.mean(2.0 * k[0] * (float(T_hot_K) - T[0]) / dx)),
            float(np.mean(2.0 * k[-1] * (T[-1] - float(T_cold_K)) / dx)))


# --------------------------------------------------------------------------- coupled solve (coupled.py:222-490)

def emission_diagonal(patches, T_cells, epsilon):  # coupled.py:65-73
    inner = patches.patch_class == INTERNAL
    owner = patches.patch_cell[inner].astype(np.int64)
    T = np.asarray(T_cells, dtype=np.float64).ravel()[owner]
    d = np.zeros(patches.solid.size)
    np.add.at(d, owner, 4.0 * float(epsilon) * SIGMA * patches.patch_area_m2[inner] * T**3)
    return d


def _radiation(operator, patches, T_cells, T_hot_K, T_cold_K, epsilon, rtol):  # coupled.py:86-105
    Tp = patch_temperature(patches, T_cells, T_hot_K, T_cold_K)
    eps = np.full(patches.n_patches, float(epsilon))
    rad = net_patch_power(operator, Tp, eps, patches.patch_area_m2, relative_tolerance=rtol)
    return types.SimpleNamespace(patch_temperature_K=Tp, patch_net_power_W=rad.net_power_W,
                                 cell_net_power_W=cell_power(patches, rad.net_power_W), radiosity=rad)


def _radiation_jvp(operator, patches, T_patch, dT_cells, epsilon, rtol):  # coupled.py:108-126
    inner = patches.patch_class == INTERNAL
    dTp = np.zeros(patches.n_patches)
    dTp[inner] = np.asarray(dT_cells, dtype=np.float64).ravel()[patches.patch_cell[inner]]
    eps = np.full(patches.n_patches, float(epsilon))
    return cell_power(patches, net_patch_power_jvp(operator, T_patch, dTp, eps, patches.patch_area_m2,
                                                   relative_tolerance=rtol))


def flexible_gmres(matvec, rhs, precondition, *, restart, max_iterations, relative_tolerance, absolute_tolerance):
    """coupled.py:230-290: right-preconditioned flexible GMRES, modified Gram-Schmidt with one
    reorthogonalisation, least squares on the Hessenberg, confirmed by the true residual."""

    b = np.asarray(rhs, dtype=np.float64)
    x = np.zeros_like(b)
    bn = max(float(np.linalg.norm(b)), _TINY)
    thr = max(float(absolute_tolerance), float(relative_tolerance) * bn)
    eps = np.finfo(np.float64).eps
    done = 0
    while done < max_iterations:
        r = b - matvec(x)
        beta = float(np.linalg.norm(r))
        if beta <= thr:
            return x, True, done, beta / bn
        m = min(restart, max_iterations - done)
        V = np.zeros((m + 1, b.size))
        Z = np.zeros((m, b.size))
        H = np.zeros((m + 1, m))
        g = np.zeros(m + 1)
        V[0] = r / beta
        g[0] = beta
        restart_x = None
        for j in range(m):
            Z[j] = precondition(V[j])
            w = matvec(Z[j])
            for _ in range(2):
                for i in range(j + 1):
                    h = float(np.dot(V[i], w))
                    H[i, j] += h
                    w -= h * V[i]
            nn = float(np.linalg.norm(w))
            H[j + 1, j] = nn
            if nn > eps * beta:
                V[j + 1] = w / nn
            y = np.linalg.lstsq(H[: j + 2, : j + 1], g[: j + 2], rcond=None)[0]
            est = float(np.linalg.norm(g[: j + 2] - H[: j + 2, : j + 1] @ y))
            done += 1
            if est <= thr or nn <= eps * beta:
                cand = x + y @ Z[: j + 1]
                tn = float(np.linalg.norm(b - matvec(cand)))
                if tn <= thr:
                    return cand, True, done, tn / bn
                restart_x = cand
                break
        if restart_x is not None:
            x = restart_x
            continue
        x = x + np.linalg.lstsq(H, g, rcond=None)[0] @ Z
    tn = float(np.linalg.norm(b - matvec(x)))
    return x, tn <= thr, done, tn / bn


def _fixed_pcg(A, shift, steps):  # coupled.py:293-320: fixed Jacobi-PCG steps on A + diag(shift) from x = 0
    inv = 1.0 / (A.diagonal() + shift)

    def apply(rhs):
        x = np.zeros_like(rhs)
        r = rhs.copy()
        z = inv * r
        p = z.copy()
        rz = r @ z
        for step in range(steps):
            Ap = A @ p + shift * p
            a = rz / (p @ Ap)
            x += a * p
            r -= a * Ap
            z = inv * r
            if step + 1 < steps:
                rzn = r @ z
                p = z + (rzn / rz) * p
                rz = rzn
        return x

    return apply


def newton_krylov(system, operator, patches, T_hot_K, T_cold_K, epsilon, T_initial, preconditioner_steps):
    """coupled.py:340-421."""

    A = system.matrix
    b = boundary_rhs(system, T_hot_K, T_cold_K)
    lo, hi = float(T_cold_K), float(T_hot_K)
    M = _fixed_pcg(A, emission_diagonal(patches, T_initial, epsilon), int(preconditioner_steps))
    T = np.asarray(T_initial, dtype=np.float64).copy()
    state = _radiation(operator, patches, T, T_hot_K, T_cold_K, epsilon, 1.0e-8)
    R = A @ T.ravel() - b - state.cell_net_power_W.ravel()
    last = 0.0 if max(float(np.linalg.norm(R, np.inf)), _TINY) <= 1.0e-13 else np.inf
    out = types.SimpleNamespace(converged=False, newton_iterations=0, linear_solves=[],
                                preconditioner_steps=int(preconditioner_steps), failure="")

    def finish(ok, failure=""):
        final = _radiation(operator, patches, T, T_hot_K, T_cold_K, epsilon, RADIOSITY_RTOL_FINAL)
        out.temperature_K, out.state, out.converged, out.failure = T, final, ok, failure
        out.final_residual_inf_W = float(np.linalg.norm(A @ T.ravel() - b - final.cell_net_power_W.ravel(), np.inf))
        return out

    for _ in range(8):
        rn = float(np.linalg.norm(R, np.inf))
        if rn <= 1.0e-13 and last <= 1.0e-10:
            return finish(True)
        Tp = state.patch_temperature_K.copy()

        def J(v):
            return A @ v - _radiation_jvp(operator, patches, Tp, v.reshape(system.shape), epsilon, 1.0e-8).ravel()

        step, ok, its, rel = flexible_gmres(J, -R, M, restart=30, max_iterations=90, relative_tolerance=1.0e-8,
                                            absolute_tolerance=1.0e-13)
        out.linear_solves.append(dict(converged=ok, gmres_iterations=its, rhs_l2_W=float(np.linalg.norm(R)),
                                      true_residual_l2_W=float(np.linalg.norm(J(step) + R)),
                                      true_residual_relative=rel))
        if not ok:
            return finish(False, "linear solve did not converge")
        if rn <= 1.0e-13 and float(np.max(np.abs(step))) <= 1.0e-10:
            return finish(True)
        alpha, accepted = 1.0, False
        while alpha >= 2.0**-20:
            cand = T.ravel() + alpha * step
            if np.all(np.isfinite(cand)) and float(np.min(cand)) >= lo and float(np.max(cand)) <= hi:
                trial = cand.reshape(system.shape)
                ts = _radiation(operator, patches, trial, T_hot_K, T_cold_K, epsilon, 1.0e-8)
                tr = A @ cand - b - ts.cell_net_power_W.ravel()
                tn = float(np.linalg.norm(tr, np.inf))
                if tn <= (1.0 - 1.0e-4 * alpha) * rn:
                    accepted = True
                    break
            alpha *= 0.5
        if not accepted:
            return finish(False, "line search failed")
        last = float(np.max(np.abs(trial - T)))
        T, state, R = trial, ts, tr
        out.newton_iterations += 1
        if tn <= 1.0e-13 and last <= 1.0e-10:
            return finish(True)
    return finish(False, "maximum Newton iterations reached")


def linear_residuals_pass(result):  # coupled.py:333-337
    return bool(result.linear_solves) and all(
        s["converged"] and s["true_residual_l2_W"] <= max(1.0e-13, 1.0e-8 * s["rhs_l2_W"]) for s in result.linear_solves)


def solve_coupled(system, operator, patches, T_hot_K, T_cold_K, epsilon, T_initial):  # coupled.py:423-440
    for steps in (10, 20):
        res = newton_krylov(system, operator, patches, T_hot_K, T_cold_K, epsilon, T_initial, steps)
        if res.converged and linear_residuals_pass(res):
            break
    return res


def wall_flux_metrics(system, patches, result, T_hot_K, T_cold_K):  # coupled.py:443-472
    qch, qcc = wall_fluxes(system, result.temperature_K, T_hot_K, T_cold_K)
    area = cross_section_area(patches)
    net = result.state.patch_net_power_W
    qrh = -float(np.sum(net[patches.patch_class == HOT])) / area
    qrc = float(np.sum(net[patches.patch_class == COLD])) / area
    th, tc = qch + qrh, qcc + qrc
    scale = max(abs(th), abs(tc), _TINY)
    T = result.temperature_K
    rad = result.state.radiosity
    return {"q_cond_hot_W_m2": qch, "q_rad_hot_W_m2": qrh, "q_total_hot_W_m2": th, "q_cond_cold_W_m2": qcc,
            "q_rad_cold_W_m2": qrc, "q_total_cold_W_m2": tc, "radiative_fraction_hot": qrh / th,
            "k_eff_apparent_W_mK": th * patches.H_m / (float(T_hot_K) - float(T_cold_K)),
            "wall_flux_mismatch_rel": abs(th - tc) / scale,
            "energy_residual_rel": abs(float(np.sum(rad.net_power_W) + rad.residual_power_W)) / max(scale * area, _TINY),
            "T_min_K": float(np.min(T)), "T_max_K": float(np.max(T)),
            "temperature_bound_violations": int(np.count_nonzero((T < float(T_cold_K)) | (T > float(T_hot_K))))}


def pcg64_state(seed: int):
    """(state, inc) of numpy.random.PCG64(seed) as Python ints (SeedSequence seeding)."""

    st = np.random.PCG64(int(seed)).state["state"]
    return int(st["state"]), int(st["inc"])


def set_threads(n: int | None = None) -> int:
    """Thread count for the OpenMP traversal (all host cores by default)."""

    n = int(n or os.cpu_count() or 1)
    os.environ["OMP_NUM_THREADS"] = str(n)
    return n

"""Surface patches, Lambertian ray sets and first-hit exchange counts on a B200.

Drop-in for ``porerad.view_factors`` (porerad/view_factors.py): the same names,
signatures, dtypes, orderings and exceptions, computed by libporerad on the GPU.
All arrays use the orientation in which the transfer axis is x: the hot wall lies
at x = 0, the cold wall at x = N_x, y and z are periodic; positions are in cell
widths.

Beyond the reference API, :func:`first_hit_counts_pooled` traces several seeded
blocks in one device pass and returns a device-resident :class:`CountTable` that
:class:`porerad_b200.exchange.ExchangeOperator` accepts without a host round trip.
"""

from __future__ import annotations

import ctypes
import hashlib

import numpy as np

from . import _lib

HOT, COLD, INTERNAL = 0, 1, 2
"""Patch classes: hot wall, cold wall, solid-pore interface (view_factors.py:25)."""

_AXIS_INDEX = {"x": 0, "y": 1, "z": 2}

_FIELDS = ("solid", "patch_class", "patch_cell", "patch_face", "patch_origin", "patch_normal", "patch_area_m2",
           "cell_face_patch", "hot_wall_patch", "cold_wall_patch")


def orient_along_x(array: np.ndarray, axis: str) -> np.ndarray:
    """Return ``array`` with the requested transfer axis moved to the first index (view_factors.py:37-40)."""

    return np.ascontiguousarray(np.moveaxis(np.asarray(array), _AXIS_INDEX[axis], 0))


class DeviceGeometry:
    """One x-oriented voxel geometry resident on the current CUDA device (a ``pr_case``)."""

    def __init__(self, phases_x, H_m: float, *, stream=None):
        if getattr(phases_x, "is_cuda", False):
            # a contiguous uint8 CUDA tensor already resident in HBM
            if str(phases_x.dtype) != "torch.uint8" or not phases_x.is_contiguous() or phases_x.dim() != 3:
                raise ValueError("device phases must be a contiguous 3-D uint8 tensor")
            src = int(phases_x.data_ptr())
            shape = tuple(int(s) for s in phases_x.shape)
        else:
            ph = np.asarray(phases_x)
            if ph.ndim != 3:
                raise ValueError("phases_x must be a 3-D array")
            if ph.dtype != np.uint8:
                ph = (ph == 1).astype(np.uint8)
            ph = np.ascontiguousarray(ph)
            src = ph.ctypes.data
            shape = tuple(int(s) for s in ph.shape)
        lib = _lib.load()
        out = ctypes.c_void_p()
        nx, ny, nz = shape
        st = _lib.stream_arg(stream) if stream is not None else _lib.stream()
        _lib.check(lib.pr_case_create(src, nx, ny, nz, float(H_m), st, ctypes.byref(out)))
        self._h = _lib.Handle(out.value, "pr_case_destroy")
        self.shape = (nx, ny, nz)
        self.H_m = float(H_m)
        n_p, n_w, nbytes = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_size_t()
        _lib.check(lib.pr_case_info(self.handle, ctypes.byref(n_p), ctypes.byref(n_w), ctypes.byref(nbytes)))
        self.n_patches = int(n_p.value)
        self.n_wall = int(n_w.value)
        self.device_bytes = int(nbytes.value)

    @property
    def handle(self) -> int:
        return self._h.value

    def close(self) -> None:
        self._h.close()

    def fetch(self, *names: str) -> dict[str, np.ndarray]:
        """Copy the requested SurfacePatches arrays to the host."""

        nx, ny, nz = self.shape
        P = self.n_patches
        shapes = {
            "solid": ((nx, ny, nz), np.uint8), "patch_class": ((P,), np.int8), "patch_cell": ((P,), np.int32),
            "patch_face": ((P,), np.int8), "patch_origin": ((P, 3), np.float64),
            "patch_normal": ((P, 3), np.float64), "patch_area_m2": ((P,), np.float64),
            "cell_face_patch": ((nx * ny * nz, 6), np.int32), "hot_wall_patch": ((ny, nz), np.int32),
            "cold_wall_patch": ((ny, nz), np.int32),
        }
        out = {n: np.empty(*shapes[n]) for n in names}
        args = [_lib.ptr(out.get(n)) for n in _FIELDS]
        _lib.check(_lib.load().pr_case_patches(self.handle, *args, _lib.stream()))
        return out


class SurfacePatches:
    """Patch table of one digital microstructure oriented along x (view_factors.py:43-67).

    ``patch_class`` is HOT, COLD or INTERNAL.  An internal patch is the face
    ``patch_face`` (0..5 for +x, -x, +y, -y, +z, -z) of the solid cell
    ``patch_cell`` (flat C index).  ``cell_face_patch``, ``hot_wall_patch`` and
    ``cold_wall_patch`` map a hit face back to its patch index.

    Tables made by :func:`build_surface_patches` live on the GPU and are copied to
    the host field by field on first access.
    """

    def __init__(self, solid=None, patch_class=None, patch_cell=None, patch_face=None, patch_origin=None,
                 patch_normal=None, patch_area_m2=None, cell_face_patch=None, hot_wall_patch=None,
                 cold_wall_patch=None, H_m=None, *, _device: DeviceGeometry | None = None):
        self._host: dict[str, np.ndarray] = {}
        given = dict(solid=solid, patch_class=patch_class, patch_cell=patch_cell, patch_face=patch_face,
                     patch_origin=patch_origin, patch_normal=patch_normal, patch_area_m2=patch_area_m2,
                     cell_face_patch=cell_face_patch, hot_wall_patch=hot_wall_patch,
                     cold_wall_patch=cold_wall_patch)
        for k, v in given.items():
            if v is not None:
                self._host[k] = v
        self._device = _device
        if _device is None:
            missing = [k for k, v in given.items() if v is None]
            if missing or H_m is None:
                raise TypeError(f"SurfacePatches needs every field; missing {missing + (['H_m'] if H_m is None else [])}")
        self.H_m = float(H_m if H_m is not None else _device.H_m)

    def _get(self, name: str) -> np.ndarray:
        if name not in self._host:
            self._host.update(self._device.fetch(name))
        return self._host[name]

    def _set(self, name: str, value) -> None:
        self._host[name] = value
        self._device = None if self._device is not None and name == "solid" else self._device

    @property
    def n_patches(self) -> int:
        if self._device is not None:
            return self._device.n_patches
        return int(self._host["patch_class"].size)

    def device(self) -> DeviceGeometry:
        """The device geometry of these patches, built from ``solid`` if needed."""

        if self._device is None:
            dev = DeviceGeometry(self._get("solid"), self.H_m)
            if dev.n_patches != int(self._host["patch_class"].size):
                raise ValueError("patch table does not match the surface of its solid array")
            self._device = dev
        return self._device

    def __repr__(self) -> str:
        shape = self._device.shape if self._device is not None else self._host["solid"].shape
        return f"SurfacePatches(shape={shape}, n_patches={self.n_patches}, H_m={self.H_m})"


def _field(name: str):
    return property(lambda self: self._get(name), lambda self, v: self._set(name, v))


for _name in _FIELDS:
    setattr(SurfacePatches, _name, _field(_name))


def build_surface_patches(phases_x: np.ndarray, H_m: float) -> SurfacePatches:
    """Enumerate wall and interface patches of an x-oriented phase array, 1 = solid (view_factors.py:70-132).

    Wall patches come first, ordered by (j, k) with the hot patch before the cold
    patch; a wall patch exists only where the adjacent boundary cell is pore.
    Internal patches follow in (i, j, k, face) order.  Lateral neighbours are
    periodic, and solid faces on the x boundaries are not patches.  Every patch
    has the area (H/N_x)^2.
    """

    dev = DeviceGeometry(phases_x, H_m)
    return SurfacePatches(H_m=H_m, _device=dev)


def _device_of(patches) -> DeviceGeometry:
    if isinstance(patches, SurfacePatches):
        return patches.device()
    # a reference-shaped object: rebuild its table on the device from the solid array
    cached = getattr(patches, "_porerad_b200_device", None)
    if cached is None:
        cached = DeviceGeometry(np.asarray(patches.solid), float(patches.H_m))
        if cached.n_patches != int(np.asarray(patches.patch_class).size):
            raise ValueError("patch table does not match the surface of its solid array")
        try:
            patches._porerad_b200_device = cached
        except AttributeError:
            pass
    return cached


def generate_rays(patches, patch_start: int, patch_end: int, rays_per_patch: int,
                  seed: int) -> tuple[np.ndarray, np.ndarray]:
    """Ray origins and directions for patches ``patch_start`` to ``patch_end - 1`` (view_factors.py:135-182).

    Each ray consumes four uniforms of one PCG64 stream: two place the origin
    uniformly on the patch face and two give a cosine-weighted (Lambertian)
    direction about the patch normal.  The stream is advanced by
    ``patch_start * rays_per_patch * 4`` draws, so any partition of the patches
    reproduces the same rays as a single pass over all of them.
    """

    dev = _device_of(patches)
    p0, p1, R = int(patch_start), int(patch_end), int(rays_per_patch)
    n = max(p1 - p0, 0) * max(R, 0)
    origins = np.empty((n, 3))
    directions = np.empty((n, 3))
    seeds = _lib.seeds_struct([_lib.pcg64_state(seed)])
    _lib.check(_lib.load().pr_generate_rays(dev.handle, p0, p1, R, ctypes.addressof(seeds), origins.ctypes.data,
                                            directions.ctypes.data, _lib.stream()))
    return origins, directions


def trace_first_hit(patches, origins: np.ndarray, directions: np.ndarray) -> np.ndarray:
    """Index of the first patch hit by each ray (view_factors.py:261-270)."""

    dev = _device_of(patches)
    o = np.ascontiguousarray(origins, dtype=np.float64)
    d = np.ascontiguousarray(directions, dtype=np.float64)
    n = int(o.shape[0])
    receiver = np.empty(n, dtype=np.int32)
    failed = ctypes.c_int64()
    status = _lib.load().pr_trace_first_hit(dev.handle, o.ctypes.data, d.ctypes.data, n, receiver.ctypes.data,
                                            ctypes.byref(failed), _lib.stream())
    if status == _lib.PR_ERR_UNRESOLVED:
        raise RuntimeError(f"{int(failed.value)} rays did not resolve a receiving patch")
    _lib.check(status)
    return receiver


PINNED_MIN_BYTES = 16 << 20  # edge lists above this size are handed back in pinned host blocks
HOST_PASS_MAX_BYTES = 16 << 30  # first_hit_counts writes straight to host up to this upper bound


class _HostBlock:
    """A pinned host block of the library; it goes back to the library's cache when the last
    array over it is freed."""

    __slots__ = ("ptr", "nbytes")

    def __init__(self, ptr: int, nbytes: int):
        self.ptr, self.nbytes = ptr, int(nbytes)

    def __del__(self):
        try:
            _lib.load().pr_host_block_release(self.ptr)
        except Exception:  # interpreter shutdown
            pass


def _pinned_block(nbytes: int) -> "_HostBlock":
    """A pinned host block for a result of ``nbytes``: a released block of about that size from
    the library's cache, else a newly pinned one."""

    out = ctypes.c_void_p()
    _lib.check(_lib.load().pr_host_block(int(nbytes), ctypes.byref(out)))
    return _HostBlock(out.value, nbytes)


def _edge_arrays(m: int):
    """Empty (origin int32, receiver int32, count int64) arrays of m pairs.

    Above PINNED_MIN_BYTES the three arrays are views of one pinned host block of the library
    (count first, then origin, then receiver), so the device writes them directly; they are
    ordinary writable NumPy arrays, and the block returns to the library's cache when all three
    are freed.
    """

    if m * 16 <= PINNED_MIN_BYTES:
        return np.empty(m, np.int32), np.empty(m, np.int32), np.empty(m, np.int64)
    blk = _pinned_block(16 * m)
    buf = (ctypes.c_char * (16 * m)).from_address(blk.ptr)
    buf._block = blk  # the buffer (the arrays' base) keeps the block alive
    c = np.frombuffer(buf, np.int64, m, 0)
    o = np.frombuffer(buf, np.int32, m, 8 * m)
    r = np.frombuffer(buf, np.int32, m, 12 * m)
    return o, r, c


def host_blocks_stats() -> dict:
    """Bytes of the library's pinned host blocks held by arrays (live) and cached for reuse."""

    v = [ctypes.c_longlong() for _ in range(4)]
    _lib.check(_lib.load().pr_host_blocks_stats(*[ctypes.byref(x) for x in v]))
    return dict(zip(("live_bytes", "cached_bytes", "allocations", "reuses"), (x.value for x in v)))


def release_host_blocks(keep_bytes: int = 0) -> None:
    """Free the library's cached pinned host blocks down to ``keep_bytes``."""

    _lib.check(_lib.load().pr_host_blocks_trim(int(keep_bytes)))


class CountTable:
    """Pooled first-hit counts resident on the GPU (a ``pr_counts``): CSR rows by origin patch."""

    def __init__(self, handle: int):
        self._h = _lib.Handle(handle, "pr_counts_destroy")
        nnz, n, rays, steps = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64()
        _lib.check(_lib.load().pr_counts_info(self.handle, ctypes.byref(nnz), ctypes.byref(n), ctypes.byref(rays),
                                              ctypes.byref(steps)))
        self.nnz = int(nnz.value)
        self.n_patches = int(n.value)
        self.rays_traced = int(rays.value)
        self.dda_steps = int(steps.value)

    @property
    def handle(self) -> int:
        return self._h.value

    def close(self) -> None:
        self._h.close()

    def to_numpy(self, with_rays: bool = False):
        """(origin int32, receiver int32, count int64) sorted by (origin, receiver) [+ rays_per_origin]."""

        o, r, c = _edge_arrays(self.nnz)
        rays = np.empty(self.n_patches, np.int64) if with_rays else None
        _lib.check(_lib.load().pr_counts_copy(self.handle, o.ctypes.data, r.ctypes.data, c.ctypes.data,
                                              _lib.ptr(rays), _lib.stream()))
        return (o, r, c, rays) if with_rays else (o, r, c)

    def rows(self, patch_begin: int, patch_end: int):
        """(origin int32, receiver int32, count int64) of the origins in [patch_begin, patch_end) only."""

        lib = _lib.load()
        m = ctypes.c_int64()
        b, e = int(patch_begin), int(patch_end)
        _lib.check(lib.pr_counts_rows(self.handle, b, e, ctypes.byref(m), None, None, None, _lib.stream()))
        o, r, c = _edge_arrays(m.value)
        _lib.check(lib.pr_counts_rows(self.handle, b, e, ctypes.byref(m), o.ctypes.data, r.ctypes.data, c.ctypes.data,
                                      _lib.stream()))
        return o, r, c

    def sha256(self) -> str:
        o, r, c, rays = self.to_numpy(with_rays=True)
        return count_sha256(o, r, c, rays)

    def merge(self, other: "CountTable") -> "CountTable":
        """Pooled counts of this table and ``other`` (same patches), computed on the device."""

        out = ctypes.c_void_p()
        _lib.check(_lib.load().pr_counts_merge(self.handle, other.handle, _lib.stream(), ctypes.byref(out)))
        return CountTable(out.value)


def first_hit_counts_pooled(patches, rays_per_patch: int, seeds) -> CountTable:
    """Counts of several seeded ray blocks pooled as ``pool_counts`` pools them, traced in one device pass."""

    dev = _device_of(patches)
    seeds = [int(s) for s in seeds]
    arr = _lib.seeds_struct([_lib.pcg64_state(s) for s in seeds])
    out = ctypes.c_void_p()
    _lib.check(_lib.load().pr_first_hit_counts(dev.handle, int(rays_per_patch), ctypes.addressof(arr), len(seeds),
                                               _lib.stream(), ctypes.byref(out)))
    return CountTable(out.value)


def first_hit_counts_batch(patches_list, rays_per_patch: int, seeds_per_case) -> list[CountTable]:
    """Pooled counts of many geometries in shared traversal launches (batched sweeps).

    ``seeds_per_case[c]`` lists the seeds of case ``c`` (the same number for every case);
    each returned table equals ``first_hit_counts_pooled(patches_list[c], R, seeds)``.
    """

    devs = [_device_of(p) for p in patches_list]
    seeds = [[int(s) for s in ss] for ss in seeds_per_case]
    if len(seeds) != len(devs) or len({len(ss) for ss in seeds}) != 1:
        raise ValueError("one list of seeds per case, all of the same length")
    arr = _lib.seeds_struct([_lib.pcg64_state(s) for ss in seeds for s in ss])
    handles = (ctypes.c_void_p * len(devs))(*[d.handle for d in devs])
    out = (ctypes.c_void_p * len(devs))()
    _lib.check(_lib.load().pr_first_hit_counts_batch(ctypes.addressof(handles), len(devs), int(rays_per_patch),
                                                     ctypes.addressof(arr), len(seeds[0]), _lib.stream(),
                                                     ctypes.addressof(out)))
    return [CountTable(h) for h in out]


def first_hit_counts(patches, rays_per_patch: int, seed: int, *,
                     patch_chunk: int = 16384) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
    """Integer counts (origin, receiver, n) of one seeded ray block, sorted by edge (view_factors.py:273-287).

    ``patch_chunk`` is accepted for signature compatibility; the device pass
    chunks by its own memory budget and the result does not depend on either.
    """

    if int(patch_chunk) <= 0:
        raise ValueError("patch_chunk must be positive")
    dev = _device_of(patches)
    cap = int(dev.n_patches) * int(rays_per_patch)  # pairs never exceed rays
    if 16 * cap <= PINNED_MIN_BYTES or 16 * cap > HOST_PASS_MAX_BYTES:
        table = first_hit_counts_pooled(patches, rays_per_patch, [seed])
        try:
            return table.to_numpy()
        finally:
            table.close()
    # The pass writes the sorted list into a pinned block sized for one pair per ray, chunk by
    # chunk while the next chunks trace; the arrays returned are views of its first pairs.
    blk = _pinned_block(16 * cap)
    buf = (ctypes.c_char * (16 * cap)).from_address(blk.ptr)
    buf._block = blk
    c = np.frombuffer(buf, np.int64, cap, 0)
    o = np.frombuffer(buf, np.int32, cap, 8 * cap)
    r = np.frombuffer(buf, np.int32, cap, 12 * cap)
    arr = _lib.seeds_struct([_lib.pcg64_state(int(seed))])
    n = ctypes.c_int64()
    _lib.check(_lib.load().pr_first_hit_counts_host(dev.handle, int(rays_per_patch), ctypes.addressof(arr), 1,
                                                    _lib.stream(), o.ctypes.data, r.ctypes.data, c.ctypes.data,
                                                    cap, ctypes.byref(n)))
    m = int(n.value)
    return o[:m], r[:m], c[:m]


def pool_counts(tables, n_patches: int) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
    """Sum integer edge counts of several ray blocks into one sorted edge list (view_factors.py:290-300)."""

    table = pool_tables_to_device(tables, n_patches)
    try:
        return table.to_numpy()
    finally:
        table.close()


def _id_array(a, n: int) -> np.ndarray:
    """Patch ids as a contiguous int32 array: int32 input as it is (its range is checked on the
    device), other integer types checked here before they are narrowed."""

    a = np.asarray(a)
    if a.dtype == np.int32:
        return np.ascontiguousarray(a)
    if a.size and (a.min() < 0 or a.max() >= n):
        raise IndexError(f"patch ids outside [0, {n})")
    return np.ascontiguousarray(a, dtype=np.int32)


def pool_tables_to_device(tables, n_patches: int) -> CountTable:
    """Pool a list of (origin, receiver, count) edge lists into a device-resident CountTable.

    The arrays go to the device as they are (no host concatenation): straight from pinned
    memory such as ``first_hit_counts``' results, through the library's staging pipeline from
    pageable memory; the ids are checked and the pairs pooled on the device.
    """

    n = int(n_patches)
    keep = []
    for t in tables:
        o, r = _id_array(t[0], n), _id_array(t[1], n)
        c = np.ascontiguousarray(np.asarray(t[2]), dtype=np.int64)
        if not (o.size == r.size == c.size):
            raise ValueError("origin, receiver and count must have the same length")
        keep.append((o, r, c))
    k = len(keep)
    ptrs = [(ctypes.c_void_p * max(k, 1))(*[x[f].ctypes.data for x in keep]) for f in range(3)]
    sizes = (ctypes.c_int64 * max(k, 1))(*[x[0].size for x in keep])
    out = ctypes.c_void_p()
    lib = _lib.load()
    status = lib.pr_counts_from_tables(*[ctypes.addressof(a) for a in ptrs], ctypes.addressof(sizes), k, n,
                                       _lib.stream(), ctypes.byref(out))
    if status == _lib.PR_ERR_ARG and "patch ids outside" in _lib.last_error():
        raise IndexError(f"patch ids outside [0, {n})")
    _lib.check(status)
    return CountTable(out.value)


def pool_to_device(origin, receiver, count, n_patches: int) -> CountTable:
    """Pool an arbitrary (origin, receiver, count) edge list into a device-resident CountTable."""

    return pool_tables_to_device([(origin, receiver, count)], n_patches)


def count_sha256(origin: np.ndarray, receiver: np.ndarray, count: np.ndarray, rays_per_origin: np.ndarray) -> str:
    """SHA256 of a pooled count table, comparable with the hashes of the case tables (view_factors.py:303-323).

    The edge list must be sorted by (origin, receiver) as returned by
    ``pool_counts``.  For origin (int32), receiver (int32), count (int64) and rays
    per origin (int64), in this order, the digest takes the array name, the NumPy
    dtype string, the shape as int64 and the C-order bytes.
    """

    digest = hashlib.sha256()
    for name, array in (
        ("origin_patch_id", np.asarray(origin, dtype=np.int32)),
        ("receiver_patch_id", np.asarray(receiver, dtype=np.int32)),
        ("count", np.asarray(count, dtype=np.int64)),
        ("rays_per_origin", np.asarray(rays_per_origin, dtype=np.int64)),
    ):
        digest.update(name.encode("ascii"))
        digest.update(array.dtype.str.encode("ascii"))
        digest.update(np.asarray(array.shape, dtype=np.int64).tobytes())
        digest.update(np.ascontiguousarray(array).tobytes())
    return digest.hexdigest()

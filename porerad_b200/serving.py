"""Continuous-batching case server for the surface-radiation path on one GPU.

A request is one geometry-axis case: an x-oriented uint8 phase array, the patch edge
length, a ray count and seeds, and a prescribed field (T_mean, dT, eps).  The server
keeps ``slots`` worker threads, each with its own CUDA stream; a worker takes the next
request in arrival order, builds its surface patches on the device, and then waits for
admission: the request's device-memory footprint (estimated from its patch count and
rays per origin, an upper bound) must fit the HBM budget next to the cases already
running.  Admitted cases trace, balance and solve on their own streams, so requests
that arrive while others are on the GPU overlap with them; every result comes back
with its arrival, admission and completion times.

Kernels are deterministic (fixed reduction trees, integer counts), so a case's result
does not depend on what else runs: alone or in the mix it is the same to the bit.
"""

from __future__ import annotations

import collections
import threading
import time
from concurrent.futures import Future
from dataclasses import dataclass, field
from typing import Any, Callable

import numpy as np

_WAVE_RAYS = 1 << 27  # rays per traversal wave of libporerad (receiver + two stage buffers of int32 per ray)


@dataclass
class GeometrySpec:
    """A seeded benchmark archetype (porerad_b200.geometry.make) generated on the device by the
    worker that serves the request, oriented so that ``axis`` becomes x."""

    archetype: str
    n: int
    phi: float
    seed: int
    axis: str = "x"

    @property
    def shape(self) -> tuple:
        return (int(self.n),) * 3

    def device_phases(self):
        from . import geometry

        import torch

        ph = geometry.make_device(self.archetype, self.n, self.phi, self.seed)
        if self.axis != "x":
            ph = ph.movedim("xyz".index(self.axis), 0).contiguous()
            torch.cuda.current_stream().synchronize()  # torch's copy, before the library's stream reads it
        return ph


@dataclass
class CaseRequest:
    """One prescribed-field case (the inputs of porerad's run_prescribed_field for one condition)."""

    phases: Any                 # uint8 (nx, ny, nz) x-oriented, NumPy array or CUDA tensor, or a GeometrySpec
    H_m: float
    rays_per_patch: int
    seeds: list
    T_mean_K: float
    delta_T_K: float
    epsilon: float
    precision: str = "mixed"
    tag: Any = None


@dataclass
class CaseResult:
    tag: Any
    q_h: float
    q_c: float
    q_i: float
    closure_rel: float
    coarse_source: np.ndarray = field(repr=False)
    n_patches: int = 0
    rays: int = 0
    pairs: int = 0
    balance: tuple = ()
    stats: dict = field(default_factory=dict, repr=False)
    footprint_bytes: int = 0
    t_submit: float = 0.0
    t_admit: float = 0.0
    t_done: float = 0.0
    slot: int = -1

    @property
    def latency_s(self) -> float:
        return self.t_done - self.t_submit

    @property
    def wait_s(self) -> float:
        return self.t_admit - self.t_submit


def geometry_bytes(n_cells: int) -> int:
    """Upper bound of the device bytes of one geometry before its patch count is known."""

    return 28 * n_cells + 6 * n_cells * 40


def footprint_bytes(n_patches: int, rays_per_origin: int) -> int:
    """Upper bound of the device bytes of one case after its surface is built.

    Traversal wave buffers (three int32 per ray of a wave), the pooled count table
    (col + count per pair), its transpose and the symmetric matrix with the radix-sort
    scratch of the transpose (about 48 B per pair in all), and the P-vectors.  Pairs
    are bounded by P * min(rays per origin, P).
    """

    P, L = int(n_patches), int(rays_per_origin)
    pairs = P * min(L, P)
    wave = min(P * L, _WAVE_RAYS)
    return 12 * wave + 48 * pairs + 400 * P + (64 << 20)


class Admission:
    """Device-memory budget shared by the workers: acquire blocks until the bytes fit.

    A request larger than the whole budget is admitted alone (when nothing else holds
    memory) rather than never.  ``grow`` enlarges a reservation in place: a worker whose
    geometry is already resident keeps it counted while it waits for the rest of its
    footprint.
    """

    def __init__(self, budget_bytes: int):
        self.budget = int(budget_bytes)
        self.reserved = 0
        self.peak = 0
        self._cv = threading.Condition()
        self._waiting: dict[int, int] = {}  # ticket -> bytes held by a worker waiting in grow
        self._tickets = 0

    def grow(self, held: int, new: int, stop: Callable[[], bool] = lambda: False) -> bool:
        """Turn a reservation of ``held`` bytes into one of ``new`` bytes, blocking until it fits.

        While it waits the held bytes stay reserved.  If nothing is running (every reserved byte
        belongs to waiting workers) the earliest waiter goes ahead even past the budget, so
        waiters that each hold a resident geometry cannot block one another for ever.
        """

        with self._cv:
            ticket = self._tickets
            self._tickets += 1
            self._waiting[ticket] = int(held)
            try:
                while self.reserved - held + new > self.budget:
                    running = self.reserved - sum(self._waiting.values())
                    if running <= 0 and ticket == min(self._waiting):
                        break
                    if stop():
                        return False
                    self._cv.wait(timeout=0.05)
                self.reserved += int(new) - int(held)
                self.peak = max(self.peak, self.reserved)
                return True
            finally:
                del self._waiting[ticket]
                self._cv.notify_all()

    def acquire(self, nbytes: int, stop: Callable[[], bool] = lambda: False) -> bool:
        with self._cv:
            while self.reserved > 0 and self.reserved + nbytes > self.budget:
                if stop():
                    return False
                self._cv.wait(timeout=0.05)
            self.reserved += nbytes
            self.peak = max(self.peak, self.reserved)
            return True

    def resize(self, old: int, new: int) -> None:
        with self._cv:
            self.reserved += new - old
            self.peak = max(self.peak, self.reserved)
            self._cv.notify_all()

    def release(self, nbytes: int) -> None:
        with self._cv:
            self.reserved -= nbytes
            self._cv.notify_all()


def run_case(req: CaseRequest, admission: Admission, on_admit: Callable[[int], None] | None = None):
    """Run one case on the calling thread's stream (libporerad via porerad_b200); returns a CaseResult."""

    from . import coupled, exchange, view_factors as vf

    shape = tuple(int(s) for s in req.phases.shape)
    n_cells = shape[0] * shape[1] * shape[2]
    geo_bytes = geometry_bytes(n_cells)
    admission.acquire(geo_bytes)
    held = geo_bytes
    geo = table = op = None
    try:
        phases = req.phases.device_phases() if isinstance(req.phases, GeometrySpec) else req.phases
        geo = vf.DeviceGeometry(phases, req.H_m)
        del phases
        L = int(req.rays_per_patch) * len(req.seeds)
        need = footprint_bytes(geo.n_patches, L)
        # the geometry stays resident (and counted) while the worker waits for the rest
        admission.grow(held, geo.device_bytes + need)
        held = geo.device_bytes + need
        t_admit = time.perf_counter()
        if on_admit:
            on_admit(held)
        p = vf.SurfacePatches(H_m=req.H_m, _device=geo)
        table = vf.first_hit_counts_pooled(p, req.rays_per_patch, req.seeds)
        area = np.full(geo.n_patches, (float(req.H_m) / shape[0]) ** 2)
        op = exchange.ExchangeOperator(table, None, None, np.full(geo.n_patches, L, np.int64), area)
        ch = coupled.prescribed_field_channels(op, p, req.T_mean_K, req.delta_T_K, req.epsilon,
                                               precision=req.precision)
        return CaseResult(req.tag, ch.q_h, ch.q_c, ch.q_i, ch.closure_rel, ch.coarse_source, geo.n_patches,
                          table.rays_traced, table.nnz, (op.balance_method, op.balance_iterations, op.row_sum_error),
                          ch.stats, held, t_admit=t_admit)
    finally:
        for obj in (op, table, geo):
            if obj is not None:
                obj.close()
        if held:
            admission.release(held)


class Server:
    """Continuous-batching server: ``slots`` workers on their own CUDA streams, HBM-budget admission."""

    def __init__(self, slots: int = 4, hbm_budget_bytes: int | None = None, device: int = 0,
                 runner: Callable = run_case, streams: bool = True):
        self.slots = int(slots)
        self.device = int(device)
        self.runner = runner
        if hbm_budget_bytes is None:
            import torch

            free, _total = torch.cuda.mem_get_info(self.device)
            hbm_budget_bytes = int(0.85 * free)
        self.admission = Admission(hbm_budget_bytes)
        self._queue: collections.deque = collections.deque()
        self._cv = threading.Condition()
        self._closed = False
        self._streams = streams
        self._threads = [threading.Thread(target=self._worker, args=(k,), daemon=True) for k in range(self.slots)]
        for t in self._threads:
            t.start()

    def submit(self, req: CaseRequest, t_submit: float | None = None) -> Future:
        fut: Future = Future()
        with self._cv:
            if self._closed:
                raise RuntimeError("server is closed")
            self._queue.append((req, fut, time.perf_counter() if t_submit is None else t_submit))
            self._cv.notify()
        return fut

    def close(self, wait: bool = True) -> None:
        with self._cv:
            self._closed = True
            self._cv.notify_all()
        if wait:
            for t in self._threads:
                t.join()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _next(self):
        with self._cv:
            while not self._queue and not self._closed:
                self._cv.wait()
            if not self._queue:
                return None
            return self._queue.popleft()

    def _worker(self, slot: int) -> None:
        ctx = None
        if self._streams:
            import torch

            from . import _lib

            torch.cuda.set_device(self.device)
            ctx = _lib.use_stream(torch.cuda.Stream(self.device))
            ctx.__enter__()
        try:
            while True:
                item = self._next()
                if item is None:
                    return
                req, fut, t_submit = item
                if not fut.set_running_or_notify_cancel():
                    continue
                try:
                    res = self.runner(req, self.admission)
                    res.t_submit = t_submit
                    res.t_done = time.perf_counter()
                    res.slot = slot
                    fut.set_result(res)
                except BaseException as exc:  # the request fails, the worker keeps serving
                    fut.set_exception(exc)
        finally:
            if ctx is not None:
                ctx.__exit__(None, None, None)


def percentile(values, q: float) -> float:
    v = np.sort(np.asarray(values, dtype=np.float64))
    if v.size == 0:
        return float("nan")
    return float(np.percentile(v, q))

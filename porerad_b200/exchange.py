"""Projected view-factor operator and the gray diffuse radiosity reflection series on a B200.

Drop-in for ``porerad.exchange`` (porerad/exchange.py).  With raw view factors
F_ij = n_ij / R_i and patch areas A, the area-weighted exchange matrix is replaced
by its symmetric part plus a small diagonal support term,

    S = 0.5 (diag(A) F + F^T diag(A)) + delta diag(A),    delta = 1e-15,

one positive diagonal factor d restores row closure, d * (S d) = A, and the
projected view factors are F_p = diag(1/A) diag(d) S diag(d).  F_p is never
stored: libporerad keeps S on the union pattern of F and F^T in HBM and applies
F_p x = (d / A) S(d x) and F_p^T x = d S(d x / A) with one sparse product each.

Diffuse reflections are summed by the reflection series of J = E + (1 - eps) F_p^T J
to the stated relative tolerance, with the convergence test on the device.
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from . import _lib
from .constants import SIGMA  # noqa: F401  (part of the module's namespace, exchange.py:28)
from .view_factors import CountTable, pool_to_device

SUPPORT_DIAGONAL_FRACTION = 1.0e-15
CLOSURE_TOLERANCE = 1.0e-10
_TINY = np.finfo(np.float64).tiny
_LOG_MAX = float(np.log(np.finfo(np.float64).max))
_LOG_MIN = float(np.log(np.nextafter(0.0, 1.0)))


class ExchangeOperator:
    """Projected view-factor matrix F_p built from integer first-hit counts (exchange.py:37-80).

    ``origin``, ``receiver`` and ``count`` hold the counts n_ij and
    ``rays_per_origin`` the rays R_i; every row must account for all of its rays
    (ValueError otherwise).  The diagonal factor d is found by Anderson
    acceleration on y = log d, with a damped multiplicative iteration as fallback,
    and the projected rows must close to within 1e-10 (RuntimeError otherwise).

    ``origin`` may also be a device-resident :class:`CountTable` (then
    ``receiver`` and ``count`` are None), which skips the host round trip.
    """

    def __init__(self, origin, receiver, count, rays_per_origin, patch_area_m2, *,
                 support_diagonal_fraction: float = SUPPORT_DIAGONAL_FRACTION,
                 balance_tolerance: float = 1.0e-11, event_chunk_size: int = 4_000_000) -> None:
        rays = np.ascontiguousarray(np.asarray(rays_per_origin, dtype=np.int64))
        n = int(rays.size)
        area = np.ascontiguousarray(np.asarray(patch_area_m2, dtype=np.float64).copy())
        if area.size != n:
            raise ValueError("patch_area_m2 and rays_per_origin must have the same length")
        own_table = not isinstance(origin, CountTable)
        table = pool_to_device(origin, receiver, count, n) if own_table else origin
        if table.n_patches != n:
            raise ValueError("count table and rays_per_origin disagree on the number of patches")
        out = ctypes.c_void_p()
        try:
            _lib.check(_lib.load().pr_operator_create(table.handle, rays.ctypes.data, area.ctypes.data,
                                                      float(support_diagonal_fraction), float(balance_tolerance),
                                                      _lib.stream(), ctypes.byref(out)))
        finally:
            if own_table:
                table.close()
        self._adopt(out.value, area, support_diagonal_fraction, event_chunk_size)

    @classmethod
    def _from_handle(cls, handle: int, area: np.ndarray, support_diagonal_fraction: float,
                     event_chunk_size: int = 4_000_000) -> "ExchangeOperator":
        op = cls.__new__(cls)
        op._adopt(handle, area, support_diagonal_fraction, event_chunk_size)
        return op

    def _adopt(self, handle: int, area: np.ndarray, support_diagonal_fraction: float, event_chunk_size: int) -> None:
        n = int(area.size)
        self._h = _lib.Handle(handle, "pr_operator_destroy")
        self.patch_area_m2 = area
        self.support_diagonal_fraction = float(support_diagonal_fraction)
        self.event_chunk_size = int(event_chunk_size)
        self.n_patches = n
        self._edges: tuple | None = None
        scale = np.empty(n)
        method, iters, rse = ctypes.c_int(), ctypes.c_int(), ctypes.c_double()
        nnz_f, nnz_s = ctypes.c_int64(), ctypes.c_int64()
        _lib.check(_lib.load().pr_operator_info(self.handle, _lib.ptr(scale), ctypes.byref(method),
                                                ctypes.byref(iters), ctypes.byref(rse), ctypes.byref(nnz_f),
                                                ctypes.byref(nnz_s), None))
        self.scale = scale
        self.balance_method = _lib.BALANCE_METHODS[int(method.value)]
        self.balance_iterations = int(iters.value)
        self.row_sum_error = float(rse.value)
        self.nnz = int(nnz_f.value)
        self.nnz_symmetric = int(nnz_s.value)

    @property
    def handle(self) -> int:
        return self._h.value

    def close(self) -> None:
        self._h.close()

    @classmethod
    def from_tables(cls, tables, rays_per_origin, patch_area_m2, *,
                    support_diagonal_fraction: float = SUPPORT_DIAGONAL_FRACTION,
                    balance_tolerance: float = 1.0e-11) -> list["ExchangeOperator"]:
        """Operators of many device count tables built together (batched sweeps).

        ``rays_per_origin`` and ``patch_area_m2`` hold one array per table.  The balancing
        iterations of all operators run in lockstep with one product launch per iteration for all
        of them; each operator equals ``ExchangeOperator(table, None, None, rays, area)`` bit for bit.
        """

        tables = list(tables)
        m = len(tables)
        rays = [np.ascontiguousarray(np.asarray(r, dtype=np.int64)) for r in rays_per_origin]
        areas = [np.ascontiguousarray(np.asarray(a, dtype=np.float64).copy()) for a in patch_area_m2]
        if not (len(rays) == len(areas) == m):
            raise ValueError("one rays array and one area array per table")
        for t, r, a in zip(tables, rays, areas):
            if not isinstance(t, CountTable):
                raise TypeError("from_tables takes device CountTables")
            if not (t.n_patches == r.size == a.size):
                raise ValueError("count table, rays_per_origin and patch_area_m2 disagree on the number of patches")
        if m == 0:
            return []
        handles = (ctypes.c_void_p * m)(*[t.handle for t in tables])
        rptr = (ctypes.c_void_p * m)(*[r.ctypes.data for r in rays])
        aptr = (ctypes.c_void_p * m)(*[a.ctypes.data for a in areas])
        out = (ctypes.c_void_p * m)()
        _lib.check(_lib.load().pr_operator_create_batch(ctypes.addressof(handles), ctypes.addressof(rptr),
                                                        ctypes.addressof(aptr), m, float(support_diagonal_fraction),
                                                        float(balance_tolerance), _lib.stream(),
                                                        ctypes.addressof(out)))
        return [cls._from_handle(h, a, support_diagonal_fraction) for h, a in zip(out, areas)]

    @property
    def spmv_calls(self) -> int:
        """Sparse products made with this operator so far (balancing, closure check, solves)."""

        calls = ctypes.c_int64()
        _lib.check(_lib.load().pr_operator_info(self.handle, None, None, None, None, None, None,
                                                ctypes.byref(calls)))
        return int(calls.value)

    def _edge_arrays(self):
        if self._edges is None:
            m = self.nnz
            o = np.empty(m, np.int32)
            r = np.empty(m, np.int32)
            w = np.empty(m, np.float64)
            _lib.check(_lib.load().pr_operator_edges(self.handle, o.ctypes.data, r.ctypes.data, w.ctypes.data, _lib.stream()))
            self._edges = (o, r, w)
        return self._edges

    @property
    def origin(self) -> np.ndarray:
        return self._edge_arrays()[0]

    @property
    def receiver(self) -> np.ndarray:
        return self._edge_arrays()[1]

    @property
    def weight(self) -> np.ndarray:
        return self._edge_arrays()[2]

    def _apply(self, which: int, x) -> np.ndarray:
        xx = np.ascontiguousarray(np.broadcast_to(np.asarray(x, dtype=np.float64), (self.n_patches,)))
        y = np.empty(self.n_patches)
        _lib.check(_lib.load().pr_operator_apply(self.handle, which, xx.ctypes.data, y.ctypes.data, _lib.stream()))
        return y

    def raw_matvec(self, x: np.ndarray) -> np.ndarray:
        """Raw row-normalised view factors applied to x, F x (exchange.py:82-93)."""

        return self._apply(_lib.APPLY_RAW, x)

    def raw_rmatvec(self, x: np.ndarray) -> np.ndarray:
        """Transpose of the raw view factors applied to x, F^T x (exchange.py:95-106)."""

        return self._apply(_lib.APPLY_RAW_T, x)

    def symmetric_matvec(self, x: np.ndarray) -> np.ndarray:
        """Symmetrised area-weighted exchange matrix applied to x, S x (exchange.py:108-112)."""

        return self._apply(_lib.APPLY_SYM, x)

    def matvec(self, x: np.ndarray) -> np.ndarray:
        """Projected view factors applied to x, F_p x (exchange.py:114-117)."""

        return self._apply(_lib.APPLY_MATVEC, x)

    def rmatvec(self, x: np.ndarray) -> np.ndarray:
        """Transpose of the projected view factors applied to x, F_p^T x (exchange.py:119-122)."""

        return self._apply(_lib.APPLY_RMATVEC, x)

    def reciprocity_error(self) -> float:
        """Largest relative defect of A_i F_p,ij = A_j F_p,ji over all sampled pairs (exchange.py:124-140)."""

        out = ctypes.c_double()
        _lib.check(_lib.load().pr_operator_reciprocity_error(self.handle, ctypes.byref(out), _lib.stream()))
        return float(out.value)

    def _closure_error(self, y: np.ndarray) -> float:
        """max |d (S d) / A - 1| for d = exp(y) (exchange.py:142-151)."""

        y = np.asarray(y, dtype=np.float64)
        if not (np.all(np.isfinite(y)) and np.max(y) < _LOG_MAX and np.min(y) > _LOG_MIN):
            return float("inf")
        scale = np.exp(y)
        row = scale * self.symmetric_matvec(scale)
        if not np.all(np.isfinite(row)) or np.any(row <= 0.0):
            return float("inf")
        return float(np.max(np.abs(row / self.patch_area_m2 - 1.0)))


@dataclass
class RadiosityResult:
    """Emitted, absorbed and net (absorbed minus emitted) patch power (exchange.py:200-214)."""

    emitted_power_W: np.ndarray
    absorbed_power_W: np.ndarray
    net_power_W: np.ndarray
    residual_power_W: float
    iterations: int

    @property
    def global_energy_residual_W(self) -> float:
        """Net power of all patches plus the power still in flight."""

        return float(np.sum(self.net_power_W) + self.residual_power_W)


def _vec(x, n: int) -> np.ndarray:
    return np.ascontiguousarray(np.broadcast_to(np.asarray(x, dtype=np.float64), (n,)))


def reflection_series(operator: ExchangeOperator, emitted_W: np.ndarray, emissivity: np.ndarray, *,
                      relative_tolerance: float, max_reflections: int = 10000) -> RadiosityResult:
    """Absorbed power after all diffuse reflections of a (possibly signed) emission (exchange.py:217-245).

    Power in flight is passed to the receiving patches by F_p^T; each patch absorbs
    the fraction eps and reflects 1 - eps.  The series stops when the L1 norm of
    the power in flight falls below ``relative_tolerance`` times the L1 norm of
    the emission (RuntimeError after ``max_reflections``).
    """

    n = operator.n_patches
    e = _vec(emitted_W, n)
    eps = _vec(emissivity, n)
    absorbed = np.empty(n)
    res, it = ctypes.c_double(), ctypes.c_int64()
    _lib.check(_lib.load().pr_reflection_series(operator.handle, e.ctypes.data, eps.ctypes.data,
                                                float(relative_tolerance), int(max_reflections),
                                                absorbed.ctypes.data, ctypes.byref(res), ctypes.byref(it), _lib.stream()))
    return RadiosityResult(e, absorbed, absorbed - e, float(res.value), int(it.value))


def net_patch_power(operator: ExchangeOperator, temperature_K: np.ndarray, emissivity: np.ndarray,
                    area_m2: np.ndarray, *, relative_tolerance: float,
                    reference_temperature_K: float | None = None) -> RadiosityResult:
    """Net radiative power of every patch for given patch temperatures (exchange.py:248-271).

    With ``reference_temperature_K`` the isothermal state at that temperature,
    which carries zero net power, is subtracted before the series is summed: only
    the signed emission eps sigma A (T^4 - T_ref^4) is propagated.
    """

    n = operator.n_patches
    T = _vec(temperature_K, n)
    eps = _vec(emissivity, n)
    area = _vec(area_m2, n)
    emitted, absorbed, net = np.empty(n), np.empty(n), np.empty(n)
    res, it = ctypes.c_double(), ctypes.c_int64()
    has_ref = reference_temperature_K is not None
    _lib.check(_lib.load().pr_net_patch_power(operator.handle, T.ctypes.data, eps.ctypes.data, area.ctypes.data,
                                              float(relative_tolerance), int(has_ref),
                                              float(reference_temperature_K) if has_ref else 0.0, 10000,
                                              emitted.ctypes.data, absorbed.ctypes.data, net.ctypes.data,
                                              ctypes.byref(res), ctypes.byref(it), _lib.stream()))
    return RadiosityResult(emitted, absorbed, net, float(res.value), int(it.value))


def net_patch_power_jvp(operator: ExchangeOperator, temperature_K: np.ndarray, delta_temperature_K: np.ndarray,
                        emissivity: np.ndarray, area_m2: np.ndarray, *, relative_tolerance: float) -> np.ndarray:
    """Derivative of the net patch power along a patch temperature perturbation (exchange.py:274-287)."""

    n = operator.n_patches
    T = _vec(temperature_K, n)
    dT = _vec(delta_temperature_K, n)
    eps = _vec(emissivity, n)
    area = _vec(area_m2, n)
    out = np.empty(n)
    _lib.check(_lib.load().pr_net_patch_power_jvp(operator.handle, T.ctypes.data, dT.ctypes.data, eps.ctypes.data,
                                                  area.ctypes.data, float(relative_tolerance), out.ctypes.data,
                                                  _lib.stream()))
    return out

"""Cell-centred finite-volume heat conduction on a digital microstructure, on a B200.

Mirrors ``porerad.conduction`` (porerad/conduction.py).  Every cell carries the
conductivity of its phase; neighbouring cells exchange heat through the harmonic-mean
face conductance times dx^2 / dx, the lateral faces y and z are periodic, and a cell next
to a wall is connected to the fixed wall temperature through 2 k dx.  The system lives in
libporerad as the face conductances of every cell (a 7-point stencil), not as a general
sparse matrix; :attr:`ConductionSystem.matrix` materialises the reference's CSR matrix on
the host for callers that want it.
"""

from __future__ import annotations

import ctypes

import numpy as np

from . import _lib


class ConductionSystem:
    """Conduction matrix A and the wall responses of an x-oriented cell grid (conduction.py:24-50).

    Constructed as the reference's dataclass is, ``ConductionSystem(matrix, hot_rhs, cold_rhs,
    conductivity, H_m)``; :func:`assemble_conduction` passes ``None`` for the first three.  The
    device system is always assembled from ``conductivity`` and ``H_m``; arrays that are given
    must equal that assembly (``ValueError`` otherwise) and are then what the accessors return.
    """

    def __init__(self, matrix, hot_rhs, cold_rhs, conductivity: np.ndarray, H_m: float):
        k = np.ascontiguousarray(conductivity, dtype=np.float64)
        if k.ndim != 3:
            raise ValueError("conductivity must be a 3-D array")
        nx, ny, nz = map(int, k.shape)
        out = ctypes.c_void_p()
        _lib.check(_lib.load().pr_conduction_create(k.ctypes.data, nx, ny, nz, float(H_m), _lib.stream(),
                                                    ctypes.byref(out)))
        self._h = _lib.Handle(out.value, "pr_conduction_destroy")
        self.conductivity = k
        self.H_m = float(H_m)
        self._arrays = None
        self._matrix = None
        if hot_rhs is not None or cold_rhs is not None or matrix is not None:
            self._adopt(matrix, hot_rhs, cold_rhs)

    def _adopt(self, matrix, hot_rhs, cold_rhs) -> None:
        """Keep caller-given arrays after checking them against the device assembly."""

        for name, given in (("hot_rhs", hot_rhs), ("cold_rhs", cold_rhs)):
            if given is not None and not np.array_equal(np.asarray(given, np.float64).ravel(),
                                                        self._host_arrays()[name]):
                raise ValueError(f"{name} does not match the conductivity field's assembly")
        if matrix is not None:
            from scipy.sparse import csr_matrix

            given = csr_matrix(matrix)
            if given.shape != self.matrix.shape or (given != self.matrix).nnz:
                raise ValueError("matrix does not match the conductivity field's assembly")
            self._matrix = given

    @property
    def handle(self) -> int:
        return self._h.value

    def close(self) -> None:
        self._h.close()

    @property
    def shape(self) -> tuple[int, int, int]:
        return tuple(map(int, self.conductivity.shape))

    def _host_arrays(self) -> dict:
        if self._arrays is None:
            n = self.conductivity.size
            names = ("gx", "gy", "gz", "diag", "hot_rhs", "cold_rhs")
            arrs = {name: np.empty(n, np.float64) for name in names}
            _lib.check(_lib.load().pr_conduction_arrays(self.handle, *[arrs[k].ctypes.data for k in names],
                                                        _lib.stream()))
            self._arrays = arrs
        return self._arrays

    @property
    def hot_rhs(self) -> np.ndarray:
        return self._host_arrays()["hot_rhs"]

    @property
    def cold_rhs(self) -> np.ndarray:
        return self._host_arrays()["cold_rhs"]

    @property
    def matrix(self):
        """A as a SciPy CSR matrix (the reference's ``ConductionSystem.matrix``), built from the device arrays."""

        if self._matrix is None:
            from scipy.sparse import coo_matrix

            a = self._host_arrays()
            nx, ny, nz = self.shape
            cell = np.arange(nx * ny * nz, dtype=np.int64).reshape(nx, ny, nz)
            rows, cols, vals = [cell.ravel()], [cell.ravel()], [a["diag"]]
            for axis, g in ((0, "gx"), (1, "gy"), (2, "gz")):
                high = np.roll(cell, -1, axis=axis)
                cond = a[g].reshape(nx, ny, nz)
                low_cells = cell if axis else cell[:-1]
                high_cells = high if axis else high[:-1]
                gv = cond if axis else cond[:-1]
                rows += [low_cells.ravel(), high_cells.ravel()]
                cols += [high_cells.ravel(), low_cells.ravel()]
                vals += [-gv.ravel(), -gv.ravel()]
            m = coo_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))),
                           shape=(cell.size, cell.size)).tocsr()
            m.sum_duplicates()
            m.sort_indices()
            self._matrix = m
        return self._matrix

    def apply(self, x: np.ndarray) -> np.ndarray:
        """A x on the device (host or device vector in, host vector out)."""

        xv = np.ascontiguousarray(np.asarray(x, dtype=np.float64).ravel())
        y = np.empty_like(xv)
        _lib.check(_lib.load().pr_conduction_apply(self.handle, xv.ctypes.data, y.ctypes.data, _lib.stream()))
        return y

    def boundary_rhs(self, T_hot_K: float, T_cold_K: float) -> np.ndarray:
        """Right-hand side b contributed by the two fixed wall temperatures (conduction.py:37-40)."""

        return self.hot_rhs * float(T_hot_K) + self.cold_rhs * float(T_cold_K)

    def wall_fluxes(self, temperature_K: np.ndarray, T_hot_K: float, T_cold_K: float) -> tuple[float, float]:
        """Conductive heat flux (W m^-2) into the slab at the hot wall and out at the cold wall (conduction.py:43-50)."""

        T = np.ascontiguousarray(np.asarray(temperature_K, dtype=np.float64).ravel())
        qh, qc = ctypes.c_double(), ctypes.c_double()
        _lib.check(_lib.load().pr_conduction_wall_fluxes(self.handle, T.ctypes.data, float(T_hot_K), float(T_cold_K),
                                                         ctypes.byref(qh), ctypes.byref(qc), _lib.stream()))
        return float(qh.value), float(qc.value)


def assemble_conduction(conductivity_x: np.ndarray, H_m: float) -> ConductionSystem:
    """Assemble A and the wall responses for a conductivity field oriented along x (conduction.py:53-92)."""

    return ConductionSystem(None, None, None, conductivity_x, H_m)


def solve_conduction(system: ConductionSystem, T_hot_K: float, T_cold_K: float, *,
                     rtol: float = 1.0e-11) -> np.ndarray:
    """Pure-conduction field by Jacobi-preconditioned conjugate gradients (conduction.py:95-120).

    The iteration starts from the linear profile between the wall temperatures and stops
    at a relative residual of ``rtol``; ``RuntimeError`` unless the true relative residual
    is at most 1e-9.
    """

    T = np.empty(system.conductivity.size, np.float64)
    it, rel = ctypes.c_int64(), ctypes.c_double()
    _lib.check(_lib.load().pr_conduction_solve(system.handle, float(T_hot_K), float(T_cold_K), float(rtol),
                                               T.ctypes.data, ctypes.byref(it), ctypes.byref(rel), _lib.stream()))
    return T.reshape(system.shape)

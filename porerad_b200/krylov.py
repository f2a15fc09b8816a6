"""Host-side Krylov helpers of the ``porerad.coupled`` API, for callers with their own operators.

The coupled solve of this package runs its flexible GMRES and its preconditioner on the device
(``csrc/coupled.cu``).  The reference also exposes them as generic helpers over host callables
(``flexible_gmres(matvec, rhs, preconditioner, ...)``, ``FixedJacobiPCG``, coupled.py:225-320);
a caller that passes its own ``matvec`` gets these host implementations, with the same
arguments, stopping rules and result type.

``flexible_gmres`` keeps the preconditioned directions (the preconditioner may change between
applications), orthogonalises each new Krylov vector with two Gram-Schmidt passes, reduces the
Hessenberg matrix with Givens rotations as the columns arrive (the least-squares residual is
then the last rotated right-hand-side entry), and accepts a solution only once its true
residual ``|rhs - matvec(x)|`` meets the threshold max(absolute, relative * |rhs|).
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

_TINY = np.finfo(np.float64).tiny
_EPS = np.finfo(np.float64).eps


@dataclass
class GMRESResult:
    """A flexible GMRES solution, whether its true residual met the threshold, the Krylov steps
    taken and the final true residual relative to |rhs| (coupled.py:225-230)."""

    solution: np.ndarray
    converged: bool
    iterations: int
    true_residual_relative: float


class _Arnoldi:
    """One restart cycle: basis V, preconditioned directions Z, rotated Hessenberg R, rotated rhs g."""

    def __init__(self, residual: np.ndarray, beta: float, width: int):
        n = residual.size
        self.V = np.zeros((width + 1, n))
        self.Z = np.zeros((width, n))
        self.R = np.zeros((width, width))
        self.rot = np.zeros((width, 2))
        self.g = np.zeros(width + 1)
        self.V[0] = residual / beta
        self.g[0] = beta
        self.k = 0

    def extend(self, matvec, preconditioner, beta: float) -> bool:
        """Add one column; False when the Krylov space stopped growing (the new vector vanished)."""

        k = self.k
        self.Z[k] = preconditioner(self.V[k])
        w = np.array(matvec(self.Z[k]), dtype=np.float64)
        h = np.zeros(k + 2)
        for _ in range(2):
            for j in range(k + 1):
                c = float(np.dot(self.V[j], w))
                h[j] += c
                w -= c * self.V[j]
        h[k + 1] = float(np.linalg.norm(w))
        grows = h[k + 1] > _EPS * beta
        if grows:
            self.V[k + 1] = w / h[k + 1]
        for j in range(k):  # earlier rotations act on the new column
            c, s = self.rot[j]
            h[j], h[j + 1] = c * h[j] + s * h[j + 1], c * h[j + 1] - s * h[j]
        r = float(np.hypot(h[k], h[k + 1]))
        c, s = (h[k] / r, h[k + 1] / r) if r > 0.0 else (1.0, 0.0)
        self.rot[k] = (c, s)
        self.R[: k + 1, k] = h[: k + 1]
        self.R[k, k] = r
        self.g[k + 1] = -s * self.g[k]
        self.g[k] = c * self.g[k]
        self.k = k + 1
        return grows

    @property
    def estimate(self) -> float:
        return abs(float(self.g[self.k]))

    def correction(self) -> np.ndarray:
        k = self.k
        y = np.linalg.lstsq(self.R[:k, :k], self.g[:k], rcond=None)[0]
        return y @ self.Z[:k]


def flexible_gmres(matvec, rhs: np.ndarray, preconditioner, *, restart: int, max_iterations: int,
                   relative_tolerance: float, absolute_tolerance: float) -> GMRESResult:
    """Solve ``matvec(x) = rhs`` from x = 0 by right-preconditioned flexible GMRES (coupled.py:233-290).

    At most ``max_iterations`` Krylov steps in cycles of ``restart``.  A cycle ends early when the
    least-squares residual estimate meets the threshold or the space stops growing; the candidate
    is returned if its true residual meets the threshold, else the next cycle restarts from it.
    """

    b = np.asarray(rhs, dtype=np.float64)
    b_norm = max(float(np.linalg.norm(b)), _TINY)
    threshold = max(float(absolute_tolerance), float(relative_tolerance) * b_norm)
    x = np.zeros_like(b)
    steps = 0
    while steps < max_iterations:
        residual = b - matvec(x)
        beta = float(np.linalg.norm(residual))
        if beta <= threshold:
            return GMRESResult(x, True, steps, beta / b_norm)
        cycle = _Arnoldi(residual, beta, min(int(restart), int(max_iterations) - steps))
        stopped = False
        while cycle.k < cycle.Z.shape[0]:
            grows = cycle.extend(matvec, preconditioner, beta)
            steps += 1
            if cycle.estimate <= threshold or not grows:
                stopped = True
                break
        candidate = x + cycle.correction()
        if stopped:
            true_norm = float(np.linalg.norm(b - matvec(candidate)))
            if true_norm <= threshold:
                return GMRESResult(candidate, True, steps, true_norm / b_norm)
        x = candidate
    true_norm = float(np.linalg.norm(b - matvec(x)))
    return GMRESResult(x, true_norm <= threshold, steps, true_norm / b_norm)


class FixedJacobiPCG:
    """``steps`` conjugate-gradient steps with a Jacobi preconditioner on P = A + diag(shift), from x = 0.

    A is ``system.matrix`` (the conduction matrix, a SciPy sparse matrix); the operator is a
    fixed linear map, so flexible GMRES can use it as a right preconditioner (coupled.py:293-320).
    """

    def __init__(self, system, shift: np.ndarray, steps: int) -> None:
        self.matrix = system.matrix
        self.shift = np.asarray(shift, dtype=np.float64)
        self.steps = int(steps)
        self.inverse_diagonal = 1.0 / (self.matrix.diagonal() + self.shift)

    def __call__(self, rhs: np.ndarray) -> np.ndarray:
        r = np.array(rhs, dtype=np.float64)
        x = np.zeros_like(r)
        z = self.inverse_diagonal * r
        direction = z.copy()
        rz = float(r @ z)
        for step in range(self.steps):
            q = self.matrix @ direction + self.shift * direction
            alpha = rz / float(direction @ q)
            x += alpha * direction
            if step + 1 == self.steps:
                break
            r -= alpha * q
            z = self.inverse_diagonal * r
            rz_next = float(r @ z)
            direction = z + (rz_next / rz) * direction
            rz = rz_next
        return x

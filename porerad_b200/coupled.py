"""Radiation channels and the strictly coupled radiation-conduction solve on a B200.

Mirrors ``porerad.coupled`` (porerad/coupled.py).  :func:`prescribed_field_channels` runs
on the GPU end to end (patch temperatures, emission, radiosity, per-class sums and the
coarse source in libporerad); :func:`solve_coupled` / :func:`newton_krylov` run the whole
Newton-Krylov iteration on the device (conduction stencil, flexible GMRES, the radiosity
JVP, the Jacobi-PCG preconditioner and the line search) with the conduction system of
:mod:`porerad_b200.conduction`.  The small helpers keep the reference's host semantics for
callers that use them directly.
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass, field

import numpy as np

from . import _lib
from .conduction import ConductionSystem  # noqa: F401  (part of the module's namespace, coupled.py:23)
from .constants import SIGMA
from .exchange import ExchangeOperator, RadiosityResult, net_patch_power, net_patch_power_jvp
from .krylov import FixedJacobiPCG, GMRESResult, flexible_gmres  # noqa: F401  (host helpers, coupled.py:225-320)
from .view_factors import COLD, HOT, INTERNAL, SurfacePatches, _device_of

_TINY = np.finfo(np.float64).tiny

RADIOSITY_RTOL_NEWTON = 1.0e-8
RADIOSITY_RTOL_FINAL = 1.0e-13
MIXED_RTOL = 1.0e-10
"""Relative binary64 residual the mixed-precision solve refines to."""


def patch_temperature(patches, T_cells: np.ndarray, T_hot_K: float, T_cold_K: float) -> np.ndarray:
    """Wall temperatures on wall patches and the owning-cell temperature on internal patches (coupled.py:45-53)."""

    cls = np.asarray(patches.patch_class)
    T = np.empty(cls.size, dtype=np.float64)
    inner = cls == INTERNAL
    T[cls == HOT] = float(T_hot_K)
    T[cls == COLD] = float(T_cold_K)
    T[inner] = np.asarray(T_cells, dtype=np.float64).ravel()[np.asarray(patches.patch_cell)[inner]]
    return T


def cell_power(patches, patch_power_W: np.ndarray) -> np.ndarray:
    """Sum the power of the internal patches into their owning solid cells (coupled.py:56-62)."""

    cls = np.asarray(patches.patch_class)
    inner = cls == INTERNAL
    solid = np.asarray(patches.solid)
    power = np.zeros(solid.size, dtype=np.float64)
    np.add.at(power, np.asarray(patches.patch_cell)[inner], np.asarray(patch_power_W)[inner])
    return power.reshape(solid.shape)


def emission_diagonal(patches, T_cells: np.ndarray, epsilon: float) -> np.ndarray:
    """Local emission derivative sum_p 4 eps sigma A_p T^3 of every cell in W/K (coupled.py:65-73)."""

    cls = np.asarray(patches.patch_class)
    inner = cls == INTERNAL
    owner = np.asarray(patches.patch_cell)[inner].astype(np.int64)
    T = np.asarray(T_cells, dtype=np.float64).ravel()[owner]
    diagonal = np.zeros(np.asarray(patches.solid).size, dtype=np.float64)
    np.add.at(diagonal, owner, 4.0 * float(epsilon) * SIGMA * np.asarray(patches.patch_area_m2)[inner] * T**3)
    return diagonal


@dataclass
class RadiationState:
    """Patch temperatures, net patch power and net cell power of one temperature field (coupled.py:76-83)."""

    patch_temperature_K: np.ndarray
    patch_net_power_W: np.ndarray
    cell_net_power_W: np.ndarray
    radiosity: RadiosityResult


def evaluate_radiation(operator: ExchangeOperator, patches, T_cells: np.ndarray, T_hot_K: float, T_cold_K: float,
                       epsilon: float, *, relative_tolerance: float,
                       reference_temperature_K: float | None = None) -> RadiationState:
    """Net radiative power of patches and cells; all surfaces share the emissivity eps (coupled.py:86-105)."""

    T_patch = patch_temperature(patches, T_cells, T_hot_K, T_cold_K)
    emissivity = np.full(T_patch.size, float(epsilon))
    radiosity = net_patch_power(operator, T_patch, emissivity, np.asarray(patches.patch_area_m2),
                                relative_tolerance=relative_tolerance,
                                reference_temperature_K=reference_temperature_K)
    return RadiationState(T_patch, radiosity.net_power_W, cell_power(patches, radiosity.net_power_W), radiosity)


def radiation_jvp(operator: ExchangeOperator, patches, T_patch: np.ndarray, dT_cells: np.ndarray, epsilon: float, *,
                  relative_tolerance: float) -> np.ndarray:
    """Change of the net cell power for a cell temperature perturbation, walls fixed (coupled.py:108-126)."""

    cls = np.asarray(patches.patch_class)
    internal = cls == INTERNAL
    dT_patch = np.zeros(cls.size, dtype=np.float64)
    dT_patch[internal] = np.asarray(dT_cells, dtype=np.float64).ravel()[np.asarray(patches.patch_cell)[internal]]
    emissivity = np.full(cls.size, float(epsilon))
    patch_jvp = net_patch_power_jvp(operator, T_patch, dT_patch, emissivity, np.asarray(patches.patch_area_m2),
                                    relative_tolerance=relative_tolerance)
    return cell_power(patches, patch_jvp)


def cross_section_area(patches) -> float:
    """Projected wall area N_y N_z (H/N_x)^2 (coupled.py:129-133)."""

    nx, ny, nz = _shape_of(patches)
    return float(ny * nz) * (patches.H_m / float(nx)) ** 2


def linear_cell_temperature(shape: tuple[int, int, int], T_mean_K: float, delta_T_K: float) -> np.ndarray:
    """The prescribed linear field at the cell centres: T_m + dT/2 at the hot wall (x = 0) falling
    by dT over the N_x cells to T_m - dT/2 at the cold wall (coupled.py:138-143)."""

    nx, ny, nz = (int(n) for n in shape)
    T_hot = T_mean_K + delta_T_K / 2.0
    centres = np.arange(nx, dtype=np.float64) + 0.5
    out = np.empty((nx, ny, nz))
    out[...] = (T_hot - centres * delta_T_K / nx)[:, None, None]
    return out


def coarse_source(cell_power_W: np.ndarray, bins: int = 8) -> np.ndarray:
    """Cell power summed over blocks of a bins^3 grid (coupled.py:146-153).  Along an axis of n
    cells there are min(bins, n) blocks; their sizes differ by at most one, the larger first."""

    out = np.asarray(cell_power_W, dtype=np.float64)
    for axis, n in enumerate(out.shape):
        k = min(int(bins), n)
        sizes = [n // k + (1 if b < n % k else 0) for b in range(k)]
        out = np.add.reduceat(out, np.cumsum([0] + sizes[:-1]), axis=axis)
    return out


@dataclass
class PrescribedChannels:
    """Radiation channels (W m^-2) under the prescribed linear field, q_h + q_c + q_i = 0 (coupled.py:156-167).

    ``stats`` (not in the reference) records how the solve ran: reflections or
    refinements, sparse products, and the final relative residual.
    """

    T_mean_K: float
    delta_T_K: float
    epsilon: float
    q_h: float
    q_c: float
    q_i: float
    closure_rel: float
    coarse_source: np.ndarray = field(repr=False)
    stats: dict = field(default_factory=dict, repr=False)


def _shape_of(patches) -> tuple[int, int, int]:
    if isinstance(patches, SurfacePatches) and patches._device is not None:
        return patches._device.shape
    return tuple(int(s) for s in np.asarray(patches.solid).shape)


def prescribed_field_channels(operator: ExchangeOperator, patches, T_mean_K: float, delta_T_K: float,
                              epsilon: float, *, precision: str = "fp64",
                              relative_tolerance: float | None = None) -> PrescribedChannels:
    """Net power leaving the hot wall, the cold wall and the internal surfaces (coupled.py:170-194).

    Walls are held at T_m +/- dT/2 and every internal surface takes the linear
    field at its owning cell.  One radiosity evaluation to a relative tolerance of
    1e-13 is made with the isothermal state at T_m subtracted.  ``precision``
    "mixed" solves with binary32 sweeps refined to a binary64 residual (not in the
    reference; its relative residual is ``relative_tolerance``, default 1e-10).
    """

    dev = _device_of(patches)
    prec = {"fp64": _lib.PRECISION_FP64, "mixed": _lib.PRECISION_MIXED}[precision]
    rtol = RADIOSITY_RTOL_FINAL if prec == _lib.PRECISION_FP64 else MIXED_RTOL
    if relative_tolerance is not None:
        rtol = float(relative_tolerance)
    nx, ny, nz = dev.shape
    bins = tuple(min(8, n) for n in (nx, ny, nz))
    coarse = np.empty(bins)
    q = np.empty(4)
    stats = np.zeros(4)
    _lib.check(_lib.load().pr_prescribed_field_channels(dev.handle, operator.handle, float(T_mean_K),
                                                        float(delta_T_K), float(epsilon), prec, rtol,
                                                        q.ctypes.data, coarse.ctypes.data, stats.ctypes.data,
                                                        _lib.stream()))
    if prec == _lib.PRECISION_FP64:
        info = {"reflections": int(stats[0]), "spmv": int(stats[1]), "residual_power_W": float(stats[2])}
    else:
        info = {"refinements": int(stats[0]), "spmv": int(stats[1]), "relative_residual": float(stats[2]),
                "sweeps_per_refinement": int(stats[3])}
    return PrescribedChannels(float(T_mean_K), float(delta_T_K), float(epsilon), float(q[0]), float(q[1]),
                              float(q[2]), float(q[3]), coarse, info)


APPEND_CHANNEL_DIFFERENCE = 0.01
APPEND_SOURCE_DIFFERENCE = 0.05
"""A/B differences above which one more ray block is appended to each set (coupled.py:216-219)."""


def relative_difference(a: float, b: float) -> float:
    """|a - b| relative to the larger magnitude (coupled.py:197-198)."""

    a, b = float(a), float(b)
    return abs(a - b) / max(abs(a), abs(b), _TINY)


def _l1(x) -> float:
    return float(np.sum(np.abs(x)))


def ab_differences(set_a: list[PrescribedChannels], set_b: list[PrescribedChannels]) -> tuple[float, float]:
    """Disagreement of two ray sets over matching conditions (coupled.py:201-213): the largest
    relative difference of a wall channel (q_h or q_c), and the largest L1 difference of the
    8^3 coarse sources relative to the larger of their L1 norms."""

    walls, sources = [], []
    for a, b in zip(set_a, set_b):
        walls.extend((relative_difference(a.q_h, b.q_h), relative_difference(a.q_c, b.q_c)))
        norm = max(_l1(a.coarse_source), _l1(b.coarse_source), _TINY)
        sources.append(_l1(a.coarse_source - b.coarse_source) / norm)
    return max(walls), max(sources)


def append_required(channel_difference: float, source_difference: float) -> bool:
    """Whether the sets disagree enough to append one more ray block to each (coupled.py:216-219)."""

    return channel_difference > APPEND_CHANNEL_DIFFERENCE or source_difference > APPEND_SOURCE_DIFFERENCE


def cell_field_channels(operator: ExchangeOperator, patches, T_cells, T_hot_K: float, T_cold_K: float,
                        epsilon: float, *, reference_temperature_K: float | None = None, precision: str = "fp64",
                        relative_tolerance: float | None = None) -> PrescribedChannels:
    """Channels q_h, q_c, q_i of an arbitrary cell temperature field on the device (not in the reference).

    The radiation evaluation of evaluate_radiation (coupled.py:86-105) followed by the
    channel sums of prescribed_field_channels (coupled.py:185-193): walls at T_hot_K /
    T_cold_K, internal patches at the temperature of their owning cell, one solve on the
    resident operator.  ``T_cells`` is a float64 array (nx, ny, nz) on the host or a
    CUDA tensor; the returned ``T_mean_K``/``delta_T_K`` are the wall mean and span.
    """

    dev = _device_of(patches)
    prec = {"fp64": _lib.PRECISION_FP64, "mixed": _lib.PRECISION_MIXED}[precision]
    rtol = RADIOSITY_RTOL_FINAL if prec == _lib.PRECISION_FP64 else MIXED_RTOL
    if relative_tolerance is not None:
        rtol = float(relative_tolerance)
    if getattr(T_cells, "is_cuda", False):
        if T_cells.numel() != int(np.prod(dev.shape)) or str(T_cells.dtype) != "torch.float64":
            raise ValueError("T_cells must hold nx*ny*nz float64 values")
        src = T_cells
    else:
        src = np.ascontiguousarray(np.asarray(T_cells, dtype=np.float64))
        if src.size != int(np.prod(dev.shape)):
            raise ValueError("T_cells must hold nx*ny*nz values")
    nx, ny, nz = dev.shape
    coarse = np.empty(tuple(min(8, n) for n in (nx, ny, nz)))
    q = np.empty(4)
    stats = np.zeros(4)
    has_ref = reference_temperature_K is not None
    _lib.check(_lib.load().pr_cell_field_channels(dev.handle, operator.handle, _lib.ptr(src), float(T_hot_K),
                                                  float(T_cold_K), float(epsilon), int(has_ref),
                                                  float(reference_temperature_K) if has_ref else 0.0, prec, rtol,
                                                  q.ctypes.data, coarse.ctypes.data, stats.ctypes.data,
                                                  _lib.stream()))
    info = {"sweeps_or_reflections": int(stats[0]), "spmv": int(stats[1]), "residual": float(stats[2])}
    return PrescribedChannels(0.5 * (T_hot_K + T_cold_K), float(T_hot_K - T_cold_K), float(epsilon), float(q[0]),
                              float(q[1]), float(q[2]), float(q[3]), coarse, info)


# Strictly coupled solve (coupled.py:222-490) on the device

NEWTON_MAX_ITERATIONS = 8
NEWTON_RESIDUAL_W = 1.0e-13
NEWTON_STEP_K = 1.0e-10
GMRES_RESTART = 30
GMRES_MAX_ITERATIONS = 90
GMRES_RTOL = 1.0e-8
GMRES_ATOL = 1.0e-13
PCG_STEPS = (10, 20)
"""Preconditioner steps of the first attempt and of the restart from the same initial field."""


@dataclass
class CoupledResult:
    """Converged coupled field, its radiation state and the iteration record (coupled.py:314-337)."""

    temperature_K: np.ndarray
    state: RadiationState
    converged: bool
    newton_iterations: int
    linear_solves: list[dict] = field(default_factory=list)
    final_residual_inf_W: float = float("nan")
    preconditioner_steps: int = 0
    failure: str = ""
    metrics: dict = field(default_factory=dict, repr=False)

    @property
    def linear_residuals_pass(self) -> bool:
        """Every linear solve met ||r||_2 <= max(1e-13, 1e-8 ||b||_2)."""

        return bool(self.linear_solves) and all(
            s["converged"] and s["true_residual_l2_W"] <= max(1.0e-13, 1.0e-8 * s["rhs_l2_W"])
            for s in self.linear_solves
        )


def _coupled(system, operator: ExchangeOperator, patches, T_hot_K: float, T_cold_K: float, epsilon: float,
             T_initial: np.ndarray, preconditioner_steps: int) -> CoupledResult:
    dev = _device_of(patches)
    shape = system.shape
    if tuple(shape) != tuple(dev.shape):
        raise ValueError("conduction grid and patch geometry differ")
    n_cells = int(np.prod(shape))
    T0 = np.ascontiguousarray(np.asarray(T_initial, dtype=np.float64).ravel())
    T = np.empty(n_cells)
    q = np.empty(n_cells)
    P = dev.n_patches
    Tp, E, ab = np.empty(P), np.empty(P), np.empty(P)
    r = _lib.CoupledResultC()
    _lib.check(_lib.load().pr_coupled_solve(dev.handle, operator.handle, system.handle, float(T_hot_K),
                                            float(T_cold_K), float(epsilon), T0.ctypes.data,
                                            int(preconditioner_steps), T.ctypes.data, Tp.ctypes.data, E.ctypes.data,
                                            ab.ctypes.data, q.ctypes.data, ctypes.byref(r), _lib.stream()))
    radiosity = RadiosityResult(E, ab, ab - E, float(r.residual_power_W), int(r.series_iterations))
    state = RadiationState(Tp, radiosity.net_power_W, q.reshape(shape), radiosity)
    linear = [{"converged": bool(L.converged), "gmres_iterations": int(L.gmres_iterations),
               "rhs_l2_W": float(L.rhs_l2_W), "true_residual_l2_W": float(L.true_residual_l2_W),
               "true_residual_relative": float(L.true_residual_relative)} for L in r.linear[:r.n_linear]]
    metrics = {name: float(getattr(r, name)) for name in (
        "q_cond_hot_W_m2", "q_rad_hot_W_m2", "q_total_hot_W_m2", "q_cond_cold_W_m2", "q_rad_cold_W_m2",
        "q_total_cold_W_m2", "radiative_fraction_hot", "k_eff_apparent_W_mK", "wall_flux_mismatch_rel",
        "energy_residual_rel", "T_min_K", "T_max_K")}
    metrics["temperature_bound_violations"] = int(r.temperature_bound_violations)
    return CoupledResult(T.reshape(shape), state, bool(r.converged), int(r.newton_iterations), linear,
                         float(r.final_residual_inf_W), int(r.preconditioner_steps),
                         _lib.COUPLED_FAILURES.get(int(r.failure), "unknown failure"), metrics)


def newton_krylov(system, operator: ExchangeOperator, patches, T_hot_K: float, T_cold_K: float, epsilon: float,
                  T_initial: np.ndarray, preconditioner_steps: int) -> CoupledResult:
    """Newton-Krylov solve of A T - b - Q_rad(T) = 0 from T_initial (coupled.py:340-421), on the device.

    Converged when ||R||_inf <= 1e-13 W and the last update is at most 1e-10 K; radiosity
    is summed to 1e-8 inside the iteration and to 1e-13 for the returned state; trial
    fields outside [T_c, T_h] are rejected by the line search.
    """

    if int(preconditioner_steps) <= 0:
        raise ValueError("preconditioner_steps must be positive")
    return _coupled(system, operator, patches, T_hot_K, T_cold_K, epsilon, T_initial, preconditioner_steps)


def solve_coupled(system, operator: ExchangeOperator, patches, T_hot_K: float, T_cold_K: float, epsilon: float,
                  T_initial: np.ndarray) -> CoupledResult:
    """Coupled solve with 10 preconditioner steps, restarted from the same field with 20 if needed (coupled.py:423-440)."""

    return _coupled(system, operator, patches, T_hot_K, T_cold_K, epsilon, T_initial, 0)


def wall_flux_metrics(system, patches, result: CoupledResult, T_hot_K: float, T_cold_K: float) -> dict[str, float]:
    """Conductive, radiative and total wall fluxes (W m^-2) and the acceptance quantities (coupled.py:443-472).

    The device solve computes them from its final field and radiation state.
    """

    if not result.metrics:
        raise ValueError("result does not come from newton_krylov / solve_coupled")
    return dict(result.metrics)


_ACCEPTANCE = (
    ("Newton iteration converged", lambda r, m: r.converged),
    ("linear residuals within max(1e-13, 1e-8 ||b||)", lambda r, m: r.linear_residuals_pass),
    ("wall-flux mismatch <= 0.5 %", lambda r, m: m["wall_flux_mismatch_rel"] <= 0.005),
    ("global energy residual <= 1e-3", lambda r, m: m["energy_residual_rel"] <= 1.0e-3),
    ("temperature within the wall temperatures", lambda r, m: m["temperature_bound_violations"] == 0),
)
"""Acceptance conditions of a coupled solution and their names (coupled.py:475-490)."""


def acceptance_failures(result: CoupledResult, metrics: dict[str, float]) -> list[str]:
    """Names of the acceptance conditions the solution does not meet; empty when it is accepted."""

    return [name for name, holds in _ACCEPTANCE if not holds(result, metrics)]
"""Penetration response of a slab of digital microstructure, on a B200.

Mirrors ``porerad.penetration`` (porerad/penetration.py).  Rays enter through x = 0 at
uniform transverse positions with Lambertian directions about the face normal; at a solid
surface a ray is absorbed with probability eps or reflected diffusely, for at most 1000
reflections.  A ray leaving through x = 0 counts as reflected (R), through x = N as
transmitted (T), one absorbed by the skeleton as absorbed (A).  The ray kernel runs in
libporerad (``pr_penetration``); the penetration flux is q_pen = q_pp T.
"""

from __future__ import annotations

import math

import numpy as np

from . import _lib
from .constants import SIGMA
from .properties import RESTART_CODES, _geometry, run_concurrently, seed_average, solid_along_x  # noqa: F401

SEEDS = (321, 654)
N_RAYS = 500_000
MAX_BOUNCES = 1000
RESTART_RULES = ("article", "hit_point")


def parallel_plate_flux(T_hot: float, T_cold: float, epsilon: float) -> float:
    """Net radiative flux between gray diffuse parallel plates of emissivity eps, W m^-2 (penetration.py:41-44)."""

    eps = float(epsilon)
    return float(SIGMA * (float(T_hot) ** 4 - float(T_cold) ** 4) / (1.0 / eps + 1.0 / eps - 1.0))


def penetration_flux(transmittance: float, epsilon: float, T_mean: float, delta_T: float = 10.0) -> float:
    """q_pen = q_pp T at mean temperature T_mean and wall temperature difference delta_T (penetration.py:47-51)."""

    T_hot = float(T_mean) + 0.5 * float(delta_T)
    T_cold = float(T_mean) - 0.5 * float(delta_T)
    return float(parallel_plate_flux(T_hot, T_cold, epsilon) * transmittance)


def _binomial(count: int, n: int) -> tuple[float, float]:
    p = float(count) / float(n)
    return p, float(math.sqrt(max(p * (1.0 - p), 0.0) / n))


def trace_penetration(phases: np.ndarray, axis: str, epsilon: float, *, n_rays: int = N_RAYS, seed: int = SEEDS[0],
                      restart: str = "article", max_bounces: int = MAX_BOUNCES, _geo=None) -> dict:
    """R, T, A with binomial standard errors for one geometry, axis, eps and seed (penetration.py:281-305)."""

    if restart not in RESTART_RULES:
        raise ValueError(f"restart must be one of {RESTART_RULES}")
    geo = _geo or _geometry(phases, axis)
    counts = np.zeros(4, np.int64)
    _lib.check(_lib.load().pr_penetration(geo.handle, float(epsilon), int(n_rays), int(seed) & 0xFFFFFFFF,
                                          RESTART_CODES[restart], int(max_bounces), counts.ctypes.data, _lib.stream()))
    n = int(n_rays)
    out = {"n_rays": n, "terminated": int(counts[3])}
    for name, count in (("reflectance", counts[0]), ("transmittance", counts[1]), ("absorptance", counts[2])):
        out[name], out[f"{name}_se"] = _binomial(int(count), n)
    return out


def penetration_response(phases: np.ndarray, axis: str, epsilon: float, *, seeds=SEEDS, n_rays: int = N_RAYS,
                         restart: str = "article") -> dict:
    """R, T, A of one geometry, axis and emissivity, averaged over independent seeds (penetration.py:308-316)."""

    geo = _geometry(phases, axis)
    try:
        runs = run_concurrently([(trace_penetration, (phases, axis, epsilon),
                                  dict(n_rays=n_rays, seed=s, restart=restart, _geo=geo)) for s in seeds])
    finally:
        geo.close()
    out = {"n_rays": int(sum(r["n_rays"] for r in runs)), "terminated": int(sum(r["terminated"] for r in runs))}
    for key in ("reflectance", "transmittance", "absorptance"):
        out[key], out[f"{key}_se"] = seed_average([r[key] for r in runs], [r[f"{key}_se"] for r in runs])
    return out

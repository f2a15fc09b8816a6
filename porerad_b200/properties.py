"""Equivalent radiative properties from pore-scale ray statistics, on a B200.

Mirrors ``porerad.properties`` (porerad/properties.py).  Rays enter the slab at normal
incidence through x = 0 at uniform transverse positions; the first path segment gives an
interception by the solid or a right-censored crossing (the extinction coefficient beta per
cell is the censored maximum-likelihood rate), and at every surface interaction a ray is
absorbed with probability eps or reflected into a Lambertian direction (albedo omega is the
reflected fraction, g the mean cosine between incoming and reflected directions).  The ray
kernel runs in libporerad (``pr_radiative_properties``); this module turns its tallies into
the reference's estimates.
"""

from __future__ import annotations

import ctypes
import math

import numpy as np

from . import _lib
from .view_factors import DeviceGeometry

SEEDS = (123, 456)
RESTART_RULES = ("article", "hit_point")
N_RAYS = 200_000
MAX_BOUNCES = 1000
RESTART_CODES = {"article": 0, "hit_point": 1}


def solid_along_x(phases: np.ndarray, axis: str) -> np.ndarray:
    """The solid indicator with the transfer axis moved to the first index (properties.py:41-44)."""

    solid = np.asarray(phases) == 1
    return np.ascontiguousarray(np.moveaxis(solid, "xyz".index(axis), 0).astype(np.uint8))


def right_censored_mle(events: np.ndarray, censored: np.ndarray) -> tuple[float, float]:
    """Rate estimate events / total exposure and its standard error (properties.py:47-53)."""

    exposure = float(np.sum(events) + np.sum(censored))
    n_events = int(np.asarray(events).size)
    if exposure <= 0.0 or n_events == 0:
        return 0.0, 0.0
    return float(n_events / exposure), float(math.sqrt(n_events) / exposure)


def _geometry(phases, axis: str) -> DeviceGeometry:
    return DeviceGeometry(solid_along_x(phases, axis), 1.0)


from .streams import WORKERS as RUN_STREAMS, run_concurrently  # noqa: E402,F401


def trace_properties(phases: np.ndarray, axis: str, epsilon: float, *, n_rays: int = N_RAYS, seed: int = SEEDS[0],
                     max_bounces: int = MAX_BOUNCES, restart: str = "article", _geo: DeviceGeometry | None = None
                     ) -> dict:
    """beta (per cell), omega and g for one geometry, transfer axis, emissivity and seed (properties.py:56-279)."""

    if restart not in RESTART_RULES:
        raise ValueError(f"restart must be one of {RESTART_RULES}")
    geo = _geo or _geometry(phases, axis)
    t = _lib.PropertiesTally()
    _lib.check(_lib.load().pr_radiative_properties(geo.handle, float(epsilon), int(n_rays), int(seed) & 0xFFFFFFFF,
                                                   RESTART_CODES[restart], int(max_bounces), ctypes.byref(t),
                                                   _lib.stream()))
    exposure = float(t.event_length) + float(t.censored_length)
    beta, beta_se = (0.0, 0.0) if exposure <= 0.0 or t.events == 0 else (
        t.events / exposure, math.sqrt(t.events) / exposure)
    interactions, scattered = int(t.interactions), int(t.scattered)
    omega = scattered / interactions if interactions else 0.0
    omega_se = math.sqrt(omega * (1.0 - omega) / interactions) if interactions else 0.0
    g, g_se = 0.0, 0.0
    if scattered > 0:
        g = float(t.sum_mu / scattered)
        if scattered > 1:
            g_se = math.sqrt(max(0.0, float((t.sum_mu2 - scattered * g * g) / (scattered - 1))) / scattered)
    return {"n_rays": int(n_rays), "beta": beta, "beta_se": beta_se, "omega": omega, "omega_se": omega_se, "g": g,
            "g_se": g_se}


def seed_average(values, ses):
    """Mean over seeds; the standard error combines within-seed and between-seed variance (properties.py:282-289)."""

    values, ses = np.asarray(values, float), np.asarray(ses, float)
    mean = float(values.mean())
    within = float(np.sum(ses**2) / values.size**2)
    between = float(values.var(ddof=1) / values.size) if values.size > 1 else 0.0
    return mean, float(np.sqrt(max(0.0, within + between)))


def identify_properties(phases: np.ndarray, axis: str, epsilon: float, *, seeds=SEEDS, n_rays: int = N_RAYS,
                        restart: str = "article") -> dict:
    """Properties of one geometry, axis and emissivity, averaged over independent seeds (properties.py:292-305)."""

    geo = _geometry(phases, axis)
    try:
        runs = run_concurrently([(trace_properties, (phases, axis, epsilon),
                                  dict(n_rays=n_rays, seed=s, restart=restart, _geo=geo)) for s in seeds])
    finally:
        geo.close()
    out = {"n_rays": int(sum(r["n_rays"] for r in runs))}
    for key in ("beta", "omega", "g"):
        mean, se = seed_average([r[key] for r in runs], [r[f"{key}_se"] for r in runs])
        out[key], out[f"{key}_se"] = mean, se
    out["beta_ci95_low"] = out["beta"] - 1.96 * out["beta_se"]
    out["beta_ci95_high"] = out["beta"] + 1.96 * out["beta_se"]
    return out

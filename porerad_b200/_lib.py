"""ctypes binding of libporerad.so (include/porerad.h).

The library is the only compute path of porerad_b200: if it is missing or no CUDA
device is visible, every call raises instead of falling back to the CPU.
"""

from __future__ import annotations

import ctypes
import os
import threading
from pathlib import Path

import numpy as np

_PKG = Path(__file__).resolve().parent
LIB_PATH = _PKG / "libporerad.so"

PR_OK = 0
PR_ERR_ARG = 1
PR_ERR_CUDA = 2
PR_ERR_OOM = 3
PR_ERR_UNRESOLVED = 4
PR_ERR_ACCOUNTING = 5
PR_ERR_NOT_CLOSED = 6
PR_ERR_BALANCE = 7
PR_ERR_SERIES = 8
PR_ERR_LIMIT = 9

BALANCE_METHODS = {0: "none", 1: "anderson", 2: "multiplicative"}

APPLY_RAW, APPLY_RAW_T, APPLY_SYM, APPLY_MATVEC, APPLY_RMATVEC = range(5)
PRECISION_FP64, PRECISION_MIXED = 0, 1


class PorerdDeviceError(RuntimeError):
    """A CUDA failure inside libporerad (not one of the reference's own errors)."""


class PCG64Seed(ctypes.Structure):
    _fields_ = [("state_hi", ctypes.c_uint64), ("state_lo", ctypes.c_uint64),
                ("inc_hi", ctypes.c_uint64), ("inc_lo", ctypes.c_uint64)]


_vp = ctypes.c_void_p
_i64 = ctypes.c_int64
_i32 = ctypes.c_int
_f64 = ctypes.c_double

COUPLED_MAX_LINEAR = 16
COUPLED_FAILURES = {0: "", 1: "linear solve did not converge", 2: "line search failed",
                    3: "maximum Newton iterations reached"}


class PropertiesTally(ctypes.Structure):
    """pr_properties_tally: tallies of one properties run."""

    _fields_ = [("events", _i64), ("censored", _i64), ("interactions", _i64), ("scattered", _i64),
                ("event_length", _f64), ("censored_length", _f64), ("sum_mu", _f64), ("sum_mu2", _f64)]


class Morphology(ctypes.Structure):
    """pr_morphology: integer counts behind the morphology descriptors."""

    _fields_ = [("cells", _i64), ("solid_cells", _i64), ("pore_cells", _i64), ("interface_faces", _i64 * 3),
                ("periodic_faces", _i64 * 3), ("pore_runs", _i64 * 3), ("all_pore_lines", _i64 * 3),
                ("pore_clusters", _i64), ("largest_pore_cluster", _i64), ("pore_percolates", _i32 * 3)]


class Shape(ctypes.Structure):
    """pr_shape: one ellipsoid or cylinder of a rendered microstructure."""

    _fields_ = [("kind", _i32), ("pad", _i32), ("center", _f64 * 3), ("R", _f64 * 9), ("radii", _f64 * 3)]


class CoupledLinear(ctypes.Structure):
    """pr_coupled_linear: one Newton correction's linear solve."""

    _fields_ = [("converged", _i32), ("gmres_iterations", _i32), ("rhs_l2_W", _f64),
                ("true_residual_l2_W", _f64), ("true_residual_relative", _f64)]


class CoupledResultC(ctypes.Structure):
    """pr_coupled_result: the returned attempt of a coupled solve and its wall-flux metrics."""

    _fields_ = [("converged", _i32), ("newton_iterations", _i32), ("preconditioner_steps", _i32),
                ("failure", _i32), ("linear_residuals_pass", _i32), ("n_linear", _i32),
                ("linear", CoupledLinear * COUPLED_MAX_LINEAR), ("final_residual_inf_W", _f64),
                ("q_cond_hot_W_m2", _f64), ("q_rad_hot_W_m2", _f64), ("q_total_hot_W_m2", _f64),
                ("q_cond_cold_W_m2", _f64), ("q_rad_cold_W_m2", _f64), ("q_total_cold_W_m2", _f64),
                ("radiative_fraction_hot", _f64), ("k_eff_apparent_W_mK", _f64), ("wall_flux_mismatch_rel", _f64),
                ("energy_residual_rel", _f64), ("global_energy_residual_W", _f64), ("residual_power_W", _f64),
                ("T_min_K", _f64), ("T_max_K", _f64), ("temperature_bound_violations", _i64),
                ("series_iterations", _i64)]

_SIGNATURES = {
    "pr_last_error": (ctypes.c_char_p, []),
    "pr_version": (_i32, []),
    "pr_case_create": (_i32, [_vp, _i64, _i64, _i64, _f64, _vp, ctypes.POINTER(_vp)]),
    "pr_case_info": (_i32, [_vp, ctypes.POINTER(_i64), ctypes.POINTER(_i64), ctypes.POINTER(ctypes.c_size_t)]),
    "pr_case_patches": (_i32, [_vp] * 11 + [_vp]),
    "pr_case_destroy": (None, [_vp]),
    "pr_generate_rays": (_i32, [_vp, _i64, _i64, _i64, _vp, _vp, _vp, _vp]),
    "pr_trace_first_hit": (_i32, [_vp, _vp, _vp, _i64, _vp, ctypes.POINTER(_i64), _vp]),
    "pr_first_hit_counts": (_i32, [_vp, _i64, _vp, _i32, _vp, ctypes.POINTER(_vp)]),
    "pr_first_hit_counts_batch": (_i32, [_vp, _i32, _i64, _vp, _i32, _vp, _vp]),
    "pr_counts_info": (_i32, [_vp, ctypes.POINTER(_i64), ctypes.POINTER(_i64), ctypes.POINTER(_i64),
                              ctypes.POINTER(_i64)]),
    "pr_counts_copy": (_i32, [_vp, _vp, _vp, _vp, _vp, _vp]),
    "pr_counts_rows": (_i32, [_vp, _i64, _i64, ctypes.POINTER(_i64), _vp, _vp, _vp, _vp]),
    "pr_first_hit_counts_host": (_i32, [_vp, _i64, _vp, ctypes.c_int, _vp, _vp, _vp, _vp, _i64,
                                        ctypes.POINTER(_i64)]),
    "pr_host_block": (_i32, [ctypes.c_longlong, ctypes.POINTER(_vp)]),
    "pr_host_block_release": (_i32, [_vp]),
    "pr_host_blocks_trim": (_i32, [ctypes.c_longlong]),
    "pr_host_blocks_stats": (_i32, [ctypes.POINTER(ctypes.c_longlong)] * 4),
    "pr_counts_from_edges": (_i32, [_vp, _vp, _vp, _i64, _i64, _vp, ctypes.POINTER(_vp)]),
    "pr_counts_from_tables": (_i32, [_vp, _vp, _vp, _vp, ctypes.c_int, _i64, _vp, ctypes.POINTER(_vp)]),
    "pr_counts_merge": (_i32, [_vp, _vp, _vp, ctypes.POINTER(_vp)]),
    "pr_counts_destroy": (None, [_vp]),
    "pr_operator_create": (_i32, [_vp, _vp, _vp, _f64, _f64, _vp, ctypes.POINTER(_vp)]),
    "pr_operator_create_batch": (_i32, [_vp, _vp, _vp, _i32, _f64, _f64, _vp, _vp]),
    "pr_operator_info": (_i32, [_vp, _vp, ctypes.POINTER(_i32), ctypes.POINTER(_i32), ctypes.POINTER(_f64),
                                ctypes.POINTER(_i64), ctypes.POINTER(_i64), ctypes.POINTER(_i64)]),
    "pr_operator_apply": (_i32, [_vp, _i32, _vp, _vp, _vp]),
    "pr_operator_reciprocity_error": (_i32, [_vp, ctypes.POINTER(_f64), _vp]),
    "pr_operator_edges": (_i32, [_vp, _vp, _vp, _vp, _vp]),
    "pr_operator_destroy": (None, [_vp]),
    "pr_reflection_series": (_i32, [_vp, _vp, _vp, _f64, _i64, _vp, ctypes.POINTER(_f64), ctypes.POINTER(_i64),
                                    _vp]),
    "pr_net_patch_power": (_i32, [_vp, _vp, _vp, _vp, _f64, _i32, _f64, _i64, _vp, _vp, _vp,
                                  ctypes.POINTER(_f64), ctypes.POINTER(_i64), _vp]),
    "pr_net_patch_power_jvp": (_i32, [_vp, _vp, _vp, _vp, _vp, _f64, _vp, _vp]),
    "pr_prescribed_field_channels": (_i32, [_vp, _vp, _f64, _f64, _f64, _i32, _f64, _vp, _vp, _vp, _vp]),
    "pr_cell_field_channels": (_i32, [_vp, _vp, _vp, _f64, _f64, _f64, _i32, _f64, _i32, _f64, _vp, _vp, _vp, _vp]),
    "pr_conduction_create": (_i32, [_vp, _i64, _i64, _i64, _f64, _vp, ctypes.POINTER(_vp)]),
    "pr_conduction_destroy": (None, [_vp]),
    "pr_conduction_arrays": (_i32, [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "pr_conduction_apply": (_i32, [_vp, _vp, _vp, _vp]),
    "pr_conduction_solve": (_i32, [_vp, _f64, _f64, _f64, _vp, ctypes.POINTER(_i64), ctypes.POINTER(_f64), _vp]),
    "pr_conduction_wall_fluxes": (_i32, [_vp, _vp, _f64, _f64, ctypes.POINTER(_f64), ctypes.POINTER(_f64), _vp]),
    "pr_coupled_solve": (_i32, [_vp, _vp, _vp, _f64, _f64, _f64, _vp, _i32, _vp, _vp, _vp, _vp, _vp,
                                ctypes.POINTER(CoupledResultC), _vp]),
    "pr_radiative_properties": (_i32, [_vp, _f64, _i64, ctypes.c_uint32, _i32, _i32,
                                       ctypes.POINTER(PropertiesTally), _vp]),
    "pr_penetration": (_i32, [_vp, _f64, _i64, ctypes.c_uint32, _i32, _i32, _vp, _vp]),
    "pr_morphology_counts": (_i32, [_vp, _i64, _i64, _i64, _i32, _vp, _vp, _vp, _vp, _vp]),
    "pr_render_shapes": (_i32, [_i64, _vp, _i32, _vp, _vp, _vp]),
    "pr_stamp_fibers": (_i32, [_i64, _vp, _vp, _vp, _vp, _i32, _i32, _vp, _vp, _vp]),
    "pr_stamp_cells": (_i32, [_i64, _vp, _vp, _vp, _vp, _i32, _i32, _i32, _vp, _vp, _vp]),
    "pr_voronoi_edge_field": (_i32, [_i64, _vp, _i32, _vp, _vp]),
    "pr_lamellar_field": (_i32, [_i64, _vp, _vp, _vp, _f64, _f64, _vp, _vp, _vp]),
    "pr_stamp_first": (_i32, [_i64, _vp, _vp, _vp, _i64, _i32, _i32, _vp, _vp, _vp, _vp]),
    "pr_first_threshold": (_i32, [_vp, _i64, _i32, _i32, _vp, _vp]),
    "pr_quantile_threshold": (_i32, [_vp, _i64, _f64, _i32, _vp, _vp, _vp, _vp]),
    "pr_timers_enable": (None, [_i32]),
    "pr_timers_reset": (None, []),
    "pr_timers_read": (_i32, [_i32, ctypes.POINTER(ctypes.c_longlong), ctypes.POINTER(_f64)]),
    "pr_kernel_launches": (ctypes.c_longlong, []),
    "pr_trace_set_variant": (_i32, [_i32]),
    "pr_memory_stats": (_i32, [_i32, ctypes.POINTER(ctypes.c_longlong), ctypes.POINTER(ctypes.c_longlong),
                               ctypes.POINTER(ctypes.c_longlong), ctypes.POINTER(ctypes.c_longlong)]),
    "pr_memory_release_cached": (_i32, [_i32]),
    "pr_trace_variant_info": (_i32, [ctypes.POINTER(_i32), ctypes.POINTER(_i32), ctypes.POINTER(ctypes.c_char_p)]),
}

TIMER_TRACE, TIMER_RLE, TIMER_BALANCE, TIMER_SERIES, TIMER_CHEB, TIMER_REFINE, TIMER_MORPH, TIMER_LABEL, TIMER_RENDER = range(9)

_lock = threading.Lock()
_lib = None


def load() -> ctypes.CDLL:
    """The loaded library; raises if it was not built or cannot be loaded."""

    global _lib
    if _lib is not None:
        return _lib
    with _lock:
        if _lib is None:
            if not LIB_PATH.is_file():
                raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m porerad_b200.build` "
                                   "(porerad_b200 has no CPU implementation)")
            lib = ctypes.CDLL(str(LIB_PATH), mode=os.RTLD_LOCAL if hasattr(os, "RTLD_LOCAL") else 0)
            for name, (res, args) in _SIGNATURES.items():
                fn = getattr(lib, name)
                fn.restype = res
                fn.argtypes = args
            _lib = lib
    return _lib


def last_error() -> str:
    msg = load().pr_last_error()
    return msg.decode("utf-8", "replace") if msg else ""


def check(status: int) -> None:
    """Map a libporerad status to the exception the reference raises in the same case."""

    if status == PR_OK:
        return
    msg = last_error()
    if status in (PR_ERR_ARG, PR_ERR_ACCOUNTING):
        raise ValueError(msg)
    if status in (PR_ERR_UNRESOLVED, PR_ERR_NOT_CLOSED, PR_ERR_BALANCE, PR_ERR_SERIES):
        raise RuntimeError(msg)
    if status == PR_ERR_OOM:
        raise MemoryError(msg)
    if status == PR_ERR_LIMIT:
        raise NotImplementedError(msg)
    raise PorerdDeviceError(msg)


def ptr(a) -> int | None:
    """Data pointer of a C-contiguous NumPy array or CUDA tensor (None stays NULL)."""

    if a is None:
        return None
    if isinstance(a, np.ndarray):
        if not a.flags["C_CONTIGUOUS"]:
            raise ValueError("array must be C-contiguous")
        return a.ctypes.data
    if hasattr(a, "data_ptr"):
        return a.data_ptr()
    raise TypeError(f"unsupported array type {type(a)!r}")


def seeds_struct(states) -> ctypes.Array:
    """pr_pcg64 array from (state, inc) pairs of Python ints."""

    arr = (PCG64Seed * len(states))()
    for k, (st, inc) in enumerate(states):
        arr[k].state_hi = (st >> 64) & 0xFFFFFFFFFFFFFFFF
        arr[k].state_lo = st & 0xFFFFFFFFFFFFFFFF
        arr[k].inc_hi = (inc >> 64) & 0xFFFFFFFFFFFFFFFF
        arr[k].inc_lo = inc & 0xFFFFFFFFFFFFFFFF
    return arr


def pcg64_state(seed: int) -> tuple[int, int]:
    """(state, inc) that numpy.random.PCG64(seed) starts from (SeedSequence seeding)."""

    st = np.random.PCG64(int(seed)).state["state"]
    return int(st["state"]), int(st["inc"])


class Handle:
    """Owner of one opaque library object; destroyed with its destructor function."""

    __slots__ = ("value", "_destroy", "__weakref__")

    def __init__(self, value: int, destroy: str):
        self.value = value
        self._destroy = destroy

    def close(self) -> None:
        if self.value:
            getattr(load(), self._destroy)(ctypes.c_void_p(self.value))
            self.value = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_tls = threading.local()


class use_stream:
    """Context manager: calls made by this thread inside it run on ``stream``.

    ``stream`` is a torch.cuda.Stream, a raw cudaStream_t (int) or None (the legacy
    default stream).  Worker threads of the serving loop each hold their own stream so
    that cases overlap on the device.
    """

    def __init__(self, stream):
        self.stream = stream_arg(stream)

    def __enter__(self):
        self.prev = getattr(_tls, "stream", None)
        _tls.stream = self.stream
        return self

    def __exit__(self, *exc):
        _tls.stream = self.prev


def memory_stats(device: int = 0) -> dict:
    """Device-memory cache counters of libporerad on one device."""

    v = [ctypes.c_longlong() for _ in range(4)]
    check(load().pr_memory_stats(int(device), *[ctypes.byref(x) for x in v]))
    return dict(zip(("cached_bytes", "live_bytes", "device_mallocs", "cache_hits"), (int(x.value) for x in v)))


def release_cached_memory(device: int = 0) -> None:
    """Return the library's cached device blocks to the driver (like emptying a caching allocator)."""

    check(load().pr_memory_release_cached(int(device)))


def trace_variant() -> tuple[int, str]:
    """(index, name) of the traversal variant the last count pass used (chosen by the autotuner)."""

    n, last, name = ctypes.c_int(), ctypes.c_int(), ctypes.c_char_p()
    check(load().pr_trace_variant_info(ctypes.byref(n), ctypes.byref(last), ctypes.byref(name)))
    return int(last.value), name.value.decode()


def stream() -> int | None:
    """The cudaStream_t of the calling thread (None = legacy default stream)."""

    return getattr(_tls, "stream", None)


def stream_arg(stream) -> int | None:
    """cudaStream_t from None (legacy default stream), an int, or a torch.cuda.Stream."""

    if stream is None:
        return None
    if isinstance(stream, int):
        return stream or None
    return int(stream.cuda_stream) or None

#!/usr/bin/env python
"""Benchmark of the surface-radiation path on B200: first-hit rays/s and cases/s.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload c2|c1|c3|c4|c5|coupled|descriptors|generators|properties|archetypes] [--impl ours|reference]

Workload c2 (default, the configuration the headline metric is quoted on): open-cell
foam (OF) N=128^3, phi = 0.10, 64 Poisson seeds, geometry seed 1; 1000 rays per patch
in two independently seeded sets A and B; eps = 0.6; prescribed field 650 -> 750 K
along x (T_m 700 K, dT 100 K); H = 1 cm.

One step = one case through the whole path, device-resident: surface patches ->
fused ray generation + first-hit counts of set A and of set B -> pooled A+B counts ->
three balanced exchange operators (A, B, A+B) -> mixed-precision radiosity channels
for each (binary32 Chebyshev sweeps in binary64 refinement) -> q_h, q_c, q_i and
the A/B wall-channel and coarse-source differences on the host.  ``value`` = rays
traced per step x steps / device time; ``e2e`` = the same step through the public
API from pinned host buffers (host->device copy of the phases and device->host copy
of the results inside the timed region); ``plain`` = the drop-in NumPy API path of
the reference's case driver (count tables and operators round-trip through host
arrays, binary64 series).

With --impl reference, the reference's CPU algorithm (the oracle port: NumPy PCG64
rays + the OpenMP C traversal + np.unique) times a bounded sample of the same
workload on all host cores.
"""

from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

WORKLOADS = {
    "c2": dict(workload="OF N=128^3 phi=0.10 (64 Poisson seeds, geometry seed 1), 1000 rays/patch x sets A,B, "
                        "eps 0.6, T 650->750 K along x, FP32+FP64-refinement radiosity",
               arch="OF", n=128, phi=0.10, seed=1, rays=1000, sets=2, eps=0.6, T_m=700.0, dT=100.0, H=0.01),
    "c4": dict(workload="serving: Poisson stream of geometry-axis cases, N in {96,128,160,192}, archetypes OF/FI/FA/TL, "
                        "phi U(0.05,0.20), seeds 0-99, eps U(0.3,0.95), T_mean U(500,900) K with 100 K span, "
                        "250-1000 rays/patch; served = continuous batching, mixed precision",
               requests=200, plain_requests=24, stream_seed=2026, slots=4, H=0.01),
    "c3": dict(workload="batched sweep: 48 geometries = OF/FI/FA/TL x phi {0.05,0.10,0.20} x seeds 0-3, N=128^3, "
                        "500 rays/patch, eps from {0.3,0.6,0.9} and axis from {x,y,z} (RNG seed 3); all first-hit "
                        "counts in shared persistent traversal launches, all operators balanced together (one "
                        "product launch per iteration for every operator), mixed-precision solves overlapped on "
                        "4 streams",
               n=128, rays=500, phis=(0.05, 0.10, 0.20), seeds=4, H=0.01, T_m=700.0, dT=20.0, slots=4, pick_seed=3),
    "c5": dict(workload="coupled-size stress: TL and FA N=192^3 phi=0.10, 1000 rays/patch x sets A,B,C, eps 0.6, "
                        "T 690->710 K along x; then 20 solves at T_cell + N(0, 5 K) per voxel (seed 2) on the resident "
                        "operator, FP32+FP64-refinement vs FP64 flux error per solve",
               archs=("TL", "FA"), n=192, phi=0.10, seed=0, rays=1000, sets=3, eps=0.6, T_m=700.0, dT=20.0, H=0.01,
               solves=20, sigma_K=5.0),
    "coupled": dict(workload="strictly coupled radiation-conduction solve of the archived case "
                             "coupled_OF_x_T700_eps0.6_N128 (canonical OF 128^3, 4 seed blocks x 64 rays/patch, eps 0.6, "
                             "690->710 K along x): counts, balanced operator, conduction assembly + PCG, Newton-Krylov "
                             "(flexible GMRES, radiosity JVP, Jacobi-PCG preconditioner, line search)",
                    case_id="coupled_OF_x_T700_eps0.6_N128"),
    "descriptors": dict(workload="morphology descriptors (scalar: phi_s, A_s, L_m, axial pore chords, 26-connected "
                                 "pore percolation and largest cluster; directional: periodic chord histograms, "
                                 "lineal path, interface normals) of the 22 stored 128^3 microstructures (OF/FI/FA/TL "
                                 "core, canonical and matched pairs); L2 flushed before each step"),
    "generators": dict(workload="the reference's core microstructure library: OF/FI/FA/TL x phi {0.05,0.10,0.15}, "
                                "N=128^3, seeds 0,1,... until 4 per cell pass the acceptance rules (scalar "
                                "descriptors); 48 accepted arrays, bit-identical to data/microstructures.csv"),
    "properties": dict(workload="multi-bounce identifications of the archived set: 12 stored core 128^3 microstructures "
                                "x axes x/y/z x eps {0.3,0.6,0.9}: radiative properties (2 seeds x 2e5 normal-incidence "
                                "rays) and penetration response (2 seeds x 5e5 Lambertian rays), restart 'article', "
                                "at most 1000 reflections"),
    "archetypes": dict(workload="benchmark archetypes generated on the device for serving: OF/FI/FA/TL at N = 128 and "
                                "192, phi 0.10, seed 1 (geometry.make_device, bit-identical to the host definition)"),
    "c1": dict(workload="FI N=64^3 phi=0.10 (r=2, seed 0), 64 rays/patch x 1 set, eps 0.9, T 600->700 K along x, "
                        "FP64 radiosity",
               arch="FI", n=64, phi=0.10, seed=0, rays=64, sets=1, eps=0.9, T_m=650.0, dT=100.0, H=0.01),
}


def parse_args():
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--workload", default="c2", choices=sorted(WORKLOADS))
    ap.add_argument("--impl", default="ours", choices=("ours", "reference"))
    ap.add_argument("--no-plain", action="store_true", help="skip the plain drop-in path measurement")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline sample")
    ap.add_argument("--cpu-seconds", type=float, default=12.0, help="target CPU time of one baseline sample")
    ap.add_argument("--rays", type=int, default=None,
                    help="override rays per patch (small cases of the same kernels for profiling; not a bench line)")
    return ap.parse_args()


def ray_seeds(cfg):
    from porerad_b200.geometry import ray_set_seed

    return [ray_set_seed(cfg["seed"], s) for s in range(cfg["sets"])]


def make_phases(cfg):
    from porerad_b200 import geometry

    return geometry.make(cfg["arch"], cfg["n"], cfg["phi"], cfg["seed"])


# --------------------------------------------------------------------------- our arm

def served_step(phases, cfg, seeds, precision="mixed", serial=False, timers=False):
    """One case, device-resident; returns host scalars (the only device->host data).

    ``serial`` builds and solves the operators one after the other on the caller's stream
    instead of on worker streams at once; ``timers`` (with ``serial``) records the library's
    kernel timers of the operator stage alone in ``out["_timers"]``.
    """

    from porerad_b200 import coupled, exchange, view_factors as vf

    geo = vf.DeviceGeometry(phases, cfg["H"])
    p = vf.SurfacePatches(H_m=cfg["H"], _device=geo)
    tables = [vf.first_hit_counts_pooled(p, cfg["rays"], [s]) for s in seeds]
    pooled = tables[0] if len(tables) == 1 else tables[0].merge(tables[1])
    area = np.full(geo.n_patches, (cfg["H"] / cfg["n"]) ** 2)
    P = geo.n_patches
    out = {"rays": sum(t.rays_traced for t in tables), "steps": sum(t.dda_steps for t in tables),
           "n_patches": P, "nnz": pooled.nnz, "sets": []}
    n_ops = len(tables) + (1 if len(tables) > 1 else 0)
    # host->device: phases (e2e form only), 128 jump maps per seed, rays + areas per operator;
    # device->host: the scale vector per operator, q (4), coarse source (8^3) and stats (4) per solve
    out["h2d"] = 32 * 130 * len(seeds) + n_ops * P * 16
    out["d2h"] = n_ops * (P * 8 + 8 * (4 + 512 + 4))
    ops = []

    def per_set(t, n_sets):
        rays = np.full(geo.n_patches, cfg["rays"] * n_sets, np.int64)
        op = exchange.ExchangeOperator(t, None, None, rays, area)
        return op, coupled.prescribed_field_channels(op, p, cfg["T_m"], cfg["dT"], cfg["eps"], precision=precision)

    # the operators and solves of the sets and of their pool are independent: on worker streams at once
    from porerad_b200 import streams

    jobs = [(per_set, (t, 1), {}) for t in (tables if len(tables) > 1 else [])] + [(per_set, (pooled, len(seeds)), {})]
    if serial:
        from porerad_b200 import _lib

        lib = _lib.load()
        if timers:
            import torch

            torch.cuda.synchronize()
            lib.pr_timers_reset()
            lib.pr_timers_enable(1)
        done = [f(*a, **kw) for f, a, kw in jobs]
        if timers:
            torch.cuda.synchronize()
            lib.pr_timers_enable(0)
            out["_timers"] = _timer_values(lib, ("balance", "series", "cheb", "refine"))
    else:
        done = streams.run_concurrently(jobs)
    for op, ch in done[:-1]:
        out["sets"].append(ch)
        ops.append(op)
    op, ch = done[-1]
    out["final"] = ch
    out["nnz_symmetric"] = op.nnz_symmetric
    # products of every operator of the step: (entries of S', products made) for the roofline
    out["products"] = [(o.nnz_symmetric, o.spmv_calls) for o in ops + [op]]
    out["balance"] = (op.balance_method, op.balance_iterations, op.row_sum_error)
    out["_keep"] = (geo, p, tables, pooled, op, ops)
    return out


def release(res):
    geo, p, tables, pooled, op, ops = res.pop("_keep")
    for o in ops + [op]:
        o.close()
    for t in set(tables + [pooled]):
        t.close()
    geo.close()


def plain_step(phases_host, cfg, seeds, stages=None):
    """The reference case driver's call sequence through the drop-in NumPy API.

    ``stages`` (a dict) receives the wall-clock seconds of each stage of the sequence.
    """

    from porerad_b200 import coupled, exchange, view_factors as vf

    st = stages if stages is not None else {}

    def lap(name, t0):
        st[name] = st.get(name, 0.0) + time.perf_counter() - t0
        return time.perf_counter()

    t = time.perf_counter()
    p = vf.build_surface_patches(phases_host, cfg["H"])
    area = p.patch_area_m2
    t = lap("patches", t)
    counts = {s: vf.first_hit_counts(p, cfg["rays"], s) for s in seeds}
    t = lap("first_hit_counts (device counts, arrays to host)", t)
    chs = []
    groups = [[s] for s in seeds] + ([seeds] if len(seeds) > 1 else [])
    for g in groups:
        o, r, c = vf.pool_counts([counts[s] for s in g], p.n_patches)
        t = lap("pool_counts (host arrays to device and back)", t)
        op = exchange.ExchangeOperator(o, r, c, np.full(p.n_patches, cfg["rays"] * len(g), np.int64), area)
        t = lap("ExchangeOperator (host arrays to device, balance)", t)
        chs.append(coupled.prescribed_field_channels(op, p, cfg["T_m"], cfg["dT"], cfg["eps"]))
        op.close()
        t = lap("prescribed_field_channels (binary64)", t)
    return chs


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms while running."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.device_index = device_index
        self.proc = None
        self.lines: list[str] = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.device_index}", f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (FileNotFoundError, OSError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for name, val in zip(names, f[5:9]):
                if val.lower() == "active":
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": smax, "reasons": sorted(reasons), "samples": len(sm)}


def measured_peaks():
    path = ROOT / "MEASURED_PEAKS.json"
    if path.is_file():
        d = json.loads(path.read_text())
        return d, "measured"
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


def fp64_peak_tflops(torch) -> float:
    """Measured binary64 throughput of this GPU: cuBLAS DGEMM 8192^3, best of 5 (CUDA events)."""

    a = torch.randn(8192, 8192, dtype=torch.float64, device="cuda")
    b = torch.randn(8192, 8192, dtype=torch.float64, device="cuda")
    torch.matmul(a, b)
    best = 0.0
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        e1.synchronize()
        best = max(best, 2.0 * 8192**3 / (e0.elapsed_time(e1) * 1e-3) / 1e12)
    del a, b
    torch.cuda.empty_cache()
    return best


class CpuCounts:
    """The oracle (the reference's CPU algorithm) timing first-hit counts of a bounded patch sample.

    The geometry and its patch table are built once.  A sample is ``blocks`` runs of consecutive
    origin patches spread evenly over all patches, traced for every ray set with all host cores
    (NumPy PCG64 rays, the OpenMP C traversal, np.unique per block as the reference does per chunk).
    """

    def __init__(self, cfg, seeds, blocks: int = 16):
        from oracle import build as ob
        from oracle import porerad_oracle as orc

        ob.build()
        self.orc = orc
        self.cores = orc.set_threads()
        self.cfg, self.seeds, self.blocks = cfg, seeds, blocks
        self.patches = orc.build_surface_patches(make_phases(cfg), cfg["H"])
        self.width = 64

    def run(self, width: int):
        P, R = self.patches.n_patches, self.cfg["rays"]
        width = max(1, min(int(width), P // self.blocks))
        starts = [int(b * P // self.blocks) for b in range(self.blocks)]
        t0 = time.perf_counter()
        for s in self.seeds:
            for p0 in starts:
                self.orc.first_hit_counts(self.patches, R, s, patch_start=p0, patch_end=p0 + width)
        dt = time.perf_counter() - t0
        return len(self.seeds) * self.blocks * width * R, dt, width

    def calibrate(self, target_s: float):
        rays, dt, w = self.run(self.width)
        self.width = max(1, int(w * target_s / max(dt, 1e-3)))
        return self.width

    def describe(self, width: int, dt: float) -> str:
        P = self.patches.n_patches
        return (f"first-hit counts (NumPy PCG64 rays + OpenMP C traversal + np.unique) of {self.blocks} blocks of "
                f"{width} consecutive origin patches spread evenly over {P} x {self.cfg['rays']} rays x "
                f"{len(self.seeds)} sets ({self.blocks * width} patches, {dt:.1f} s); patch table built "
                f"outside the timed sample")


def cpu_sample(cfg, seeds, target_s: float):
    """One timed sample of about ``target_s`` seconds; the cpu_baseline object of a bench line."""

    cc = CpuCounts(cfg, seeds)
    cc.calibrate(min(2.0, target_s / 4))
    rays, dt, width = cc.run(cc.calibrate(target_s))
    return {"value": rays / dt, "unit": "rays/s", "cores": cc.cores, "kind": "port",
            "sample": cc.describe(width, dt)}


def counts_step(phases, cfg, seeds, host_out=False):
    """The count stage of one case: patch table, then per ray set fused generation + traversal + count rows.

    ``phases`` is a device tensor (``host_out`` False: count tables stay in HBM) or pinned host
    memory (``host_out`` True: the reference-facing calls ``build_surface_patches`` and
    ``first_hit_counts``, whose (origin, receiver, count) arrays are copied to host NumPy).
    """

    from porerad_b200 import view_factors as vf

    p = vf.build_surface_patches(phases, cfg["H"])
    P = p.n_patches
    out = {"rays": 0, "steps": 0, "pairs": [], "d2h": 0, "n_patches": P}
    for s in seeds:
        if host_out:
            o, r, c = vf.first_hit_counts(p, cfg["rays"], s)
            out["pairs"].append(int(o.size))
            out["d2h"] += o.nbytes + r.nbytes + c.nbytes
            out["rays"] += P * cfg["rays"]
            del o, r, c
        else:
            t = vf.first_hit_counts_pooled(p, cfg["rays"], [s])
            out["rays"] += t.rays_traced
            out["steps"] += t.dda_steps
            out["pairs"].append(t.nnz)
            t.close()
    p.device().close()
    # host->device per step: the phases (host form) and 130 PCG64 jump maps of 32 B per seed
    out["h2d"] = 32 * 130 * len(seeds)
    return out


def _timer_values(lib, names):
    """(launches, ms) of the library's CUDA-event timers, by name."""

    from porerad_b200 import _lib

    ids = {"trace": _lib.TIMER_TRACE, "rle": _lib.TIMER_RLE, "balance": _lib.TIMER_BALANCE,
           "series": _lib.TIMER_SERIES, "cheb": _lib.TIMER_CHEB, "refine": _lib.TIMER_REFINE}
    out = {}
    for name in names:
        n, t = _lib.ctypes.c_longlong(), _lib.ctypes.c_double()
        lib.pr_timers_read(ids[name], _lib.ctypes.byref(n), _lib.ctypes.byref(t))
        out[name] = (int(n.value), float(t.value))
    return out


def trace_profile(workload: str):
    """Per-launch figures of the traversal kernel from the committed ncu summary (profiles/), or None."""

    path = ROOT / "profiles" / f"trace_{workload}.md"
    if not path.is_file():
        return None
    vals = {}
    for line in path.read_text().splitlines():
        for key in ("dram_bytes_per_ray", "warp_inst_per_step"):
            if line.startswith(key + ":"):
                vals[key] = float(line.split(":", 1)[1].split()[0])
    return vals if "dram_bytes_per_ray" in vals else None


def bench_config(cfg, seeds):
    """The workload keys both arms print (the reference arm's line carries the same dict)."""

    return {"workload": cfg["workload"], "archetype": cfg["arch"], "N": cfg["n"], "phi": cfg["phi"],
            "geometry_seed": cfg["seed"], "rays_per_patch": cfg["rays"], "ray_sets": len(seeds),
            "step": "first-hit counts of every ray set (ray generation, first-hit traversal, per-origin "
                    "(receiver, count) rows); GPU steps also build the patch table",
            "parallelism": "replicas", "l2": "256 MiB flush write before every timed GPU step; count tables > L2"}


def whole_case(args, cfg, seeds, phases_dev, phases_host, pinned, lib, flush, rank):
    """cases/s of the whole case (patches, counts, 3 balanced operators, 3 mixed-precision solves)."""

    import torch

    from porerad_b200 import replicas

    k = max(1, min(args.steps, 10))
    for _ in range(max(1, args.warmup)):  # the library's memory cache holds the count stage's blocks
        release(served_step(phases_dev, cfg, seeds))
    torch.cuda.synchronize()
    lib.pr_timers_reset()
    lib.pr_timers_enable(1)
    replicas.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    last = None
    for _ in range(k):
        flush.fill_(1)
        last = served_step(phases_dev, cfg, seeds)
        release(last)
    e1.record()
    torch.cuda.synchronize()
    lib.pr_timers_enable(0)
    ms = e0.elapsed_time(e1)
    timers = _timer_values(lib, ("balance", "series", "cheb", "refine"))
    t0 = time.perf_counter()
    for _ in range(k):
        res = served_step(pinned.numpy(), cfg, seeds)
        release(res)
    torch.cuda.synchronize()
    e2e_s = time.perf_counter() - t0
    ms, e2e_s = replicas.max_over_ranks([ms, e2e_s])
    if rank != 0:
        return None
    # one operator at a time: the products of each operator alone, for a per-launch rate that no
    # other stream's work inflates
    solo = served_step(phases_dev, cfg, seeds, serial=True, timers=True)
    solo_timers = solo.pop("_timers")
    release(solo)
    res64 = served_step(phases_dev, cfg, seeds, precision="fp64")
    resm = served_step(phases_dev, cfg, seeds, precision="mixed")
    f64, fm = res64["final"], resm["final"]
    flux_err = max(abs(fm.q_h - f64.q_h) / abs(f64.q_h), abs(fm.q_c - f64.q_c) / abs(f64.q_c))
    ab = None
    if len(seeds) > 1:
        from porerad_b200 import coupled

        ab = coupled.ab_differences([resm["sets"][0]], [resm["sets"][1]])
    release(res64)
    release(resm)
    plain = None
    if not args.no_plain:
        plain_step(phases_host, cfg, seeds)
        torch.cuda.synchronize()
        stages = {}
        t0 = time.perf_counter()
        plain_step(phases_host, cfg, seeds, stages=stages)
        torch.cuda.synchronize()
        plain_s = time.perf_counter() - t0
        plain = {"cases_per_s": 1.0 / plain_s, "s_per_case": plain_s, "stages_s": stages,
                 "path": "drop-in NumPy API: build_surface_patches, first_hit_counts per set, pool_counts, "
                         "ExchangeOperator from host arrays, binary64 prescribed_field_channels"}
    peaks, kind = measured_peaks()
    P = last["n_patches"]

    def spmv_rates(tm, prods):
        nnz_avg = sum(z * c for z, c in prods) / max(sum(c for _, c in prods), 1)
        out = {}
        for name in ("balance", "series", "cheb", "refine"):
            n_k, t_k = tm[name]
            if n_k == 0:
                continue
            # packed 4-byte words per entry, row offsets, and the P-vectors each kernel streams
            bytes_per = nnz_avg * 4 + P * (8 + 5 * (8 if name != "cheb" else 4))
            out[name] = {"launches": n_k, "ms": t_k, "GB_per_s": bytes_per * n_k / (t_k * 1e-3) / 1e9,
                         "frac": bytes_per * n_k / (t_k * 1e-3) / 1e9 / peaks["hbm_gbs"]}
        tot_b = sum(v["GB_per_s"] * v["ms"] for v in out.values())
        tot_t = sum(v["ms"] for v in out.values())
        return out, (tot_b / tot_t if tot_t else None), tot_t, nnz_avg

    kern, ach, tot_t, nnz_avg = spmv_rates(timers, last["products"])
    kern_solo, ach_solo, _, _ = spmv_rates(solo_timers, solo["products"])
    roof_spmv = {"bound": "hbm", "achieved": ach_solo, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                 "frac": ach_solo / peaks["hbm_gbs"] if ach_solo else None,
                 "peak_source": f"MEASURED_PEAKS.json ({kind})", "kernels": kern_solo,
                 "timing": "one operator at a time (the three operators of one case built and solved in turn)",
                 "overlapped": {"achieved": ach, "kernels": kern, "share_of_step": tot_t / (ms / k),
                                "note": "the three operators on three streams at once, as in the timed case: "
                                        "a launch's event time includes the other streams' work (lower bound)"},
                 "bytes": "4 B per packed S' entry + P x (8 + 5 x 8) B (f32 sweep: 5 x 4 B)",
                 "nnz_symmetric_per_product": round(nnz_avg)}
    return {
        "cases_per_s": args.gpus * k / (ms * 1e-3), "ms_per_case": ms / k, "steps": k,
        "e2e_cases_per_s": args.gpus * k / e2e_s,
        "work": "patches, counts A+B, pooled A+B, 3 balanced operators, 3 mixed-precision channel solves",
        "plain": plain, "served_over_plain": (args.gpus * k / e2e_s) / plain["cases_per_s"] if plain else None,
        "mixed_vs_fp64_rel_flux_error": flux_err,
        "mixed_vs_fp64_reference": "the device binary64 series on the same operator (pinned to the oracle's "
                                   "binary64 series at 1e-9 by the parity tests)",
        "ab_differences": {"wall_channel": ab[0], "coarse_source": ab[1]} if ab else None,
        "q": {"q_h": f64.q_h, "q_c": f64.q_c, "q_i": f64.q_i},
        "balance": {"method": last["balance"][0], "iterations": last["balance"][1],
                    "row_sum_error": last["balance"][2]},
        "nnz_symmetric": last["nnz_symmetric"], "pairs_pooled": last["nnz"],
        "roofline_spmv": roof_spmv,
    }


def run_ours(args, cfg):
    import torch

    from porerad_b200 import _lib, replicas

    world, rank, local = replicas.world_size(), replicas.rank(), replicas.local_rank()
    if world != args.gpus:
        raise SystemExit(f"--gpus {args.gpus} but WORLD_SIZE={world}")
    torch.cuda.set_device(local)
    replicas.init("nccl")
    lib = _lib.load()
    seeds = ray_seeds(cfg)
    phases_host = make_phases(cfg)
    phases_dev = torch.from_numpy(phases_host).cuda()
    pinned = torch.from_numpy(phases_host).pin_memory()
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device="cuda")

    for _ in range(args.warmup):
        counts_step(phases_dev, cfg, seeds)
    counts_step(pinned.numpy(), cfg, seeds, host_out=True)
    torch.cuda.synchronize()

    # ---- timed region: device-resident inputs, count tables left in HBM
    lib.pr_timers_reset()
    lib.pr_timers_enable(1)
    launches0 = lib.pr_kernel_launches()
    rays = steps = 0
    last = None
    replicas.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clocks:
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(args.steps):
            flush.fill_(1)  # 256 MiB write: L2 (126 MB) holds nothing of the previous step
            last = counts_step(phases_dev, cfg, seeds)
            rays += last["rays"]
            steps += last["steps"]
        e1.record()
        torch.cuda.synchronize()
    replicas.barrier()
    launches = lib.pr_kernel_launches() - launches0
    lib.pr_timers_enable(0)
    ms = e0.elapsed_time(e1)
    timers = _timer_values(lib, ("trace", "rle"))

    # ---- end to end through the reference-facing API from pinned host memory, host arrays out
    replicas.barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    e2e_rays = 0
    for _ in range(args.steps):
        flush.fill_(1)
        res = counts_step(pinned.numpy(), cfg, seeds, host_out=True)
        e2e_rays += res["rays"]
    torch.cuda.synchronize()
    e2e_s = time.perf_counter() - t0
    h2d = int(phases_host.nbytes) + int(res["h2d"])
    d2h = int(res["d2h"])

    t_max, e2e_s = replicas.max_over_ranks([ms, e2e_s])
    # every replica traced the same seeded case: DDA steps and pairs per set agree on all ranks
    agree = replicas.all_equal([steps, *last["pairs"]])
    value = rays * world / (t_max * 1e-3)
    case = whole_case(args, cfg, seeds, phases_dev, phases_host, pinned, lib, flush, rank)
    line = None
    if rank == 0:
        fp64 = fp64_peak_tflops(torch)
        n_tr, t_tr = timers["trace"]
        flops = 4.0 * steps + 30.0 * rays
        achieved = flops / (t_tr * 1e-3) / 1e12 if t_tr > 0 else None
        prof = trace_profile(args.workload)
        roof = {"kernel": "k_trace_pool (fused PCG64 ray generation + FP64 DDA, pooled lanes)", "bound": "fp64",
                "achieved": achieved, "peak": fp64, "unit": "TFLOP/s",
                "frac": achieved / fp64 if achieved else None,
                "traffic": prof["dram_bytes_per_ray"] * rays / max(n_tr, 1) if prof else None,
                "launches": n_tr, "ms": t_tr,
                "work": "4 FP64 ops per DDA step + 30 per ray (generation/setup); steps counted by the kernel",
                "peak_source": "cuBLAS DGEMM 8192^3 measured in this run",
                "share_of_step": t_tr / ms}
        if prof and "warp_inst_per_step" in prof and t_tr > 0:
            # the bound that binds: warp instructions issued per second against one per cycle on each of
            # the 4 schedulers of the 148 SMs (instructions per DDA step include the rays' generation)
            inst = prof["warp_inst_per_step"] * steps
            clk = (clocks.summary().get("sm_mhz") or 1965.0) * 1e6
            peak_issue = 4 * 148 * clk
            roof["issue"] = {"achieved_warp_inst_per_s": inst / (t_tr * 1e-3), "peak": peak_issue,
                             "frac": inst / (t_tr * 1e-3) / peak_issue,
                             "warp_inst_per_step": prof["warp_inst_per_step"],
                             "source": f"profiles/trace_{args.workload}.md (ncu smsp__inst_executed.sum / "
                                       "DDA steps of the captured launch)"}
        cpu = None if args.no_cpu else cpu_sample(cfg, seeds, args.cpu_seconds)
        pairs = last["pairs"]
        line = {
            "metric": "first-hit rays/s",
            "value": value, "unit": "rays/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": t_max / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": bench_config(cfg, seeds),
            "case": {"n_patches": last["n_patches"], "pairs_per_set": pairs, "rays_per_step": rays / args.steps,
                     "dda_steps_per_ray": steps / rays},
            "timing": "value: CUDA events on the launching stream around the K steps (each step: 256 MiB L2 "
                      "flush, patch table, counts of every set); e2e: wall clock around the same K steps through "
                      "build_surface_patches + first_hit_counts from pinned host phases, NumPy arrays out",
            "e2e": {"value": e2e_rays * world / e2e_s, "unit": "rays/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h,
                    "d2h": "origin i32 + receiver i32 + count i64 per pair of every set (the reference's arrays)"},
            "roofline": roof, "trace_variant": _lib.trace_variant()[1],
            "stage_ms_per_step": {"traversal": timers["trace"][1] / args.steps,
                                  "per_origin_rows": timers["rle"][1] / args.steps,
                                  "other": t_max / args.steps - (timers["trace"][1] + timers["rle"][1]) / args.steps,
                                  "note": "device time of the traversal and row kernels from CUDA events; other = "
                                          "the rest of the step (patch table, CSR assembly, flush, host gaps)"},
            "clocks": clocks.summary(), "gpu_launches": int(launches), "cpu_baseline": cpu,
            "whole_case": case,
        }
        if world > 1:
            line["replicas_agree"] = agree
        if case is not None:
            line["cases_per_s"] = case["cases_per_s"]
    replicas.finalize()
    return line


# --------------------------------------------------------------------------- serving (c4)

def c4_specs(cfg):
    """The request stream: (archetype, N, phi, geometry seed, axis, eps, T_mean, rays) per request."""

    from porerad_b200.geometry import ARCHETYPES

    rng = np.random.default_rng(cfg["stream_seed"])
    out = []
    for _ in range(cfg["requests"]):
        out.append(dict(arch=str(rng.choice(ARCHETYPES)), n=int(rng.choice([96, 128, 160, 192])),
                        phi=float(rng.uniform(0.05, 0.20)), seed=int(rng.integers(0, 100)),
                        axis=str(rng.choice(["x", "y", "z"])), eps=float(rng.uniform(0.3, 0.95)),
                        T_mean=float(rng.uniform(500.0, 900.0)), rays=int(rng.integers(250, 1001))))
    return out


def _c4_geometry(spec):
    from porerad_b200 import geometry

    ph = geometry.make(spec["arch"], spec["n"], spec["phi"], spec["seed"])
    return np.ascontiguousarray(np.moveaxis(ph, "xyz".index(spec["axis"]), 0))


def plain_case(req, stages=None):
    """One request through the drop-in NumPy API (the reference driver's sequence, binary64 series);
    ``stages`` (a dict) receives the wall-clock seconds of each stage."""

    from porerad_b200 import coupled, exchange, view_factors as vf

    st = stages if stages is not None else {}

    def lap(name, t0):
        st[name] = st.get(name, 0.0) + time.perf_counter() - t0
        return time.perf_counter()

    t = time.perf_counter()
    p = vf.build_surface_patches(req.phases, req.H_m)
    t = lap("patches", t)
    tables = [vf.first_hit_counts(p, req.rays_per_patch, s) for s in req.seeds]
    t = lap("first_hit_counts", t)
    o, r, c = vf.pool_counts(tables, p.n_patches)
    t = lap("pool_counts", t)
    op = exchange.ExchangeOperator(o, r, c, np.full(p.n_patches, req.rays_per_patch * len(req.seeds), np.int64),
                                   p.patch_area_m2)
    t = lap("ExchangeOperator", t)
    ch = coupled.prescribed_field_channels(op, p, req.T_mean_K, req.delta_T_K, req.epsilon)
    op.close()
    lap("prescribed_field_channels", t)
    return ch


def _replay(arrivals, submit):
    """Submit request k at t0 + arrivals[k] (real time); returns t0."""

    t0 = time.perf_counter()
    for k, a in enumerate(arrivals):
        delay = t0 + a - time.perf_counter()
        if delay > 0:
            time.sleep(delay)
        submit(k, t0 + a)
    return t0


def run_c4(args, cfg):
    import torch

    from porerad_b200 import _lib, geometry, serving
    from porerad_b200.geometry import ray_set_seed

    torch.cuda.set_device(0)
    lib = _lib.load()
    specs = c4_specs(cfg)

    def request(k, sp, phases=None):
        geo = phases if phases is not None else serving.GeometrySpec(sp["arch"], sp["n"], sp["phi"], sp["seed"],
                                                                     sp["axis"])
        return serving.CaseRequest(geo, cfg["H"], sp["rays"], [ray_set_seed(sp["seed"] * 131 + k, 0)],
                                   sp["T_mean"], 100.0, sp["eps"], precision="mixed", tag=k)

    reqs = [request(k, sp) for k, sp in enumerate(specs)]
    with serving.Server(slots=cfg["slots"]) as srv:  # warm-up: pools, autotuning of the first classes
        [f.result() for f in [srv.submit(r) for r in reqs[:8]]]

    # ---- saturated: every request at t0
    launches0 = lib.pr_kernel_launches()
    with ClockSampler(0) as clocks:
        t0 = time.perf_counter()
        with serving.Server(slots=cfg["slots"]) as srv:
            sat = [f.result() for f in [srv.submit(r, t_submit=t0) for r in reqs]]
        t_sat = time.perf_counter() - t0
        peak_reserved = srv.admission.peak
    launches = lib.pr_kernel_launches() - launches0
    served_rate = len(reqs) / t_sat
    rays = sum(r.rays for r in sat)

    # ---- Poisson arrivals at 0.8 x the saturated served rate, all requests, replayed in real time
    rng = np.random.default_rng(cfg["stream_seed"] + 1)
    lam = 0.8 * served_rate
    arr = np.cumsum(rng.exponential(1.0 / lam, size=len(reqs)))
    arr -= arr[0]
    with serving.Server(slots=cfg["slots"]) as srv:
        futs = []
        _replay(arr, lambda k, ts: futs.append(srv.submit(reqs[k], t_submit=ts)))
        pois = [f.result() for f in futs]
    lat = [r.latency_s for r in pois]
    same = all((a.q_h, a.q_c, a.q_i) == (b.q_h, b.q_c, b.q_i) for a, b in zip(pois, sat))

    # ---- the plain per-case path on the first requests: host phases made before the clock starts,
    # one FIFO server (each request runs to completion before the next), real-time arrivals
    m = min(cfg["plain_requests"], len(specs))
    host = []
    for sp in specs[:m]:
        ph = geometry.make_device(sp["arch"], sp["n"], sp["phi"], sp["seed"])
        host.append(np.ascontiguousarray(np.moveaxis(ph.cpu().numpy(), "xyz".index(sp["axis"]), 0)))
    plain_reqs = [request(k, sp, host[k]) for k, sp in enumerate(specs[:m])]
    plain_case(plain_reqs[0])
    stages, service = {}, []
    for r in plain_reqs[:3]:
        t = time.perf_counter()
        plain_case(r, stages)
        service.append(time.perf_counter() - t)
    plain_rate = len(service) / sum(service)
    lam_p = 0.8 * plain_rate
    arr_p = np.cumsum(np.random.default_rng(cfg["stream_seed"] + 2).exponential(1.0 / lam_p, size=m))
    arr_p -= arr_p[0]
    plain_done = []
    t0 = time.perf_counter()
    for k, a in enumerate(arr_p):
        delay = t0 + a - time.perf_counter()
        if delay > 0:
            time.sleep(delay)
        plain_case(plain_reqs[k], stages)
        plain_done.append(time.perf_counter() - t0 - a)
    plain_wall = time.perf_counter() - t0
    # the served system under the same arrivals of the same requests
    with serving.Server(slots=cfg["slots"]) as srv:
        futs = []
        _replay(arr_p, lambda k, ts: futs.append(srv.submit(reqs[k], t_submit=ts)))
        served_at_plain = [f.result().latency_s for f in futs]
    n_stage = len(service) + m
    pct = serving.percentile
    return {
        "metric": "served cases/s (continuous batching, mixed precision), saturated request stream",
        "value": served_rate, "unit": "cases/s", "n_gpus": 1, "steps": len(reqs), "warmup": 8,
        "ms_per_step": 1e3 * t_sat / len(reqs), "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64 (traversal), f32+f64 (radiosity)", "data": "synthetic",
        "config": {"workload": cfg["workload"], "requests": len(reqs), "slots": cfg["slots"],
                   "stream_seed": cfg["stream_seed"], "hbm_peak_reserved_GB": peak_reserved / 1e9,
                   "geometry": "requests carry generator specs; each worker generates its geometry on the device"},
        "rays_per_s_served": rays / t_sat,
        "saturated_latency_s": {"p50": pct([r.latency_s for r in sat], 50),
                                "p99": pct([r.latency_s for r in sat], 99)},
        "poisson": {"rate_per_s": lam, "requests": len(reqs), "served_p50_s": pct(lat, 50),
                    "served_p99_s": pct(lat, 99), "results_equal_to_saturated_run": same},
        "plain": {"cases_per_s": plain_rate, "service_s_first3": service, "requests": m,
                  "stages_s_per_case": {k: v / n_stage for k, v in stages.items()},
                  "poisson_rate_per_s": lam_p, "p50_s": pct(plain_done, 50), "p95_s": pct(plain_done, 95),
                  "max_s": max(plain_done), "wall_s": plain_wall,
                  "latency": "measured: one FIFO worker running the drop-in NumPy path on real-time arrivals"},
        "served_at_plain_rate": {"p50_s": pct(served_at_plain, 50), "p95_s": pct(served_at_plain, 95),
                                 "max_s": max(served_at_plain)},
        "served_over_plain": served_rate / plain_rate,
        "clocks": clocks.summary(), "gpu_launches": int(launches),
    }


# --------------------------------------------------------------------------- batched sweep (c3)

def c3_specs(cfg):
    from porerad_b200.geometry import ARCHETYPES

    rng = np.random.default_rng(cfg["pick_seed"])
    out = []
    for arch in ARCHETYPES:
        for phi in cfg["phis"]:
            for seed in range(cfg["seeds"]):
                out.append(dict(arch=arch, n=cfg["n"], phi=phi, seed=seed, axis=str(rng.choice(["x", "y", "z"])),
                                eps=float(rng.choice([0.3, 0.6, 0.9]))))
    return out


def run_c3(args, cfg):
    import concurrent.futures
    import multiprocessing

    specs = c3_specs(cfg)
    with multiprocessing.get_context("spawn").Pool(min(8, os.cpu_count() or 1)) as pool:
        phases = pool.map(_c4_geometry, specs)
    import torch

    from porerad_b200 import _lib, coupled, exchange, view_factors as vf
    from porerad_b200.geometry import ray_set_seed

    torch.cuda.set_device(0)
    lib = _lib.load()
    dev_phases = [torch.from_numpy(ph).cuda() for ph in phases]
    seeds = [[ray_set_seed(1000 + k, 0)] for k in range(len(specs))]
    R, H = cfg["rays"], cfg["H"]
    streams = [torch.cuda.Stream() for _ in range(cfg["slots"])]

    def solve(k, geo, op):
        with _lib.use_stream(streams[k % len(streams)]):
            p = vf.SurfacePatches(H_m=H, _device=geo)
            if not isinstance(op, exchange.ExchangeOperator):  # a count table: the operator built here alone
                table = op
                op = exchange.ExchangeOperator(table, None, None, np.full(geo.n_patches, R, np.int64),
                                               np.full(geo.n_patches, (H / cfg["n"]) ** 2))
                table.close()
            ch = coupled.prescribed_field_channels(op, p, cfg["T_m"], cfg["dT"], specs[k]["eps"], precision="mixed")
            op.close()
            return ch

    stage_s = {}

    def lap(name, t0):
        torch.cuda.synchronize()
        stage_s[name] = time.perf_counter() - t0
        return time.perf_counter()

    def sweep(batched=True):
        stage_s.clear()
        t = time.perf_counter()
        geos = [vf.DeviceGeometry(ph, H) for ph in dev_phases]
        pats = [vf.SurfacePatches(H_m=H, _device=g) for g in geos]
        tables = vf.first_hit_counts_batch(pats, R, seeds)
        t = lap("patches_and_counts", t)
        if batched:
            # the operators of all cases, their balancing iterations in shared product launches
            ops = exchange.ExchangeOperator.from_tables(
                tables, [np.full(g.n_patches, R, np.int64) for g in geos],
                [np.full(g.n_patches, (H / cfg["n"]) ** 2) for g in geos])
            for tb in tables:
                tb.close()
            t = lap("operators", t)
        else:
            ops = tables  # each operator built alone by its solve's worker (4 streams)
        with concurrent.futures.ThreadPoolExecutor(cfg["slots"]) as ex:
            chs = list(ex.map(lambda a: solve(*a), [(k, g, o) for k, (g, o) in enumerate(zip(geos, ops))]))
        lap("solves" if batched else "operators_and_solves", t)
        rays = sum(g.n_patches for g in geos) * R
        patches = [g.n_patches for g in geos]
        for g in geos:
            g.close()
        return rays, chs, patches

    sweep()  # warm-ups of both modes (autotuning, memory pools)
    sweep(batched=False)
    timed = {}
    for batched in (True, False):
        lib.pr_timers_reset()
        lib.pr_timers_enable(1)
        launches0 = lib.pr_kernel_launches()
        with ClockSampler(0) as clocks:
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            rays, chs, patches = sweep(batched)
            dt = time.perf_counter() - t0
        lib.pr_timers_enable(0)
        n, ms = _lib.ctypes.c_longlong(), _lib.ctypes.c_double()
        lib.pr_timers_read(_lib.TIMER_TRACE, _lib.ctypes.byref(n), _lib.ctypes.byref(ms))
        timed[batched] = dict(dt=dt, chs=chs, stages=dict(stage_s), clocks=clocks.summary(), trace_n=int(n.value),
                              trace_ms=ms.value, launches=int(lib.pr_kernel_launches() - launches0))
    # bitwise the same channels either way (operators built together equal operators built alone)
    same = all(a.q_h == b.q_h and a.q_c == b.q_c and a.q_i == b.q_i for a, b in zip(timed[True]["chs"], timed[False]["chs"]))
    best = min(timed, key=lambda k: timed[k]["dt"])
    other = not best
    mode = {True: "all operators balanced together (one product launch per iteration for every operator), "
                  "then the mixed-precision solves on 4 streams",
            False: "each case's operator built and solved by one of 4 worker threads on its own stream"}
    w = timed[best]
    dt, chs, clocks = w["dt"], w["chs"], w["clocks"]
    return {
        "metric": "first-hit rays/s and cases/s of the 48-case batched sweep (one count pass, overlapped solves)",
        "value": rays / dt, "unit": "rays/s", "n_gpus": 1, "steps": 1, "warmup": 2, "ms_per_step": dt * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64 (traversal), f32+f64 (radiosity)", "data": "synthetic",
        "config": {"workload": cfg["workload"], "cases": len(specs), "patches_min": min(patches),
                   "patches_max": max(patches), "rays": rays, "operators": mode[best]},
        "cases_per_s": len(specs) / dt, "stages_s": w["stages"],
        "other_mode": {"operators": mode[other], "s": timed[other]["dt"],
                       "cases_per_s": len(specs) / timed[other]["dt"], "stages_s": timed[other]["stages"]},
        "modes_bitwise_equal": bool(same),
        "trace_launches": w["trace_n"],
        "trace_ms": w["trace_ms"],
        "trace_launches": int(n.value),
        "trace_ms": ms.value,
        "trace_variant": _lib.trace_variant()[1], "max_closure_rel": max(c.closure_rel for c in chs),
        "clocks": clocks, "gpu_launches": w["launches"],
    }


# --------------------------------------------------------------------------- coupled solve

def _coupled_case(case_id):
    golden = ROOT / "tests" / "golden"
    row = next(r for r in json.loads((golden / "coupled.json").read_text())["rows"] if r["case_id"] == case_id)
    with np.load(golden / f"canonical_{row['microstructure']}.npz") as z:
        ph = np.unpackbits(z["bits"])[: int(np.prod(z["shape"]))].reshape(tuple(z["shape"])).astype(np.uint8)
    ph = np.moveaxis(ph, "xyz".index(row["axis"]), 0)
    ph = np.ascontiguousarray(np.concatenate([ph] * row["repeats"], axis=0))
    return row, ph


def coupled_step(row, ph):
    """One archived coupled case from its phases: the run_coupled.py sequence on the device."""

    import torch

    from porerad_b200 import conduction, coupled, exchange, view_factors as vf
    from porerad_b200.constants import K_GAS, K_SOLID

    H = row["H_m"]
    Th, Tc = row["T_mean_K"] + row["delta_T_K"] / 2.0, row["T_mean_K"] - row["delta_T_K"] / 2.0
    marks = [time.perf_counter()]
    p = vf.build_surface_patches(ph, H)
    seeds = row["seeds_A"] + row["seeds_B"]
    table = vf.first_hit_counts_pooled(p, row["rays_per_patch"], seeds)
    torch.cuda.synchronize()
    marks.append(time.perf_counter())
    n = p.n_patches
    op = exchange.ExchangeOperator(table, None, None, np.full(n, row["rays_per_patch"] * len(seeds), np.int64),
                                   np.full(n, (H / ph.shape[0]) ** 2))
    marks.append(time.perf_counter())
    system = conduction.assemble_conduction(np.where(ph == 1, K_SOLID, K_GAS), H)
    T0 = conduction.solve_conduction(system, Th, Tc)
    marks.append(time.perf_counter())
    res = coupled.solve_coupled(system, op, p, Th, Tc, row["epsilon"], T0)
    m = coupled.wall_flux_metrics(system, p, res, Th, Tc)
    marks.append(time.perf_counter())
    out = dict(metrics=m, newton=res.newton_iterations, gmres=[s["gmres_iterations"] for s in res.linear_solves],
               failures=coupled.acceptance_failures(res, m), n_patches=n, nnz=op.nnz_symmetric,
               phases_ms={k: 1e3 * (marks[i + 1] - marks[i]) for i, k in
                          enumerate(("patches_counts", "operator", "conduction", "newton_krylov"))})
    op.close()
    table.close()
    system.close()
    return out


def run_coupled_bench(args, cfg):
    import torch

    from porerad_b200 import _lib

    torch.cuda.set_device(0)
    lib = _lib.load()
    row, ph = _coupled_case(cfg["case_id"])
    for _ in range(max(args.warmup, 1)):
        coupled_step(row, ph)
    torch.cuda.synchronize()
    launches0 = lib.pr_kernel_launches()
    outs = []
    with ClockSampler(0) as clocks:
        t0 = time.perf_counter()
        for _ in range(args.steps):
            outs.append(coupled_step(row, ph))
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
    last = outs[-1]
    m = last["metrics"]
    rel = {k: abs(m[k] - row[k]) / abs(row[k]) for k in ("q_total_hot_W_m2", "q_rad_hot_W_m2", "k_eff_apparent_W_mK")}
    cpu = None
    if not args.no_cpu:
        cpu = coupled_cpu_sample(row, ph)
    return {
        "metric": "strictly coupled solves/s (whole archived case from its phases)", "value": args.steps / dt,
        "unit": "cases/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * dt / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "reference fixture",
        "config": {"workload": cfg["workload"], "n_patches": last["n_patches"], "nnz_symmetric": last["nnz"],
                   "cells": int(ph.size)},
        "phases_ms": last["phases_ms"], "newton_updates": last["newton"], "gmres_iterations": last["gmres"],
        "acceptance_failures": last["failures"], "rel_error_vs_archived": rel,
        "archived_newton_updates": row["newton_updates"], "clocks": clocks.summary(),
        "gpu_launches": int(lib.pr_kernel_launches() - launches0) // max(args.steps, 1), "cpu_baseline": cpu,
    }


def coupled_cpu_sample(row, ph):
    """The oracle (NumPy/SciPy restatement of run_coupled.py's path) on the same case, timed on the host cores."""

    from oracle import build as ob
    from oracle import porerad_oracle as orc

    ob.build()
    cores = orc.set_threads()
    H = row["H_m"]
    Th, Tc = row["T_mean_K"] + row["delta_T_K"] / 2.0, row["T_mean_K"] - row["delta_T_K"] / 2.0
    t0 = time.perf_counter()
    p = orc.build_surface_patches(ph, H)
    seeds = row["seeds_A"] + row["seeds_B"]
    o, r, c = orc.pool_counts([orc.first_hit_counts(p, row["rays_per_patch"], s) for s in seeds], p.n_patches)
    op = orc.ExchangeOperator(o, r, c, np.full(p.n_patches, row["rays_per_patch"] * len(seeds), np.int64),
                              p.patch_area_m2)
    system = orc.assemble_conduction(np.where(ph == 1, orc.K_SOLID, orc.K_GAS), H)
    T0 = orc.solve_conduction(system, Th, Tc)
    orc.solve_coupled(system, op, p, Th, Tc, row["epsilon"], T0)
    dt = time.perf_counter() - t0
    return {"value": 1.0 / dt, "unit": "cases/s", "cores": cores, "kind": "port",
            "sample": f"the whole case once on the CPU ({dt:.1f} s): oracle patches, counts (OpenMP C traversal), "
                      "SciPy-Anderson operator, SciPy CG conduction, NumPy/SciPy Newton-Krylov"}


# --------------------------------------------------------------------------- coupled-size stress (c5)

def run_c5(args, cfg):
    import torch

    from porerad_b200 import _lib, coupled, exchange, geometry, view_factors as vf
    from porerad_b200.geometry import ray_set_seed

    torch.cuda.set_device(0)
    lib = _lib.load()
    n = cfg["n"]
    base = coupled.linear_cell_temperature((n, n, n), cfg["T_m"], cfg["dT"])
    rng = np.random.default_rng(2)
    fields = [torch.from_numpy(base + rng.normal(0.0, cfg["sigma_K"], base.shape)).cuda() for _ in range(cfg["solves"])]
    Th, Tc = cfg["T_m"] + cfg["dT"] / 2.0, cfg["T_m"] - cfg["dT"] / 2.0
    # warm-up on a small case
    w = vf.build_surface_patches(geometry.make("FA", 48, cfg["phi"], 0), cfg["H"])
    t = vf.first_hit_counts_pooled(w, 64, [1])
    wo = exchange.ExchangeOperator(t, None, None, np.full(w.n_patches, 64, np.int64), w.patch_area_m2)
    coupled.cell_field_channels(wo, w, base[:48, :48, :48].copy(), Th, Tc, cfg["eps"], precision="mixed")
    wo.close(); t.close()
    out = {}
    total_rays, total_ms = 0, 0.0
    launches0 = lib.pr_kernel_launches()
    with ClockSampler(0) as clocks:
        for arch in cfg["archs"]:
            phases = torch.from_numpy(geometry.make(arch, n, cfg["phi"], cfg["seed"])).cuda()
            seeds = [ray_set_seed(cfg["seed"] + 7919 * (arch == "FA"), k) for k in range(cfg["sets"])]
            torch.cuda.synchronize()
            e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
            e0.record()
            geo = vf.DeviceGeometry(phases, cfg["H"])
            p = vf.SurfacePatches(H_m=cfg["H"], _device=geo)
            tables = [vf.first_hit_counts_pooled(p, cfg["rays"], [s]) for s in seeds]
            rays = sum(tb.rays_traced for tb in tables)
            pooled = tables[0]
            for tb in tables[1:]:
                merged = pooled.merge(tb)
                pooled.close()
                tb.close()
                pooled = merged
            op = exchange.ExchangeOperator(pooled, None, None, np.full(geo.n_patches, cfg["rays"] * cfg["sets"],
                                                                       np.int64),
                                           np.full(geo.n_patches, (cfg["H"] / n) ** 2))
            e1.record()
            mixed = [coupled.cell_field_channels(op, p, f, Th, Tc, cfg["eps"], reference_temperature_K=cfg["T_m"],
                                                 precision="mixed") for f in fields]
            e2.record()
            torch.cuda.synchronize()
            build_ms, solve_ms = e0.elapsed_time(e1), e1.elapsed_time(e2)
            fp64 = [coupled.cell_field_channels(op, p, f, Th, Tc, cfg["eps"], reference_temperature_K=cfg["T_m"])
                    for f in fields]
            errs = [max(abs(m.q_h - d.q_h) / abs(d.q_h), abs(m.q_c - d.q_c) / abs(d.q_c)) for m, d in zip(mixed, fp64)]
            out[arch] = {"n_patches": geo.n_patches, "rays": rays, "pairs_pooled": pooled.nnz,
                         "nnz_symmetric": op.nnz_symmetric, "build_ms": build_ms,
                         "solve_ms_each": solve_ms / len(fields), "balance": [op.balance_method, op.balance_iterations],
                         "mixed_vs_fp64_rel_flux_error_max": max(errs), "per_solve_error": errs,
                         "q_first": [fp64[0].q_h, fp64[0].q_c, fp64[0].q_i]}
            total_rays += rays
            total_ms += build_ms + solve_ms
            op.close()
            pooled.close()
            geo.close()
            del phases
    return {
        "metric": "first-hit rays/s (N=192 stress: build + 20 resident-operator solves per geometry)",
        "value": total_rays / (total_ms * 1e-3), "unit": "rays/s", "n_gpus": 1, "steps": len(cfg["archs"]),
        "warmup": 1, "ms_per_step": total_ms / len(cfg["archs"]), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64 (traversal), f32+f64 (radiosity)", "data": "synthetic",
        "config": {"workload": cfg["workload"]}, "cases": out, "clocks": clocks.summary(),
        "gpu_launches": int(lib.pr_kernel_launches() - launches0),
    }


# --------------------------------------------------------------------------- reference arm

# --------------------------------------------------------------------------- morphology descriptors

def _stored_microstructures():
    golden = ROOT / "tests" / "golden"
    out = []
    for path in sorted(golden.glob("canonical_*.npz")):
        with np.load(path) as z:
            shape = tuple(int(v) for v in z["shape"])
            out.append((path.name[len("canonical_"):-4],
                        np.unpackbits(z["bits"])[: int(np.prod(shape))].reshape(shape).astype(np.uint8)))
    return out


def _descriptor_cpu_one(ph):
    from oracle import morphology as om

    return om.scalar_descriptors(ph), om.directional_descriptors(ph)


def descriptors_cpu_sample(arrays, target_s: float):
    """The oracle (NumPy/SciPy restatement of porerad.descriptors, scipy.ndimage.label for the clusters) on
    the stored microstructures, one per process on every host core, until about target_s seconds of work."""

    import multiprocessing as mp

    cores = os.cpu_count() or 1
    t0 = time.perf_counter()
    done = 0
    with mp.get_context("spawn").Pool(cores) as pool:
        pool.map(_descriptor_cpu_one, [arrays[0]])  # start-up of the workers, untimed
        t0 = time.perf_counter()
        while True:
            batch = [arrays[(done + i) % len(arrays)] for i in range(max(cores, len(arrays)))]
            pool.map(_descriptor_cpu_one, batch, chunksize=1)
            done += len(batch)
            if time.perf_counter() - t0 >= target_s:
                break
    dt = time.perf_counter() - t0
    return {"value": done / dt, "unit": "microstructures/s", "cores": cores, "kind": "port",
            "sample": f"{done} descriptor evaluations of the stored 128^3 microstructures in {dt:.1f} s "
                      f"(scalar + directional, oracle, {cores} spawn workers)"}


def run_descriptors_bench(args, cfg):
    import torch

    from porerad_b200 import _lib, descriptors as dm

    torch.cuda.set_device(0)
    lib = _lib.load()
    named = _stored_microstructures()
    host = [ph for _, ph in named]
    dev = [torch.from_numpy(ph).cuda() for ph in host]
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")  # 256 MB > L2
    peaks, kind = measured_peaks()
    cells = sum(int(ph.size) for ph in host)

    def step(arrays):  # the microstructures at once on worker streams
        return dm.all_descriptors_many(arrays)

    for _ in range(max(args.warmup, 3)):
        step(dev)
    torch.cuda.synchronize()
    lib.pr_timers_reset()
    lib.pr_timers_enable(1)
    launches0 = lib.pr_kernel_launches()
    total_ms = 0.0
    with ClockSampler(0) as clocks:
        for _ in range(args.steps):
            flush.fill_(1)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record()
            out = step(dev)
            e1.record()
            torch.cuda.synchronize()
            total_ms += e0.elapsed_time(e1)
    lib.pr_timers_enable(0)
    launches = lib.pr_kernel_launches() - launches0
    timers = {}
    for name, tid in (("morph", _lib.TIMER_MORPH), ("label", _lib.TIMER_LABEL)):
        n, t = _lib.ctypes.c_longlong(), _lib.ctypes.c_double()
        lib.pr_timers_read(tid, _lib.ctypes.byref(n), _lib.ctypes.byref(t))
        timers[name] = (int(n.value), float(t.value))
    value = args.steps * len(dev) / (total_ms * 1e-3)

    # end to end from host arrays (pageable numpy, as a user passes them)
    e2e_ms = 0.0
    for _ in range(args.steps):
        flush.fill_(1)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        step(host)
        torch.cuda.synchronize()
        e2e_ms += 1e3 * (time.perf_counter() - t0)
    e2e = args.steps * len(host) / (e2e_ms * 1e-3)

    # roofline of the counts pass: one byte read per cell (the neighbours come from cache)
    n_m, t_m = timers["morph"]
    per_launch_bytes = cells / len(dev)
    achieved = per_launch_bytes / (t_m / n_m * 1e-3) / 1e9 if n_m else None
    n_l, t_l = timers["label"]
    cpu = None if args.no_cpu else descriptors_cpu_sample(host, args.cpu_seconds)
    check = out[0][0]
    return {
        "metric": "morphology descriptors (scalar + directional) per second", "value": value,
        "unit": "microstructures/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": total_ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "u8", "data": "reference microstructures (tests/golden)",
        "config": {"workload": cfg["workload"], "microstructures": len(dev), "cells": cells,
                   "l2": "flushed (256 MB write) before each step, outside the timed region"},
        "e2e": {"value": e2e, "unit": "microstructures/s", "h2d_bytes_per_step": cells,
                "d2h_bytes_per_step": int(sum(8 * (18 + sum(n + 1 for n in ph.shape)) for ph in host))},
        "roofline": {"bound": "hbm", "kernel": "k_morph_counts", "achieved": achieved, "peak": peaks["hbm_gbs"],
                     "unit": "GB/s", "frac": achieved / peaks["hbm_gbs"] if achieved else None,
                     "peak_source": f"MEASURED_PEAKS.json ({kind})", "traffic": None,
                     "bytes_per_launch": per_launch_bytes, "ms_per_launch": t_m / n_m if n_m else None},
        "kernel_ms_per_microstructure": {"morph_counts": t_m / max(n_m, 1), "labelling": t_l / max(n_l, 1)},
        "clocks": clocks.summary(), "gpu_launches": int(launches) // max(args.steps, 1), "cpu_baseline": cpu,
        "first_result": {"phi_solid": check["phi_solid"], "mean_beam_length": check["mean_beam_length"]},
    }


# --------------------------------------------------------------------------- microstructure generators

def _generator_cpu_one(job):
    from oracle import generators as og
    from oracle import morphology as om

    structure, phi, seed = job
    ph = og.build(structure, 128, phi, seed)
    om.scalar_descriptors(ph)
    return int(ph.sum())


def generators_cpu_sample(target_s: float):
    """The oracle (NumPy/SciPy restatement of porerad.geometry, the reference's CPU algorithm) building
    and describing core-library arrays, one per process on every host core, until about target_s
    seconds of work: the 16 trials at phi 0.10 (4 seeds per structure) per round."""

    import multiprocessing as mp

    cores = os.cpu_count() or 1
    jobs = [(s, 0.10, k) for s in ("OF", "FI", "FA", "TL") for k in range(4)]
    done = 0
    with mp.get_context("spawn").Pool(min(cores, len(jobs))) as pool:
        pool.map(_generator_cpu_one, [("TL", 0.10, 0)])  # worker start-up, untimed
        t0 = time.perf_counter()
        while True:
            pool.map(_generator_cpu_one, jobs, chunksize=1)
            done += len(jobs)
            if time.perf_counter() - t0 >= target_s:
                break
    dt = time.perf_counter() - t0
    return {"value": done / dt, "unit": "microstructures/s", "cores": min(cores, len(jobs)), "kind": "port",
            "sample": f"{done} core-library trials at phi 0.10 (4 seeds x OF/FI/FA/TL, build + scalar "
                      f"descriptors) in {dt:.1f} s on {min(cores, len(jobs))} spawn workers"}


def run_generators_bench(args, cfg):
    import torch

    from porerad_b200 import _lib, generators as gen

    torch.cuda.set_device(0)
    lib = _lib.load()

    def step(device=True):  # the 12 cells at once (gen.core_library), TL's host fields overlapping
        return [x for cell in gen.core_library(device=device).values() for x in cell]

    for _ in range(max(args.warmup, 3)):
        step()
    torch.cuda.synchronize()
    lib.pr_timers_reset()
    lib.pr_timers_enable(1)
    launches0 = lib.pr_kernel_launches()
    total_ms = 0.0
    with ClockSampler(0) as clocks:
        for _ in range(args.steps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record()
            out = step()
            e1.record()
            torch.cuda.synchronize()
            total_ms += e0.elapsed_time(e1)
    lib.pr_timers_enable(0)
    launches = lib.pr_kernel_launches() - launches0
    n_r, t_r = _lib.ctypes.c_longlong(), _lib.ctypes.c_double()
    lib.pr_timers_read(_lib.TIMER_RENDER, _lib.ctypes.byref(n_r), _lib.ctypes.byref(t_r))
    value = args.steps * len(out) / (total_ms * 1e-3)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        host = step(device=False)
    e2e = args.steps * len(host) / (time.perf_counter() - t0)
    ms_render = t_r.value / max(n_r.value, 1)
    achieved = 128 ** 3 / (ms_render * 1e-3) / 1e9 if n_r.value else None
    peaks, kind = measured_peaks()
    cpu = None if args.no_cpu else generators_cpu_sample(args.cpu_seconds)
    return {
        "metric": "core-library microstructures per second (generation + acceptance)", "value": value,
        "unit": "microstructures/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": total_ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64 (shape tests), u8", "data": "the reference's generators (seeded)",
        "config": {"workload": cfg["workload"], "accepted": len(out),
                   "l2": "every trial writes a fresh 2 MiB array; outputs stay resident"},
        "e2e": {"value": e2e, "unit": "microstructures/s",
                "h2d_bytes_per_step": int(12 * 8 * 128 ** 3),  # TL's normal draws, one N^3 f64 array per TL trial
                "d2h_bytes_per_step": int(len(host) * 128 ** 3)},
        "roofline": {"bound": "hbm", "kernel": "k_render_shapes / k_stamp", "achieved": achieved,
                     "peak": peaks["hbm_gbs"], "unit": "GB/s", "frac": achieved / peaks["hbm_gbs"] if achieved else None,
                     "peak_source": f"MEASURED_PEAKS.json ({kind})", "traffic": None,
                     "note": "algorithmic bytes = the 2 MiB array written per rendering; the shape tests are "
                             "FP64 compute, so this fraction is low by construction"},
        "renders_per_step": int(n_r.value) // max(args.steps, 1), "ms_per_render": ms_render,
        "clocks": clocks.summary(), "gpu_launches": int(launches) // max(args.steps, 1), "cpu_baseline": cpu,
    }


# --------------------------------------------------------------------------- multi-bounce statistics

def _multibounce_jobs():
    from tests.helpers import multibounce_rows

    rows = multibounce_rows()
    jobs = []
    for kind in ("properties", "penetration"):
        for r in rows[kind]:
            jobs.append((kind, r["microstructure"], r["transfer_axis"], float(r["epsilon"])))
    return jobs


def _solid_x(name, axis):
    from tests.helpers import load_canonical

    ph = load_canonical(name)
    return np.ascontiguousarray(np.moveaxis(ph == 1, "xyz".index(axis), 0)).astype(np.uint8)


_MB_SEEDS = {"properties": ((123, 456), 200_000), "penetration": ((321, 654), 500_000)}


def _multibounce_cpu_one(job):
    from oracle import multibounce as om

    kind, name, axis, eps = job
    seeds, n = _MB_SEEDS[kind]
    solid = _solid_x(name, axis)
    for s in seeds:
        om.run(solid, eps, n, s, penetration=kind == "penetration")
    return len(seeds) * n


def multibounce_cpu_sample(target_s: float):
    """The oracle (C restatement of the reference's ray kernels, OpenMP over rays on every host core)
    on identifications of the archived set in order until about target_s seconds."""

    jobs = _multibounce_jobs()
    rays, done = 0, 0
    t0 = time.perf_counter()
    while time.perf_counter() - t0 < target_s and done < len(jobs):
        rays += _multibounce_cpu_one(jobs[(done * 37) % len(jobs)])  # a spread over structures and kinds
        done += 1
    dt = time.perf_counter() - t0
    return {"value": rays / dt, "unit": "rays/s", "cores": os.cpu_count() or 1, "kind": "port",
            "sample": f"{done} identifications ({rays} source rays) of the archived set in {dt:.1f} s, "
                      "oracle/multibounce.c with OpenMP"}


def run_properties_bench(args, cfg):
    import torch

    from porerad_b200 import _lib, penetration, properties

    torch.cuda.set_device(0)
    lib = _lib.load()
    jobs = _multibounce_jobs()
    geos = {}
    for kind, name, axis, eps in jobs:
        if (name, axis) not in geos:
            geos[(name, axis)] = properties._geometry(np.asarray(load_phases(name)), axis)
    rays_per_step = sum(len(_MB_SEEDS[k][0]) * _MB_SEEDS[k][1] for k, *_ in jobs)

    def step(resident=True):
        if resident:  # every run of the set at once, RUN_STREAMS in flight
            calls = []
            for kind, name, axis, eps in jobs:
                seeds, n = _MB_SEEDS[kind]
                fn = properties.trace_properties if kind == "properties" else penetration.trace_penetration
                calls += [(fn, (None, axis, eps), dict(n_rays=n, seed=s, _geo=geos[(name, axis)])) for s in seeds]
            return properties.run_concurrently(calls)
        out = []
        for kind, name, axis, eps in jobs:
            if kind == "properties":
                out.append(properties.identify_properties(load_phases(name), axis, eps))
            else:
                out.append(penetration.penetration_response(load_phases(name), axis, eps))
        return out

    for _ in range(max(args.warmup, 3)):
        step()
    torch.cuda.synchronize()
    launches0 = lib.pr_kernel_launches()
    total_ms = 0.0
    with ClockSampler(0) as clocks:
        for _ in range(args.steps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record()
            step()
            e1.record()
            torch.cuda.synchronize()
            total_ms += e0.elapsed_time(e1)
    launches = lib.pr_kernel_launches() - launches0
    value = args.steps * rays_per_step / (total_ms * 1e-3)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        step(resident=False)
    e2e = args.steps * rays_per_step / (time.perf_counter() - t0)
    for g in geos.values():
        g.close()
    cpu = None if args.no_cpu else multibounce_cpu_sample(args.cpu_seconds)
    return {
        "metric": "multi-bounce source rays per second (archived identification set)", "value": value,
        "unit": "rays/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": total_ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "reference microstructures (tests/golden)",
        "config": {"workload": cfg["workload"], "identifications": len(jobs), "rays_per_step": rays_per_step,
                   "l2": "the 12 solid grids (2 MiB each) stay resident; rays carry no memory traffic"},
        "e2e": {"value": e2e, "unit": "rays/s", "h2d_bytes_per_step": int(len(jobs) * 128 ** 3),
                "d2h_bytes_per_step": int(len(jobs) * 2 * 64)},
        "roofline": None,
        "roofline_note": "one thread follows one ray through cell steps and reflections: issue- and "
                         "divergence-bound integer/FP64 control work with no bandwidth or tensor bound",
        "clocks": clocks.summary(), "gpu_launches": int(launches) // max(args.steps, 1), "cpu_baseline": cpu,
    }


def load_phases(name):
    from tests.helpers import load_canonical

    return load_canonical(name)


# --------------------------------------------------------------------------- archetype generation

_ARCH_CASES = [(a, n) for n in (128, 192) for a in ("OF", "FI", "FA", "TL")]


def archetypes_cpu_sample(target_s: float):
    """The host definitions (geometry.make, NumPy/SciPy) of the same archetypes, one per process on
    every host core, until about target_s seconds."""

    import multiprocessing as mp

    cores = os.cpu_count() or 1
    done = 0
    with mp.get_context("spawn").Pool(min(cores, len(_ARCH_CASES))) as pool:
        pool.starmap(_arch_host_one, [("TL", 32)])  # worker start-up, untimed
        t0 = time.perf_counter()
        while True:
            pool.starmap(_arch_host_one, _ARCH_CASES, chunksize=1)
            done += len(_ARCH_CASES)
            if time.perf_counter() - t0 >= target_s:
                break
    dt = time.perf_counter() - t0
    return {"value": done / dt, "unit": "microstructures/s", "cores": min(cores, len(_ARCH_CASES)), "kind": "port",
            "sample": f"{done} host generations (OF/FI/FA/TL x N 128, 192) in {dt:.1f} s"}


def _arch_host_one(arch, n):
    from porerad_b200 import geometry

    return int(geometry.make(arch, n, 0.10, 1).sum())


def run_archetypes_bench(args, cfg):
    import torch

    from porerad_b200 import _lib, geometry

    torch.cuda.set_device(0)
    lib = _lib.load()
    for _ in range(max(args.warmup, 3)):
        for a, n in _ARCH_CASES:
            geometry.make_device(a, n, 0.10, 1)
    torch.cuda.synchronize()
    per = {}
    launches0 = lib.pr_kernel_launches()
    with ClockSampler(0) as clocks:
        total_ms = 0.0
        for _ in range(args.steps):
            for a, n in _ARCH_CASES:
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                torch.cuda.synchronize()
                e0.record()
                geometry.make_device(a, n, 0.10, 1)
                e1.record()
                torch.cuda.synchronize()
                ms = e0.elapsed_time(e1)
                total_ms += ms
                per.setdefault(f"{a}{n}", []).append(ms)
    launches = lib.pr_kernel_launches() - launches0
    t0 = time.perf_counter()
    for _ in range(args.steps):
        for a, n in _ARCH_CASES:
            geometry.make_device(a, n, 0.10, 1).cpu()
    e2e = args.steps * len(_ARCH_CASES) / (time.perf_counter() - t0)
    cpu = None if args.no_cpu else archetypes_cpu_sample(args.cpu_seconds)
    return {
        "metric": "benchmark archetypes generated per second (device, bit-identical to the host definition)",
        "value": args.steps * len(_ARCH_CASES) / (total_ms * 1e-3), "unit": "microstructures/s", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64 (fields), u8", "data": "synthetic (seeded)",
        "config": {"workload": cfg["workload"], "l2": "each generation writes fresh arrays of 2-7 MiB"},
        "ms_per_generation": {k: float(np.median(v)) for k, v in per.items()},
        "e2e": {"value": e2e, "unit": "microstructures/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": int(sum(n ** 3 for _, n in _ARCH_CASES))},
        "roofline": None, "clocks": clocks.summary(), "gpu_launches": int(launches) // max(args.steps, 1),
        "cpu_baseline": cpu,
    }


def run_reference(args, cfg):
    from porerad_b200 import replicas

    if replicas.rank() != 0:
        return None  # the CPU reference runs once, on rank 0
    if args.workload == "archetypes":
        vals, last = [], None
        for _ in range(args.steps):
            last = archetypes_cpu_sample(max(1.0, args.cpu_seconds / 2))
            vals.append(last["value"])
        value = float(np.mean(vals))
        return {"impl": "reference", "metric": "benchmark archetypes generated per second (device, bit-identical to "
                                               "the host definition)",
                "value": value, "unit": "microstructures/s", "n_gpus": args.gpus, "steps": args.steps, "warmup": 0,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64 (fields), u8",
                "data": "synthetic (seeded)", "config": {"workload": cfg["workload"]},
                "cpu_baseline": {**last, "value": value},
                "e2e": {"value": value, "unit": "microstructures/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    if args.workload == "properties":
        vals, last = [], None
        for _ in range(args.steps):
            last = multibounce_cpu_sample(max(1.0, args.cpu_seconds / 2))
            vals.append(last["value"])
        value = float(np.mean(vals))
        return {"impl": "reference", "metric": "multi-bounce source rays per second (archived identification set)",
                "value": value, "unit": "rays/s", "n_gpus": args.gpus, "steps": args.steps, "warmup": 0,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "reference microstructures (tests/golden)", "config": {"workload": cfg["workload"]},
                "cpu_baseline": {**last, "value": value},
                "e2e": {"value": value, "unit": "rays/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    if args.workload == "generators":
        vals, last = [], None
        for _ in range(args.steps):
            last = generators_cpu_sample(max(1.0, args.cpu_seconds / 2))
            vals.append(last["value"])
        value = float(np.mean(vals))
        return {"impl": "reference", "metric": "core-library microstructures per second (generation + acceptance)",
                "value": value, "unit": "microstructures/s", "n_gpus": args.gpus, "steps": args.steps, "warmup": 0,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64 (shape tests), u8",
                "data": "the reference's generators (seeded)", "config": {"workload": cfg["workload"]},
                "cpu_baseline": {**last, "value": value},
                "e2e": {"value": value, "unit": "microstructures/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    if args.workload == "descriptors":
        arrays = [ph for _, ph in _stored_microstructures()]
        vals, last = [], None
        for _ in range(args.steps):
            last = descriptors_cpu_sample(arrays, max(1.0, args.cpu_seconds / 2))
            vals.append(last["value"])
        value = float(np.mean(vals))
        return {"impl": "reference", "metric": "morphology descriptors (scalar + directional) per second",
                "value": value, "unit": "microstructures/s", "n_gpus": args.gpus, "steps": args.steps, "warmup": 0,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u8",
                "data": "reference microstructures (tests/golden)", "config": {"workload": cfg["workload"]},
                "cpu_baseline": {**last, "value": value},
                "e2e": {"value": value, "unit": "microstructures/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    if "case_id" in cfg:  # the coupled workload: the whole case on the host cores
        row, ph = _coupled_case(cfg["case_id"])
        vals, last = [], None
        for _ in range(args.steps):
            last = coupled_cpu_sample(row, ph)
            vals.append(last["value"])
        value = float(np.mean(vals))
        return {"impl": "reference", "metric": "strictly coupled solves/s (whole archived case from its phases)",
                "value": value, "unit": "cases/s", "n_gpus": args.gpus, "steps": args.steps, "warmup": 0,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "reference fixture", "config": {"workload": cfg["workload"]},
                "cpu_baseline": {**last, "value": value},
                "e2e": {"value": value, "unit": "cases/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    if "arch" not in cfg:
        raise SystemExit("--impl reference times the CPU path of the c1, c2 and coupled workloads")
    seeds = ray_seeds(cfg)
    cc = CpuCounts(cfg, seeds)
    # each step is one bounded sample of the workload (about cpu_seconds / 3 of CPU work); warm-up
    # steps run the calibration and the first samples untimed
    width = cc.calibrate(0.5)
    for _ in range(max(0, args.warmup)):
        width = cc.calibrate(max(0.5, args.cpu_seconds / 3))
    rays = dt = 0.0
    for _ in range(args.steps):
        r, t, width = cc.run(width)
        rays += r
        dt += t
    value = rays / dt
    return {
        "impl": "reference", "metric": "first-hit rays/s", "value": value, "unit": "rays/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * dt / max(args.steps, 1),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": bench_config(cfg, seeds),
        "cpu_baseline": {"value": value, "unit": "rays/s", "cores": cc.cores, "kind": "port",
                         "sample": cc.describe(width, dt / max(args.steps, 1)) + " per step"},
        "e2e": {"value": value, "unit": "rays/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def main():
    args = parse_args()
    cfg = dict(WORKLOADS[args.workload])
    if args.rays is not None and "rays" in cfg:
        cfg["rays"] = int(args.rays)
        cfg["workload"] += f" [rays/patch overridden to {args.rays}: profiling case]"
    if args.impl != "reference" and args.workload not in ("c1", "c2") and int(os.environ.get("WORLD_SIZE", "1")) > 1:
        # one process per GPU with independent replicas is the c1/c2 path; the others time one GPU
        raise SystemExit(f"workload {args.workload} runs on one GPU; launch it without torchrun")
    if args.impl == "reference":
        line = run_reference(args, cfg)
    elif args.workload == "c3":
        line = run_c3(args, cfg)
    elif args.workload == "coupled":
        line = run_coupled_bench(args, cfg)
    elif args.workload == "descriptors":
        line = run_descriptors_bench(args, cfg)
    elif args.workload == "generators":
        line = run_generators_bench(args, cfg)
    elif args.workload == "properties":
        line = run_properties_bench(args, cfg)
    elif args.workload == "archetypes":
        line = run_archetypes_bench(args, cfg)
    elif args.workload == "c4":
        line = run_c4(args, cfg)
    elif args.workload == "c5":
        line = run_c5(args, cfg)
    else:
        line = run_ours(args, cfg)
    if line is not None:
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()

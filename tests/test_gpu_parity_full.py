"""Parity at the full sizes of the benchmark configurations.

* the benchmark SOCP itself (n = 2M, m = 1.5M, nnz(A) = 25M, 5000-row cones,
  2000-nonzero rows): 150 iterates, residuals, M-norm and sigma terms at the
  1e-10 bar with sigma and lambda injected identically, and a full solve to
  1e-6 KKT against the oracle's solve;
* the reduced-precision streams on the same instance: the error of their
  solutions against the oracle's FP64 solution;
* the portfolio QP-SOCP at n = 200k with Q = D + F'F as an operator:
  150 iterates at 1e-10.

The oracle runs on every host thread.  These tests take a few minutes.
"""
import numpy as np
import pytest

from helpers import branch_disagreements, rel_err
from hprsocp_b200 import Context, HPRSOCP_parameters, instances
from oracle_ctx import OracleContext

pytestmark = [pytest.mark.gpu, pytest.mark.slow]

ITER_TOL = 1e-10
VECS = ["x", "x_hat", "x_bar", "z_bar", "y", "y_bar", "s", "dx", "dy"]


@pytest.fixture(scope="module")
def config1():
    return instances.config1(1)


def _inject(o, g, so, lamq=0.0):
    # lambda from the GPU power iteration (fast), the same value on both sides
    lam = 1.05 * g.power_A()
    sigma = so["norm_b"] / so["norm_c"]
    for c in (o, g):
        c.set_sigma_lambda(sigma, lam, lamq)
        c.set_inner(0)


def test_config1_iterates_residuals_at_full_size(config1):
    p = HPRSOCP_parameters(verbose=False)
    with OracleContext(config1, threads=0) as o, Context(config1) as g:
        so = o.scale(p)
        g.scale(p)
        _inject(o, g, so)
        o.iterate(150, True)
        g.iterate(150, True)
        for v in VECS:
            e = rel_err(g.get(v), o.get(v))
            assert e <= ITER_TOL, (v, e)
        assert branch_disagreements(g, o, config1) == (0, 0)
        ro = o.residuals(include_bounds=True)
        rg = g.residuals(include_bounds=True)
        for k, v in ro.items():
            assert abs(rg[k] - v) <= ITER_TOL * max(1.0, abs(v)), (k, rg[k], v)
        mo, mg = o.mnorm(), g.mnorm()
        assert abs(mo - mg) <= ITER_TOL * max(1.0, mo)
        for a, b in zip(o.sigma_terms(), g.sigma_terms()):
            assert abs(a - b) <= ITER_TOL * max(1.0, abs(a))


@pytest.fixture(scope="module")
def config1_oracle_solution(config1):
    p = HPRSOCP_parameters(verbose=False, stoptol=1e-6, max_iter=20000, time_limit=1800)
    with OracleContext(config1, threads=0) as o:
        return o.solve(p)


def _rel(a, b):
    return float(np.max(np.abs(a - b)) / max(1.0, np.max(np.abs(b))))


def test_config1_solve_matches_oracle(config1, config1_oracle_solution):
    ro = config1_oracle_solution
    p = HPRSOCP_parameters(verbose=False, stoptol=1e-6, max_iter=20000, time_limit=1800)
    with Context(config1) as g:
        rg = g.solve(p)
    assert ro.status == rg.status == "OPTIMAL"
    assert rg.residuals <= 1e-6
    assert abs(rg.primal_obj - ro.primal_obj) <= 1e-6 * max(1.0, abs(ro.primal_obj))
    assert abs(rg.iter - ro.iter) <= max(10, ro.iter // 20), (rg.iter, ro.iter)
    print(f"config1 solve: GPU {rg.iter} iterations, oracle {ro.iter}; objective {rg.primal_obj:.10e} vs "
          f"{ro.primal_obj:.10e}; x err {_rel(rg.x, ro.x):.2e}, y err {_rel(rg.y, ro.y):.2e}")


@pytest.mark.parametrize("prec,x_tol,obj_tol", [("fp32", 1e-4, 1e-6), ("bf16", 1e-2, 1e-5)])
def test_reduced_precision_errors_against_oracle(config1, config1_oracle_solution, prec, x_tol, obj_tol):
    """The mixed-precision streams (FP32 values and gathers; BF16 values with
    FP32 products; both with the FP64 finish) reach 1e-6 KKT, and their
    solutions are compared with the oracle's FP64 solution."""
    ro = config1_oracle_solution
    p = HPRSOCP_parameters(verbose=False, stoptol=1e-6, max_iter=40000, time_limit=1800, precision=prec)
    with Context(config1) as g:
        rg = g.solve(p)
    assert rg.status == "OPTIMAL" and rg.residuals <= 1e-6
    ex, ey = _rel(rg.x, ro.x), _rel(rg.y, ro.y)
    eo = abs(rg.primal_obj - ro.primal_obj) / max(1.0, abs(ro.primal_obj))
    print(f"{prec}: x err {ex:.2e}, y err {ey:.2e}, objective err {eo:.2e}, KKT {rg.residuals:.2e} "
          f"(oracle {ro.residuals:.2e}), iterations {rg.iter} (oracle {ro.iter})")
    assert ex <= x_tol and eo <= obj_tol


def test_config2_iterates_at_full_size():
    model = instances.config2(2)
    p = HPRSOCP_parameters(verbose=False)
    with OracleContext(model, threads=0) as o, Context(model) as g:
        so = o.scale(p)
        g.scale(p)
        lamq = 1.05 * g.power_Q()
        _inject(o, g, so, lamq)
        o.iterate(150, True)
        g.iterate(150, True)
        for v in VECS:
            e = rel_err(g.get(v), o.get(v))
            assert e <= ITER_TOL, (v, e)
        assert branch_disagreements(g, o, model) == (0, 0)

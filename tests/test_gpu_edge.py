"""Parity with the oracle on degenerate problem shapes: no cone at all, one
cone holding every variable, no linear row, cones of dimension 1 and 2,
empty rows and columns in A, and no rows at all (m = 0).  Each case runs a
fixed number of iterations from identical scaled data, sigma and lambda
(iterates within 1e-10, the same projection branch in every cone) and a
full solve (same status, objective within 1e-6, iterations within 5%)."""
import numpy as np
import pytest

from helpers import branch_disagreements, edge_model, rel_err
from hprsocp_b200 import Context, HPRSOCP_parameters
from oracle_ctx import OracleContext

pytestmark = pytest.mark.gpu

KINDS = ["lp_box", "one_cone", "cones_only", "dim_one", "sparse", "no_rows"]
VECS = ["x", "x_hat", "x_bar", "z_bar", "y", "y_bar", "s", "dx", "dy"]


@pytest.mark.parametrize("kind", KINDS)
def test_edge_iterates_match_the_oracle(kind):
    model = edge_model(kind)
    o, g = OracleContext(model, threads=0), Context(model)
    p = HPRSOCP_parameters(verbose=False)
    so = o.scale(p)
    g.scale(p)
    lam = o.power_A() * 1.05
    # sigma_0 as the solve sets it: norm_b / norm_c when both are usable
    ok = 1e-16 < so["norm_b"] < 1e16 and 1e-16 < so["norm_c"] < 1e16
    sigma = so["norm_b"] / so["norm_c"] if ok else 1.0
    for c in (o, g):
        c.set_sigma_lambda(sigma, lam, 0.0)
        c.set_inner(0)
        c.iterate(100, True)
    for v in VECS:
        a, b = g.get(v), o.get(v)
        assert a.shape == b.shape, v
        assert rel_err(a, b) <= 1e-10, (kind, v, rel_err(a, b))
    assert branch_disagreements(g, o, model) == (0, 0)


@pytest.mark.parametrize("kind", KINDS)
def test_edge_solve_matches_the_oracle(kind):
    model = edge_model(kind)
    p = HPRSOCP_parameters(verbose=False, stoptol=1e-6, max_iter=200000)
    ro = OracleContext(model, threads=0).solve(p)
    with Context(model) as g:
        rg = g.solve(p)
    assert ro.status == rg.status == "OPTIMAL", (kind, ro.status, rg.status)
    assert abs(rg.primal_obj - ro.primal_obj) <= 1e-6 * max(1.0, abs(ro.primal_obj)), kind
    assert abs(rg.iter - ro.iter) <= max(10, ro.iter // 20), (kind, rg.iter, ro.iter)
    assert rg.residuals <= 1e-6
    assert np.all(np.isfinite(rg.x)) and np.all(np.isfinite(rg.y))

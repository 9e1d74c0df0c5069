"""Iterate-level parity of the CUDA path with the FP64 oracle.

Bar (from the workload definition): FP64 iterates within 1e-10 relative after
a fixed number of iterations with identical sigma and lambda; scaled data
within 1e-13; residuals/M-norm within 1e-10; full solves reach 1e-6 KKT with
the objective within 1e-6 relative of the oracle's.
"""
import numpy as np
import pytest

from helpers import branch_disagreements, rel_err, stress_model, tall_model
from hprsocp_b200 import HPRSOCP_parameters, instances
from oracle_ctx import OracleContext

pytestmark = pytest.mark.gpu

ITER_TOL = 1e-10
SCALE_TOL = 1e-13
VECS = ["x", "x_hat", "x_bar", "z_bar", "y", "y_bar", "s", "dx", "dy"]


@pytest.fixture(scope="module")
def models():
    # small_* fit the single-CTA multi-iteration kernel (a few tiles per side)
    return {"config0": instances.config0(0), "stress": stress_model(5),
            "config1_small": instances.config1(11, scale=0.004),
            "small_noq": instances.small_socp(21, n=300, diag_q=False),
            "small_q": instances.small_socp(22, n=300, diag_q=True),
            # Q = D + F'F applied as an operator (no scaling, as the reference
            # does for operator Q)
            "config2_small": instances.config2(2, scale=0.01),
            "tall": tall_model(3),
            # general sparse Q with off-diagonal entries, scaled with A; the
            # first runs on the multi-CTA engine, the second on the
            # single-CTA kernel
            "qp_csr": instances.qp_csr(4, n=3000),
            "qp_csr_small": instances.qp_csr(6, n=400, density=0.03)}


def _pair(model):
    from hprsocp_b200 import Context
    return OracleContext(model, threads=0), Context(model)


def _setup(o, g, params=None):
    params = params or HPRSOCP_parameters(verbose=False)
    so = o.scale(params)
    sg = g.scale(params)
    lam = o.power_A() * 1.05
    # operator Q (D + F'F) and a non-diagonal CSR Q: lambda_max(Q) by the
    # power iteration, injected identically on both sides; a diagonal CSR Q
    # keeps 0 (its factors use diag(Q))
    general_q = getattr(o.model, "F", None) is not None or not so["Q_is_diag"]
    lamq = o.power_Q() * 1.05 if general_q else 0.0
    sigma = so["norm_b"] / so["norm_c"] if so["norm_c"] > 1e-16 else 1.0
    for c in (o, g):
        c.set_sigma_lambda(sigma, lam, lamq)
        c.set_inner(0)
    return so, sg


@pytest.mark.parametrize("name", ["config0", "stress", "config1_small", "config2_small", "tall"])
def test_scaling_parity(models, name):
    o, g = _pair(models[name])
    so = o.scale(HPRSOCP_parameters(verbose=False))
    sg = g.scale(HPRSOCP_parameters(verbose=False))
    for k in ("b_scale", "c_scale", "norm_b", "norm_c", "norm_b_org", "norm_c_org"):
        assert abs(so[k] - sg[k]) <= SCALE_TOL * max(1.0, abs(so[k])), (k, so[k], sg[k])
    assert so["Q_is_diag"] == sg["Q_is_diag"]
    for v in ("row_norm", "col_norm", "c", "soc_rhs", "A_values", "AT_values"):
        assert rel_err(g.get(v), o.get(v)) <= SCALE_TOL, v
    for v in ("AL", "AU", "l", "u"):
        a, b = g.get(v), o.get(v)
        assert np.array_equal(np.isinf(a), np.isinf(b)), v
        fin = np.isfinite(b)
        assert rel_err(a[fin], b[fin]) <= SCALE_TOL, v


@pytest.mark.parametrize("name", ["config0", "stress", "config1_small", "small_noq", "small_q", "config2_small",
                                  "tall", "qp_csr", "qp_csr_small"])
@pytest.mark.parametrize("K", [1, 150, 1000])
def test_iterate_parity(models, name, K):
    o, g = _pair(models[name])
    _setup(o, g)
    o.iterate(K, True)
    g.iterate(K, True)
    for v in VECS:
        e = rel_err(g.get(v), o.get(v))
        assert e <= ITER_TOL, (name, K, v, e)
    assert g.scalars()[3] == o.scalars()[3] == K
    # the last (full) iteration took the same projection branch on every cone
    assert branch_disagreements(g, o, models[name]) == (0, 0)


@pytest.mark.parametrize("name", ["config0", "stress", "qp_csr"])
def test_cone_branches_agree_every_iteration(models, name):
    """The harness's cone-branch report: after each of 150 single full
    iterations, the number of cones whose projection branch differs between
    the CUDA path and the oracle (variable cones, constraint cones)."""
    o, g = _pair(models[name])
    _setup(o, g)
    counts = []
    for _ in range(150):
        o.iterate(1, True)
        g.iterate(1, True)
        counts.append(branch_disagreements(g, o, models[name]))
    print(name, "branch disagreements per iteration:", sorted(set(counts)))
    assert all(c == (0, 0) for c in counts), [i for i, c in enumerate(counts) if c != (0, 0)][:10]
    for v in VECS:
        assert rel_err(g.get(v), o.get(v)) <= ITER_TOL, v


def test_single_iteration_agrees_to_rounding(models):
    """A row that lies inside one lane's run of a tile is summed in the
    reference's order (bit for bit); a row that spans runs adds its run
    partials in a fixed order.  From identical scaled data, one iteration
    therefore agrees with the oracle to rounding level (1e-14), far inside
    the 1e-10 iterate bar, and some entries match bit for bit."""
    o, g = _pair(models["config0"])
    _setup(o, g)
    # identical scaled data (b_scale/c_scale are reductions whose last bit
    # depends on summation order)
    for v in ("c", "AL", "AU", "l", "u", "soc_rhs", "A_values", "AT_values"):
        g.set(v, o.get(v))
    o.iterate(1, True)
    g.iterate(1, True)
    same = 0
    for v in VECS:
        a, b = g.get(v), o.get(v)
        assert rel_err(a, b) <= 1e-14, (v, rel_err(a, b))
        same += int(np.sum(a == b))
    assert same > 0


@pytest.mark.parametrize("name", ["config0", "stress", "tall", "config2_small", "qp_csr"])
def test_residual_mnorm_sigma_parity(models, name):
    o, g = _pair(models[name])
    _setup(o, g)
    for c in (o, g):
        c.iterate(149, True)
    ro = o.residuals(include_bounds=True)
    rg = g.residuals(include_bounds=True)
    for k, v in ro.items():
        assert abs(rg[k] - v) <= 1e-10 * max(1.0, abs(v)), (k, rg[k], v)
    mo, mg = o.mnorm(), g.mnorm()
    assert abs(mo - mg) <= 1e-10 * max(1.0, mo)
    to, tg = o.sigma_terms(), g.sigma_terms()
    for a, b in zip(to, tg):
        assert abs(a - b) <= 1e-10 * max(1.0, abs(a))


def test_restart_parity(models):
    o, g = _pair(models["stress"])
    _setup(o, g)
    for c in (o, g):
        c.iterate(150, True)
        c.restart()
        c.iterate(75, True)
    for v in VECS + ["last_x", "last_y"]:
        assert rel_err(g.get(v), o.get(v)) <= ITER_TOL, v


@pytest.mark.parametrize("name", ["stress", "small_noq", "small_q"])
def test_power_iteration_parity(models, name):
    o, g = _pair(models[name])
    p = HPRSOCP_parameters(verbose=False)
    o.scale(p)
    g.scale(p)
    lo, lg = o.power_A(), g.power_A()
    assert abs(lo - lg) <= 1e-6 * lo


@pytest.mark.parametrize("name", ["qp_csr", "config2_small"])
def test_power_iteration_q_parity(models, name):
    """lambda_max(Q) of a non-diagonal CSR Q (scaled) and of the D + F'F
    operator (unscaled)."""
    o, g = _pair(models[name])
    p = HPRSOCP_parameters(verbose=False)
    o.scale(p)
    g.scale(p)
    lo, lg = o.power_Q(), g.power_Q()
    assert abs(lo - lg) <= 1e-6 * lo


def test_solve_parity_config0(models):
    p = HPRSOCP_parameters(verbose=False, stoptol=1e-6, max_iter=100000)
    o, g = _pair(models["config0"])
    ro = o.solve(p)
    rg = g.solve(p)
    assert ro.status == rg.status == "OPTIMAL"
    assert rg.residuals <= 1e-6
    assert abs(rg.primal_obj - ro.primal_obj) <= 1e-6 * max(1.0, abs(ro.primal_obj))
    assert abs(rg.iter - ro.iter) <= max(10, ro.iter // 20), (rg.iter, ro.iter)


def test_solve_is_deterministic(models):
    from hprsocp_b200 import Context
    p = HPRSOCP_parameters(verbose=False, stoptol=1e-6, max_iter=3000)
    r1 = Context(models["stress"]).solve(p)
    r2 = Context(models["stress"]).solve(p)
    assert r1.iter == r2.iter
    assert np.array_equal(r1.x, r2.x) and np.array_equal(r1.y, r2.y)


@pytest.mark.parametrize("name", ["small_noq", "small_q", "config2_small", "tall", "qp_csr", "qp_csr_small"])
def test_solve_parity_small(models, name):
    p = HPRSOCP_parameters(verbose=False, stoptol=1e-6, max_iter=100000)
    o, g = _pair(models[name])
    ro = o.solve(p)
    rg = g.solve(p)
    assert ro.status == rg.status == "OPTIMAL"
    assert abs(rg.primal_obj - ro.primal_obj) <= 1e-6 * max(1.0, abs(ro.primal_obj))
    assert abs(rg.iter - ro.iter) <= max(10, ro.iter // 20), (rg.iter, ro.iter)


@pytest.mark.parametrize("name", ["small_noq", "small_q"])
def test_schedules_give_identical_iterates(models, name):
    """The single-CTA multi-iteration kernel and the multi-CTA engine run
    the same per-row arithmetic: 300 iterations (two batches) agree bit for
    bit."""
    from hprsocp_b200 import Context
    res = {}
    for mode in ("engine", "fused", "auto"):
        with Context(models[name]) as g:
            g.set_schedule(mode)
            info = g.scale(HPRSOCP_parameters(verbose=False))
            g.set_sigma_lambda(info["norm_b"] / info["norm_c"], 1.05 * g.power_A(), 0.0)
            g.set_inner(0)
            g.iterate(150, True)
            g.iterate(150, True)
            res[mode] = [g.get(v) for v in VECS]
    for mode in ("fused", "auto"):
        for a, b in zip(res[mode], res["engine"]):
            assert np.array_equal(a, b), mode


def test_warm_start_parity_and_speed(models):
    """initial_x / initial_y (HPRSOCP_parameters, src/structs.jl:208-277):
    the GPU and the oracle take the same warm-started path, and a start at a
    previous solution converges in fewer iterations."""
    model = models["config0"]
    p = HPRSOCP_parameters(verbose=False, stoptol=1e-6, max_iter=100000)
    o, g = _pair(model)
    cold = g.solve(p)
    assert cold.status == "OPTIMAL"
    pw = HPRSOCP_parameters(verbose=False, stoptol=1e-6, max_iter=100000, initial_x=cold.x, initial_y=cold.y)
    o2, g2 = _pair(model)
    rg = g2.solve(pw)
    ro = o2.solve(pw)
    assert rg.status == ro.status == "OPTIMAL"
    assert rg.iter < cold.iter
    assert abs(rg.iter - ro.iter) <= max(10, ro.iter // 20), (rg.iter, ro.iter)
    assert abs(rg.primal_obj - ro.primal_obj) <= 1e-6 * max(1.0, abs(ro.primal_obj))

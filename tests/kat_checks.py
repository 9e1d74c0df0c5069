"""Known-answer checks shared by the oracle (CPU) and the CUDA library (GPU).

Each check takes a context class with the hprsocp_b200.Context interface, so
the same reference test cases (tests/golden/reference_kats.json) pin both the
oracle and the device kernels.
"""
import math

import numpy as np

from helpers import kat_model, load_kats
from hprsocp_b200 import HPRSOCP_parameters

KATS = load_kats()


def run_kat(ctx_cls, name):
    case = KATS["kats"][name]
    model = kat_model(case)
    ctx = ctx_cls(model)
    try:
        ctx.scale(HPRSOCP_parameters(verbose=False))
        ctx.set_sigma_lambda(case.get("sigma", 1.0), case.get("lambda_max_A", 1.0), case.get("lambda_max_Q", 0.0))
        for k, v in case.get("set", {}).items():
            ctx.set(k, np.array(v, dtype=float))
        if "expect" in case:
            ctx.set_inner(0)
            ctx.iterate(1, True)
            for k, v in case["expect"].items():
                np.testing.assert_allclose(ctx.get(k), v, atol=1e-12, err_msg=f"{name}:{k}")
        if "expect_residuals" in case:
            exp = case["expect_residuals"]
            res = ctx.residuals(include_bounds="bounds_violation" in exp)
            for k, v in exp.items():
                key = "err_Rp_org_bar" if k == "bounds_violation" else k
                assert abs(res[key] - v) <= 1e-12, (name, key, res[key], v)
        if case.get("expect_mnorm_finite_nonnegative"):
            mn = ctx.mnorm()
            assert math.isfinite(mn) and mn >= 0.0
    finally:
        ctx.close()


def run_solve_kat(ctx_cls, name):
    case = KATS["solves"][name]
    model = kat_model(case)
    p = HPRSOCP_parameters(verbose=False, stoptol=case["stoptol"], max_iter=case["max_iter"], time_limit=120.0)
    ctx = ctx_cls(model)
    try:
        r = ctx.solve(p)
    finally:
        ctx.close()
    assert r.status == "OPTIMAL", (name, r.status, r.residuals, r.iter)
    x = r.x
    if "expect_x" in case:
        np.testing.assert_allclose(x, case["expect_x"], atol=case["atol"], err_msg=name)
    if "expect_obj" in case:
        assert abs(r.primal_obj - case["expect_obj"]) <= case["atol"], (name, r.primal_obj)
    if "expect_x_norm_le" in case:
        assert np.linalg.norm(x) <= case["expect_x_norm_le"], (name, np.linalg.norm(x))
    if "expect_feas_atol" in case:
        A = model.A.toarray()
        b = np.array(case["rhs"], dtype=float)
        assert np.linalg.norm(A @ x - b) <= case["expect_feas_atol"]
        assert x[0] + 1e-8 >= np.linalg.norm(x[1:])
    return r

"""Reduced-precision SpMV streams (FP32 values and gathers, BF16 values with
FP32 accumulation) with FP64 residuals, restart and sigma logic, and the FP64
finish of the stream.  The error of each result against the FP64 path is
bounded here; the tolerance reached is the solve's own 1e-6 KKT.
"""
import numpy as np
import pytest

from hprsocp_b200 import Context, HPRSOCP_parameters, instances
from helpers import rel_err, stress_model

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def fp64_solutions():
    out = {}
    for name, model in (("config0", instances.config0(0)), ("stress", stress_model(5))):
        with Context(model) as ctx:
            out[name] = (model, ctx.solve(HPRSOCP_parameters(verbose=False, stoptol=1e-6)))
    return out


@pytest.mark.parametrize("name", ["config0", "stress"])
@pytest.mark.parametrize("prec", ["fp32", "bf16"])
def test_reduced_stream_solves_to_tolerance(fp64_solutions, name, prec):
    model, ref = fp64_solutions[name]
    with Context(model) as ctx:
        r = ctx.solve(HPRSOCP_parameters(verbose=False, stoptol=1e-6, precision=prec))
    assert ref.status == "OPTIMAL" and r.status == "OPTIMAL"
    assert r.residuals <= 1e-6
    # both solutions are 1e-6-KKT points: objectives agree to that order; the
    # points themselves only to the conditioning of the optimal face
    assert abs(r.primal_obj - ref.primal_obj) <= 1e-5 * max(1.0, abs(ref.primal_obj))
    assert rel_err(r.x, ref.x) <= 1e-2 and rel_err(r.y, ref.y) <= 1e-2


def test_fp32_stream_without_finish_still_reaches_tolerance(fp64_solutions):
    model, ref = fp64_solutions["config0"]
    with Context(model) as ctx:
        r = ctx.solve(HPRSOCP_parameters(verbose=False, stoptol=1e-6, precision="fp32", refine=-1))
    assert r.status == "OPTIMAL" and r.residuals <= 1e-6
    assert abs(r.primal_obj - ref.primal_obj) <= 1e-5 * max(1.0, abs(ref.primal_obj))


def test_fp32_iterates_track_fp64():
    """150 iterations with identical sigma and lambda: the FP32 stream stays
    within 1e-5 relative of the FP64 iterates (FP32 products, FP64 sums)."""
    model = stress_model(5)
    its = {}
    for prec in ("fp64", "fp32"):
        with Context(model) as ctx:
            info = ctx.scale(HPRSOCP_parameters(verbose=False))
            ctx.set_precision(prec)
            ctx.set_sigma_lambda(info["norm_b"] / info["norm_c"], 1.05 * ctx.power_A(), 0.0)
            ctx.set_inner(0)
            ctx.iterate(150, True)
            its[prec] = {v: ctx.get(v) for v in ("x", "y", "x_bar", "y_bar")}
    for v in its["fp64"]:
        assert rel_err(its["fp32"][v], its["fp64"][v]) <= 1e-5, v


def test_precision_set_before_scaling_uses_scaled_values():
    """The reduced-precision copies are re-packed after scaling, so the order
    of hpr_set_precision and hpr_scale does not matter."""
    model = instances.config0(0)
    res = []
    for first in ("scale", "precision"):
        with Context(model) as ctx:
            if first == "precision":
                ctx.set_precision("fp32")
            info = ctx.scale(HPRSOCP_parameters(verbose=False))
            if first == "scale":
                ctx.set_precision("fp32")
            ctx.set_sigma_lambda(info["norm_b"] / info["norm_c"], 1.05 * ctx.power_A(), 0.0)
            ctx.set_inner(0)
            ctx.iterate(50, True)
            res.append(ctx.get("x"))
    assert np.array_equal(res[0], res[1])

"""hpr_compute_residuals_noalloc: the allocation-free residual entry point
gives the same residuals as hpr_compute_residuals, call after call, and
refuses what its fixed scratch cannot hold.

Collected last on purpose: it must pass alone and after every other test.
"""
import pytest

from hprsocp_b200 import Context, HPRSOCP_parameters, _abi, instances
from helpers import stress_model

pytestmark = pytest.mark.gpu

# Same kernels and the same fixed reduction order as the existing entry
# point, so the results agree to the last bit; the bar leaves room only for
# the division order of the host-side formulas, which is also identical.
TOL = 1e-15


def _model(name):
    if name == "config0":
        return instances.config0(0)
    if name == "stress":
        return stress_model(5)
    return instances.config2(2, scale=0.01)  # Q = D + F'F operator


def _iterated(model, k=150):
    ctx = Context(model)
    info = ctx.scale(HPRSOCP_parameters(verbose=False))
    lam = ctx.power_A() * 1.05 if model.m > 0 else 0.0
    lamq = ctx.power_Q() * 1.05 if (getattr(model, "F", None) is not None or model.Q is not None) else 0.0
    sigma = info["norm_b"] / info["norm_c"] if info["norm_c"] > 1e-16 else 1.0
    ctx.set_sigma_lambda(sigma, lam, lamq)
    ctx.set_inner(0)
    ctx.iterate(k, True)
    return ctx


def _close(a, b):
    return abs(a - b) <= TOL * max(1.0, abs(b))


def _free_device_bytes():
    import torch
    return torch.cuda.mem_get_info()[0]


@pytest.mark.parametrize("name", ["config0", "stress", "config2_small"])
@pytest.mark.parametrize("bounds", [False, True])
def test_matches_existing_entry_point_on_two_calls(name, bounds):
    with _iterated(_model(name)) as ctx:
        ref = ctx.residuals(include_bounds=bounds)
        # the promise itself: the context allocates nothing more and the
        # device's free memory does not move across the two calls
        _free_device_bytes()  # torch's CUDA state is set up before the measurement
        mem0, free0 = ctx.device_memory(), _free_device_bytes()
        first = ctx.residuals_noalloc(include_bounds=bounds)
        second = ctx.residuals_noalloc(include_bounds=bounds)
        assert ctx.device_memory() == mem0
        assert _free_device_bytes() == free0
        again = ctx.residuals(include_bounds=bounds)
    for k, v in ref.items():
        assert _close(first[k], v), (k, first[k], v)
        assert _close(second[k], v), (k, second[k], v)
        assert again[k] == v, k


def test_problem_beyond_the_static_scratch_is_refused():
    model = instances.config1(1)  # ~36k tiles per side > 32,765 slots
    with Context(model) as ctx:
        ctx.scale(HPRSOCP_parameters(verbose=False))
        with pytest.raises(_abi.HPRError, match="static scratch holds 2097152") as e:
            ctx.residuals_noalloc()
        assert e.value.code == _abi.HPR_E_UNSUPPORTED
        ctx.residuals()  # the allocating entry point still serves it


def test_reduced_precision_stream_is_refused():
    with _iterated(_model("config0"), k=10) as ctx:
        ctx.set_precision("fp32")
        with pytest.raises(_abi.HPRError, match="FP64 stream") as e:
            ctx.residuals_noalloc()
        assert e.value.code == _abi.HPR_E_UNSUPPORTED

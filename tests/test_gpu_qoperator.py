"""A caller's Q operator through the C ABI (hpr_set_q_operator), the
counterpart of a user AbstractQOperator of the reference
(src/Q_operators/Q_operator_interface.jl:32-151).

The callback here is an ordinary user operator: it computes Q v = D v + F'(F v)
with torch on the stream the library hands it, from zero-copy views of the
library's device vectors.  The oracle applies the same Q as its diagonal +
low-rank operator.  An operator Q turns scaling off on both sides, as in the
reference (src/utils/scaling.jl:800-846).
"""
import ctypes as C
import dataclasses

import numpy as np
import pytest

from helpers import rel_err
from hprsocp_b200 import Context, HPRSOCP_parameters, _abi, instances
from oracle_ctx import OracleContext

pytestmark = pytest.mark.gpu

VECS = ["x", "x_hat", "x_bar", "z_bar", "y", "y_bar", "s", "dx", "dy"]
APPLY = C.CFUNCTYPE(None, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p)


class _DeviceVector:
    """A device vector of the library seen by torch without a copy."""

    def __init__(self, ptr, n):
        self.__cuda_array_interface__ = {"shape": (int(n),), "typestr": "<f8", "data": (int(ptr), False),
                                         "version": 3, "strides": None}


def _operator(model):
    import torch
    D = torch.tensor(model.q_diag, dtype=torch.float64, device="cuda")
    F = torch.tensor(model.F.toarray(), dtype=torch.float64, device="cuda")
    calls = [0]

    def apply(user, vin, vout, n, stream):
        with torch.cuda.stream(torch.cuda.ExternalStream(int(stream))):
            v = torch.as_tensor(_DeviceVector(vin, n), device="cuda")
            o = torch.as_tensor(_DeviceVector(vout, n), device="cuda")
            o.copy_(D * v + F.t() @ (F @ v))
        calls[0] += 1

    return APPLY(apply), calls


@pytest.fixture(scope="module")
def model():
    return instances.config2(2, scale=0.01)


def _with_operator(model, lam_q=0.0):
    plain = dataclasses.replace(model, F=None, q_diag=None, Q=None, AT=None)
    g = Context(plain)
    cb, calls = _operator(model)
    g._keep_cb = cb
    rc = g.lib.hpr_set_q_operator(g.h, C.cast(cb, C.c_void_p), None, lam_q)
    assert rc == _abi.HPR_OK, g.lib.hpr_last_error(g.h)
    return g, calls


def test_operator_iterates_match_the_oracle(model):
    o = OracleContext(model, threads=0)
    g, calls = _with_operator(model)
    p = HPRSOCP_parameters(verbose=False)
    so = o.scale(p)
    sg = g.scale(p)
    assert sg["b_scale"] == sg["c_scale"] == 1.0  # no scaling with an operator Q
    lam = 1.05 * o.power_A()
    lamq = 1.05 * o.power_Q()
    assert abs(g.power_Q() - o.power_Q()) <= 1e-6 * o.power_Q()
    sigma = so["norm_b"] / so["norm_c"]
    for c in (o, g):
        c.set_sigma_lambda(sigma, lam, lamq)
        c.set_inner(0)
        c.iterate(150, True)
    for v in VECS:
        e = rel_err(g.get(v), o.get(v))
        assert e <= 1e-10, (v, e)
    assert calls[0] >= 300  # Q w and Q w_bar every iteration
    ro, rg = o.residuals(), g.residuals()
    for k, v in ro.items():
        assert abs(rg[k] - v) <= 1e-10 * max(1.0, abs(v)), (k, rg[k], v)


def test_operator_solve_matches_the_oracle(model):
    p = HPRSOCP_parameters(verbose=False, stoptol=1e-6, max_iter=100000)
    ro = OracleContext(model, threads=0).solve(p)
    g, _ = _with_operator(model)
    rg = g.solve(p)
    assert ro.status == rg.status == "OPTIMAL"
    assert abs(rg.primal_obj - ro.primal_obj) <= 1e-6 * max(1.0, abs(ro.primal_obj))
    assert abs(rg.iter - ro.iter) <= max(10, ro.iter // 20), (rg.iter, ro.iter)


def test_operator_refusals(model):
    g, _ = _with_operator(model)
    # a second problem with an explicit Q cannot take an operator
    qp = Context(instances.qp_csr(6, n=400, density=0.03))
    cb, _ = _operator(model)
    assert qp.lib.hpr_set_q_operator(qp.h, C.cast(cb, C.c_void_p), None, 0.0) == _abi.HPR_E_STATE
    assert g.lib.hpr_set_q_operator(g.h, None, None, 0.0) == _abi.HPR_E_BAD_INPUT
    # once scaled, the operator can no longer change the scaling decision
    g.scale(HPRSOCP_parameters(verbose=False))
    assert g.lib.hpr_set_q_operator(g.h, C.cast(g._keep_cb, C.c_void_p), None, 0.0) == _abi.HPR_E_STATE

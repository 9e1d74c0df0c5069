"""Error statuses that are reached from the host without a GPU fault.

HPR_E_NUMERIC: a start point with a NaN makes the iteration-0 residual check
NaN, and the solve stops with the numeric status instead of iterating on NaN
(the reference's loop would carry the NaN to max_iter).  HPR_E_TIMEOUT: a
bounded wait on the serving queue gives up and leaves the request running.
"""
import ctypes as C

import numpy as np
import pytest

from hprsocp_b200 import Context, HPRSOCP_parameters, _abi, instances
from hprsocp_b200.serving import Server

pytestmark = pytest.mark.gpu


def test_nan_start_point_is_a_numeric_error():
    model = instances.config0(0)
    x0 = np.zeros(model.n)
    x0[7] = np.nan
    with Context(model) as ctx:
        with pytest.raises(_abi.HPRError) as ei:
            ctx.solve(HPRSOCP_parameters(verbose=False, initial_x=x0))
        assert ei.value.code == _abi.HPR_E_NUMERIC
        assert "NaN" in str(ei.value)
    # a clean solve of the same instance in a new context is unaffected
    with Context(model) as ctx:
        r = ctx.solve(HPRSOCP_parameters(verbose=False, stoptol=1e-4))
    assert r.status == "OPTIMAL"


def test_serve_poll_times_out_on_a_running_request():
    model = instances.small_socp(5, n=2000, diag_q=False)
    # stoptol 0 with a time limit: the request runs for about a second
    p = HPRSOCP_parameters(verbose=False, stoptol=0.0, time_limit=1.0, max_iter=10**9)
    with Server(slots=1) as srv:
        t = srv.submit(model, p)
        r = _abi.hpr_results()
        x, y, z, w = np.zeros(model.n), np.zeros(model.m), np.zeros(model.n), np.zeros(model.n)
        r.x, r.y, r.z, r.w = _abi.dptr(x), _abi.dptr(y), _abi.dptr(z), _abi.dptr(w)
        lat = C.c_double()
        rc = srv.lib.hpr_serve_poll(srv.h, t, 1, C.byref(r), C.byref(lat))
        assert rc == _abi.HPR_E_TIMEOUT
        # the request is still there and finishes normally
        res, latency = srv.poll(t)
        assert res.status == "TIME_LIMIT" and latency >= 0.9

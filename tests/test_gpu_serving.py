"""Continuous-batching server (hpr_serve_*): every request's result is the
same alone and in the mix, each retires at its own tolerance, and admission
respects the HBM budget."""
import numpy as np
import pytest

from hprsocp_b200 import Context, HPRSOCP_parameters, _abi, instances
from hprsocp_b200.serving import ReplicatedServer, Server

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def stream():
    return instances.serving_stream(7, 40)


def _params(tol):
    return HPRSOCP_parameters(verbose=False, stoptol=tol, max_iter=200000)


@pytest.mark.parametrize("resident", [False, True])
def test_each_result_is_the_same_alone_and_in_the_mix(stream, resident):
    """A request solved alone (a one-slot server, nothing else on the
    device) and the same request among 40 submitted at once to 16 slots give
    the same bits, with the solve loops on the host or, for the problems
    small enough, in the device-resident request loop (one CTA per solve):
    every reduction has a fixed order."""
    alone = []
    with Server(slots=1, resident=resident) as srv:
        for model, tol, _ in stream:
            alone.append(srv.poll(srv.submit(model, _params(tol)))[0])
    with Server(slots=16, resident=resident) as srv:
        tickets = [srv.submit(model, _params(tol)) for model, tol, _ in stream]
        mixed = [srv.poll(t)[0] for t in tickets]
    for (model, tol, _), a, b in zip(stream, alone, mixed):
        assert a.status == b.status == "OPTIMAL"
        assert a.iter == b.iter
        assert b.residuals <= tol
        assert np.array_equal(a.x, b.x) and np.array_equal(a.y, b.y) and np.array_equal(a.z, b.z)


def test_device_loop_agrees_with_the_host_loop(stream):
    """The device-resident loop runs the host loop's logic with its
    reductions summed in another fixed order: each request reaches the same
    status at its tolerance with the objective within 10 x tol and the
    iteration count within one check interval.  With the loops on the host
    (the default), a server solve is hpr_solve on a private context, bit for
    bit."""
    host = []
    for model, tol, _ in stream:
        with Context(model) as ctx:
            host.append(ctx.solve(_params(tol)))
    with Server(slots=16, resident=True) as srv:
        dev = [srv.poll(t)[0] for t in [srv.submit(m, _params(tol)) for m, tol, _ in stream]]
    with Server(slots=16) as srv:
        off = [srv.poll(t)[0] for t in [srv.submit(m, _params(tol)) for m, tol, _ in stream]]
    for (model, tol, _), h, d, o in zip(stream, host, dev, off):
        assert h.status == d.status == "OPTIMAL" and d.residuals <= tol
        # both are tol-accurate solutions (tol 1e-4 or 1e-6)
        assert abs(d.primal_obj - h.primal_obj) <= 10 * tol * max(1.0, abs(h.primal_obj))
        assert abs(d.iter - h.iter) <= 150, (d.iter, h.iter)
        assert o.iter == h.iter and np.array_equal(o.x, h.x) and np.array_equal(o.y, h.y)


def test_each_request_retires_at_its_own_tolerance(stream):
    model = stream[0][0]
    with Server(slots=2) as srv:
        t4 = srv.submit(model, _params(1e-4))
        t6 = srv.submit(model, _params(1e-6))
        r4, _ = srv.poll(t4)
        r6, _ = srv.poll(t6)
    assert r4.residuals <= 1e-4 and r6.residuals <= 1e-6
    assert r4.iter <= r6.iter


def test_admission_by_hbm_budget(stream):
    """A small budget still serves every request that fits it; a request
    larger than the whole budget is refused at submission."""
    with Server(slots=4, hbm_budget=64 << 20) as srv:
        small = [m for m, _, _ in stream if m.n <= 600][:4]
        tickets = [srv.submit(m, _params(1e-4)) for m in small]
        assert srv.stats()["reserved_bytes"] <= 64 << 20
        for t in tickets:
            r, lat = srv.poll(t)
            assert r.status == "OPTIMAL" and lat > 0
        big = instances.small_socp(3, n=12000)
        with pytest.raises(_abi.HPRError) as e:
            srv.submit(big, _params(1e-4))
        assert e.value.code == _abi.HPR_E_BUDGET


def test_a_ticket_is_consumed_by_its_poll(stream):
    with Server(slots=2) as srv:
        t = srv.submit(stream[0][0], _params(1e-4))
        r, _ = srv.poll(t)
        assert r.status == "OPTIMAL"
        with pytest.raises(_abi.HPRError) as e:
            srv.poll(t)
        assert e.value.code == _abi.HPR_E_BAD_INPUT
        # the C entry point refuses it as well
        import ctypes as C
        lat = C.c_double()
        assert srv.lib.hpr_serve_poll(srv.h, t, 0, None, C.byref(lat)) == _abi.HPR_E_BAD_INPUT


def test_replicated_servers_give_the_single_server_results(stream):
    """Requests routed across replicas (two servers on device 0 here, one
    per GPU in production) give the bits a single server gives."""
    with Server(slots=8) as srv:
        single = [srv.poll(t)[0] for t in [srv.submit(m, _params(tol)) for m, tol, _ in stream[:12]]]
    with ReplicatedServer([0, 0], slots=4) as rs:
        tickets = [rs.submit(m, _params(tol)) for m, tol, _ in stream[:12]]
        assert {rs.device_of(t) for t in tickets} == {0} and min(rs._load) > 0
        routed = [rs.poll(t)[0] for t in tickets]
    for a, b in zip(single, routed):
        assert a.status == b.status == "OPTIMAL" and a.iter == b.iter
        assert np.array_equal(a.x, b.x) and np.array_equal(a.y, b.y)

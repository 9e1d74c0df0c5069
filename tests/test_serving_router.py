"""Routing of the serving stream across devices (ReplicatedServer), on CPU
with stand-in servers: each request goes to the device with the least
outstanding work, tickets are global, and a poll reaches the device that
holds the ticket.  The stand-ins record what they were given; the real
per-device server is covered by the GPU serving tests."""
import numpy as np
import pytest

from hprsocp_b200 import _abi, instances
from hprsocp_b200.serving import ReplicatedServer


class FakeServer:
    def __init__(self, device):
        self.device = device
        self.pending = {}
        self.next = 100 * device
        self.closed = False

    def submit(self, model, params=None):
        t = self.next
        self.next += 1
        self.pending[t] = model
        return t

    def poll(self, ticket, wait_ms=-1):
        if wait_ms == 0:
            return None
        model = self.pending.pop(ticket)
        return ("result", self.device, model.n), 0.0

    def stats(self):
        return {"queued": len(self.pending), "running": 0, "reserved_bytes": 10 * len(self.pending)}

    def close(self):
        self.closed = True


def _stream(k):
    return [instances.small_socp(s, n=n, diag_q=False) for s, n in zip(range(k), [400, 60, 60, 900, 120, 60][:k])]


def test_requests_go_to_the_least_loaded_device():
    srv = ReplicatedServer([0, 1, 2], make_server=FakeServer)
    models = _stream(6)
    tickets = [srv.submit(m) for m in models]
    assert tickets == list(range(6))
    # first three spread one per device, then each goes where the load is lowest
    loads = [0, 0, 0]
    for t, m in zip(tickets, models):
        i = min(range(3), key=lambda j: (loads[j], j))
        assert srv.device_of(t) == i
        loads[i] += ReplicatedServer.work_of(m)
    assert srv._load == loads
    assert srv.stats()["queued"] == 6 and set(srv.stats()["per_device"]) == {0, 1, 2}


def test_poll_reaches_the_holding_device_and_releases_its_load():
    srv = ReplicatedServer([3, 5], make_server=FakeServer)
    models = _stream(4)
    tickets = [srv.submit(m) for m in models]
    assert srv.poll(tickets[1], wait_ms=0) is None  # not finished: still held
    for t, m in zip(tickets, models):
        holder = srv.device_of(t)
        assert holder in (3, 5)
        (tag, dev, n), _ = srv.poll(t)
        assert tag == "result" and n == m.n and dev == holder
    assert srv._load == [0, 0] and srv.stats()["queued"] == 0
    with pytest.raises(_abi.HPRError):
        srv.poll(tickets[0])


def test_close_and_failed_construction_close_every_server():
    built = []

    def make(d):
        if d == 2:
            raise RuntimeError("no device 2")
        s = FakeServer(d)
        built.append(s)
        return s

    with pytest.raises(RuntimeError):
        ReplicatedServer([0, 1, 2], make_server=make)
    assert len(built) == 2 and all(s.closed for s in built)
    with ReplicatedServer([0, 1], make_server=FakeServer) as srv:
        servers = list(srv.servers)
    assert all(s.closed for s in servers)
    with pytest.raises(ValueError):
        ReplicatedServer([], make_server=FakeServer)


def test_work_counts_every_matrix():
    m = instances.small_socp(1, n=300, diag_q=True)
    w = ReplicatedServer.work_of(m)
    expect = m.A.nnz + m.m + m.n + (m.Q.nnz if m.Q is not None else 0) + (2 * m.F.nnz if m.F is not None else 0)
    assert w == expect and w > 0
    assert np.isscalar(w)

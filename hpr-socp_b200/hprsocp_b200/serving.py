"""Continuous-batching server (hpr_serve_*): many small SOCPs solved
concurrently on one device, each with its own parameters and tolerance."""
from __future__ import annotations

import ctypes as C
from typing import Optional

import numpy as np

from . import _abi
from .model import SOCPModel
from .solver import HPRSOCP_parameters, HPRSOCP_results, results_from_c


class Server:
    """`slots` solver contexts on one device; requests are admitted while
    their estimated device memory fits `hbm_budget` bytes (0 = 90% of free)."""

    def __init__(self, slots: int = 16, device: int = 0, hbm_budget: int = 0, resident: bool = False):
        self.lib = _abi.load_library()
        h = C.c_void_p()
        rc = self.lib.hpr_serve_create(device, slots, hbm_budget, C.byref(h))
        if rc != _abi.HPR_OK:
            raise _abi.HPRError(rc, self.lib.hpr_status_string(rc).decode())
        self.h = h
        self._shapes = {}
        # resident: small problems run their whole solve loop in the
        # device-resident request loop; False (default) keeps every loop on
        # the host
        self.lib.hpr_serve_set_resident(self.h, 1 if resident else 0)

    def _err(self, rc):
        msg = self.lib.hpr_serve_last_error(self.h).decode() if self.h else ""
        return _abi.HPRError(rc, f"{self.lib.hpr_status_string(rc).decode()}: {msg}")

    def submit(self, model: SOCPModel, params: Optional[HPRSOCP_parameters] = None) -> int:
        prob = model.to_c()
        p = (params or HPRSOCP_parameters(verbose=False)).to_c()
        t = C.c_int64()
        rc = self.lib.hpr_serve_submit(self.h, C.byref(prob), C.byref(p), C.byref(t))
        if rc != _abi.HPR_OK:
            raise self._err(rc)
        self._shapes[t.value] = (model.m, model.n)
        return t.value

    def poll(self, ticket: int, wait_ms: int = -1):
        """(HPRSOCP_results, latency_s), or None if not finished within wait_ms."""
        if ticket not in self._shapes:
            raise _abi.HPRError(_abi.HPR_E_BAD_INPUT, f"unknown or already consumed ticket {ticket}")
        m, n = self._shapes[ticket]
        x, y, z, w = np.zeros(n), np.zeros(m), np.zeros(n), np.zeros(n)
        r = _abi.hpr_results()
        r.x, r.y, r.z, r.w = _abi.dptr(x), _abi.dptr(y), _abi.dptr(z), _abi.dptr(w)
        lat = C.c_double()
        rc = self.lib.hpr_serve_poll(self.h, ticket, wait_ms, C.byref(r), C.byref(lat))
        if rc == _abi.HPR_E_TIMEOUT:
            return None
        del self._shapes[ticket]
        if rc != _abi.HPR_OK:
            raise self._err(rc)
        return results_from_c(r, x, y, z, w), lat.value

    def stats(self):
        q, run, res = C.c_int64(), C.c_int64(), C.c_size_t()
        self.lib.hpr_serve_stats(self.h, C.byref(q), C.byref(run), C.byref(res))
        return {"queued": q.value, "running": run.value, "reserved_bytes": res.value}

    def phase_times(self):
        """Mean per finished request: wall seconds of queue wait, upload,
        scaling, eigenvalue estimate, solve loop, read-back; the device
        loop's seconds in iterations, residual checks, M-norms, sigma
        updates, restarts, and its residual checks."""
        sec = (C.c_double * 12)()
        n = C.c_int64()
        self.lib.hpr_serve_phase_times(self.h, sec, C.byref(n))
        names = ("queue_wait", "upload", "scaling", "power_iteration", "solve_loop", "readback",
                 "device_iterations", "device_residual_checks", "device_mnorm", "device_sigma", "device_restart",
                 "device_checks")
        return {k: (sec[i] / n.value if n.value else 0.0) for i, k in enumerate(names)}

    def close(self):
        if getattr(self, "h", None):
            self.lib.hpr_serve_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class ReplicatedServer:
    """One `Server` per device, with each request routed to the device that
    has the least outstanding work (the sum of nnz(A) + nnz(Q) + m + n over
    its unfinished requests; ties go to the lowest device).  The serving
    stream shards with no exchange between devices, so each device runs its
    own server and the router only balances them.  Tickets are global:
    ``poll`` finds the device that holds a ticket.

    ``make_server(device)`` builds each device's server (default: ``Server``
    with this object's slots, budget and mode); anything with ``submit``,
    ``poll``, ``stats`` and ``close`` works, which is how the routing is
    tested without a GPU."""

    def __init__(self, devices, slots: int = 16, hbm_budget: int = 0, resident: bool = False, make_server=None):
        self.devices = list(devices)
        if not self.devices:
            raise ValueError("ReplicatedServer needs at least one device")
        if make_server is None:
            def make_server(d):
                return Server(slots=slots, device=d, hbm_budget=hbm_budget, resident=resident)
        self.servers = []
        try:
            for d in self.devices:
                self.servers.append(make_server(d))
        except Exception:
            self.close()
            raise
        self._load = [0] * len(self.servers)
        self._where = {}  # global ticket -> (replica index, local ticket, work)
        self._next = 0

    @staticmethod
    def work_of(model: SOCPModel) -> int:
        w = int(model.A.nnz) + int(model.m) + int(model.n)
        if model.Q is not None:
            w += int(model.Q.nnz)
        if model.F is not None:
            w += 2 * int(model.F.nnz)
        return w

    def route(self) -> int:
        """Replica index for the next request (least loaded first)."""
        return min(range(len(self.servers)), key=lambda i: (self._load[i], i))

    def submit(self, model: SOCPModel, params: Optional[HPRSOCP_parameters] = None) -> int:
        work = self.work_of(model)
        i = self.route()
        local = self.servers[i].submit(model, params)
        t = self._next
        self._next += 1
        self._where[t] = (i, local, work)
        self._load[i] += work
        return t

    def device_of(self, ticket: int) -> int:
        return self.devices[self._where[ticket][0]]

    def poll(self, ticket: int, wait_ms: int = -1):
        """(HPRSOCP_results, latency_s), or None if not finished within wait_ms."""
        if ticket not in self._where:
            raise _abi.HPRError(_abi.HPR_E_BAD_INPUT, f"unknown or already consumed ticket {ticket}")
        i, local, work = self._where[ticket]
        out = self.servers[i].poll(local, wait_ms)
        if out is None:
            return None
        del self._where[ticket]
        self._load[i] -= work
        return out

    def stats(self):
        per = [s.stats() for s in self.servers]
        tot = {k: sum(p[k] for p in per) for k in ("queued", "running", "reserved_bytes")}
        tot["per_device"] = {d: p for d, p in zip(self.devices, per)}
        return tot

    def close(self):
        for s in getattr(self, "servers", []):
            s.close()
        self.servers = []

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

"""Host API mirroring the reference's solver interface.

``HPRSOCP_parameters`` / ``HPRSOCP_results`` / ``optimize`` follow
src/structs.jl:208-314 and src/algorithm.jl:2538-2581; ``Context`` exposes the
fine-grained C-ABI operations (upload, scale, iterate, residuals, ...), which
the parity tests drive step by step.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass, field
from typing import Optional

import numpy as np

from . import _abi
from .model import SOCPModel


@dataclass
class HPRSOCP_parameters:
    """HPRSOCP_parameters (src/structs.jl:208-277) with the same defaults."""

    stoptol: float = 1e-6
    sigma: float = -1.0
    max_iter: int = 2147483647
    time_limit: float = 3600.0
    check_iter: int = 150
    warm_up: bool = False
    print_frequency: int = -1
    device_number: int = 0
    use_Ruiz_scaling: bool = True
    ruiz_iterations: int = 10
    use_bc_scaling: bool = True
    bc_scaling_norm_type: str = "l2"
    use_l2_scaling: bool = False  # accepted and unused, as in the reference
    use_Pock_Chambolle_scaling: bool = True
    soc_block_scaling_strategy: str = "phase_taper"
    initial_x: Optional[np.ndarray] = None
    initial_y: Optional[np.ndarray] = None
    # auto-save: current and best iterates on print iterations and at the end,
    # as a .npz archive whose member names are the reference's HDF5 paths
    auto_save: bool = False
    save_filename: str = "HPRSOCP_autosave.npz"
    verbose: bool = True
    use_gpu: bool = True
    # extensions: injected eigenvalue bounds and SpMV precision
    lambda_max_A: float = -1.0
    lambda_max_Q: float = -1.0
    precision: str = "fp64"
    refine: int = 0  # reduced precision: FP64 finish below refine x stoptol (0: 10x); < 0: never
    _keep: list = field(default_factory=list, repr=False)

    def to_c(self) -> _abi.hpr_params:
        if self.sigma != -1 and not self.sigma > 0:
            raise ValueError(f"Invalid sigma value: {self.sigma}. It should be a positive number or -1 for automatic.")
        if self.print_frequency != -1 and self.print_frequency <= 0:
            raise ValueError(f"Invalid print_frequency: {self.print_frequency}. It should be a positive integer "
                             "or -1 for automatic printing.")
        if self.soc_block_scaling_strategy not in _abi.SOC_SCALE_STRATEGIES:
            raise ValueError(f"Unsupported soc_block_scaling_strategy={self.soc_block_scaling_strategy}.")
        if self.bc_scaling_norm_type not in _abi.HPR_BC_NORM:
            raise ValueError(f"Unsupported bc scaling norm_type: {self.bc_scaling_norm_type}. Use :l2, :rms, or :linf.")
        p = _abi.hpr_params()
        p.stoptol = self.stoptol
        p.sigma = self.sigma
        p.max_iter = int(min(self.max_iter, 2**62))
        p.time_limit = self.time_limit
        p.check_iter = self.check_iter
        p.print_frequency = self.print_frequency
        p.device_number = self.device_number
        p.use_Ruiz_scaling = int(self.use_Ruiz_scaling)
        p.ruiz_iterations = self.ruiz_iterations
        p.use_bc_scaling = int(self.use_bc_scaling)
        p.bc_scaling_norm_type = _abi.HPR_BC_NORM[self.bc_scaling_norm_type]
        p.use_Pock_Chambolle_scaling = int(self.use_Pock_Chambolle_scaling)
        p.soc_block_scaling_strategy = _abi.SOC_SCALE_STRATEGIES[self.soc_block_scaling_strategy]
        p.verbose = int(self.verbose)
        keep = []
        if self.initial_x is not None:
            ix = np.ascontiguousarray(self.initial_x, dtype=np.float64)
            keep.append(ix)
            p.initial_x = _abi.dptr(ix)
        if self.initial_y is not None:
            iy = np.ascontiguousarray(self.initial_y, dtype=np.float64)
            keep.append(iy)
            p.initial_y = _abi.dptr(iy)
        p.lambda_max_A = self.lambda_max_A
        p.lambda_max_Q = self.lambda_max_Q
        p.precision = _abi.HPR_PREC[self.precision]
        p.refine = int(self.refine)
        p.auto_save = int(self.auto_save)
        fn = os.fsencode(self.save_filename)
        keep.append(fn)
        p.save_filename = fn
        self._keep = keep
        return p


@dataclass
class HPRSOCP_results:
    """HPRSOCP_results (src/structs.jl:297-314)."""

    iter: int = 0
    iter_4: int = 0
    iter_6: int = 0
    time: float = 0.0
    time_4: float = 0.0
    time_6: float = 0.0
    power_time: float = 0.0
    primal_obj: float = 0.0
    residuals: float = 0.0
    gap: float = 0.0
    status: str = ""
    x: np.ndarray = None
    y: np.ndarray = None
    z: np.ndarray = None
    w: np.ndarray = None
    restarts: int = 0
    sigma: float = 0.0
    lambda_max_A: float = 0.0
    lambda_max_Q: float = 0.0
    last: dict = None


def results_from_c(r: _abi.hpr_results, x, y, z, w) -> HPRSOCP_results:
    return HPRSOCP_results(
        iter=r.iter, iter_4=r.iter_4, iter_6=r.iter_6, time=r.time, time_4=r.time_4,
        time_6=r.time_6, power_time=r.power_time, primal_obj=r.primal_obj,
        residuals=r.residuals, gap=r.gap, status=_abi.HPR_STATUS.get(r.status, "ERROR"),
        x=x, y=y, z=z, w=w, restarts=r.restarts, sigma=r.sigma_final,
        lambda_max_A=r.lambda_max_A, lambda_max_Q=r.lambda_max_Q, last=r.last.as_dict())


class Context:
    """One device context holding one uploaded problem (hpr_create/upload)."""

    def __init__(self, model: SOCPModel, device: int = 0, budget: int = 0, problem=None,
                 with_transpose: bool = False):
        """``problem`` uploads a caller-built hpr_problem (whose arrays the
        caller keeps alive) instead of ``model.to_c(with_transpose)``."""
        self.lib = _abi.load_library()
        self.model = model
        h = C.c_void_p()
        rc = self.lib.hpr_create(device, budget, C.byref(h))
        if rc != _abi.HPR_OK:
            raise _abi.HPRError(rc, self.lib.hpr_status_string(rc).decode())
        self.h = h
        self._prob = problem if problem is not None else model.to_c(with_transpose)
        self._check(self.lib.hpr_upload(self.h, C.byref(self._prob)))

    # -- plumbing ---------------------------------------------------------------
    def _check(self, rc: int):
        if rc != _abi.HPR_OK:
            msg = self.lib.hpr_last_error(self.h).decode() if self.h else ""
            raise _abi.HPRError(rc, f"{self.lib.hpr_status_string(rc).decode()}: {msg}")

    def close(self):
        if getattr(self, "h", None):
            self.lib.hpr_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # -- operations ---------------------------------------------------------------
    def scale(self, params: Optional[HPRSOCP_parameters] = None) -> dict:
        p = (params or HPRSOCP_parameters()).to_c()
        info = _abi.hpr_scale_info()
        self._check(self.lib.hpr_scale(self.h, C.byref(p), C.byref(info)))
        return {k: getattr(info, k) for k, _ in info._fields_}

    def power_A(self, maxit: int = 5000, tol: float = 1e-4) -> float:
        v = C.c_double()
        self._check(self.lib.hpr_power_A(self.h, maxit, tol, C.byref(v)))
        return v.value

    def power_Q(self, maxit: int = 5000, tol: float = 1e-4) -> float:
        v = C.c_double()
        self._check(self.lib.hpr_power_Q(self.h, maxit, tol, C.byref(v)))
        return v.value

    def set_sigma_lambda(self, sigma: float, lamA: float, lamQ: float = 0.0):
        self._check(self.lib.hpr_set_sigma_lambda(self.h, sigma, lamA, lamQ))

    def set_inner(self, inner: int):
        self._check(self.lib.hpr_set_inner(self.h, inner))

    def scalars(self):
        s, a, q = C.c_double(), C.c_double(), C.c_double()
        k = C.c_int64()
        self._check(self.lib.hpr_get_scalars(self.h, C.byref(s), C.byref(a), C.byref(q), C.byref(k)))
        return s.value, a.value, q.value, k.value

    def iterate(self, k: int, full_last: bool = True):
        self._check(self.lib.hpr_iterate(self.h, k, int(full_last)))

    def device_memory(self):
        """(bytes held within the HBM budget, live device allocations)."""
        used, n = C.c_size_t(), C.c_int64()
        self._check(self.lib.hpr_device_memory(self.h, C.byref(used), C.byref(n)))
        return used.value, n.value

    def last_iterate(self):
        ms = C.c_double()
        n = C.c_int64()
        self._check(self.lib.hpr_last_iterate_ms(self.h, C.byref(ms), C.byref(n)))
        return ms.value, n.value

    def iteration_bytes(self) -> float:
        b = C.c_double()
        self._check(self.lib.hpr_iteration_bytes(self.h, C.byref(b)))
        return b.value

    def residuals(self, include_bounds: bool = False) -> dict:
        r = _abi.hpr_residuals()
        self._check(self.lib.hpr_compute_residuals(self.h, int(include_bounds), C.byref(r)))
        return r.as_dict()

    def residuals_noalloc(self, include_bounds: bool = False) -> dict:
        r = _abi.hpr_residuals()
        self._check(self.lib.hpr_compute_residuals_noalloc(self.h, int(include_bounds), C.byref(r)))
        return r.as_dict()

    def mnorm(self) -> float:
        v = C.c_double()
        self._check(self.lib.hpr_mnorm(self.h, C.byref(v)))
        return v.value

    def sigma_terms(self):
        a, b, c, d = C.c_double(), C.c_double(), C.c_double(), C.c_double()
        self._check(self.lib.hpr_sigma_terms(self.h, C.byref(a), C.byref(b), C.byref(c), C.byref(d)))
        return a.value, b.value, c.value, d.value

    def golden_diag(self, a, b, lo=1e-12, hi=1e12, tol=1e-13) -> float:
        v = C.c_double()
        self._check(self.lib.hpr_sigma_golden_diag(self.h, a, b, lo, hi, tol, C.byref(v)))
        return v.value

    def restart(self):
        self._check(self.lib.hpr_restart(self.h))

    def _len(self, name: str) -> int:
        m, n = self.model.m, self.model.n
        if name in ("y", "y_bar", "last_y", "s", "dy", "row_norm", "AL", "AU"):
            return m
        if name == "soc_rhs":
            return m - self.model.number_linear_con
        if name in ("A_values", "AT_values"):
            return self.model.A.nnz
        return n

    def get(self, name: str) -> np.ndarray:
        out = np.zeros(self._len(name))
        self._check(self.lib.hpr_get_vector(self.h, _abi.VEC[name], _abi.dptr(out), len(out)))
        return out

    def set(self, name: str, arr):
        a = np.ascontiguousarray(arr, dtype=np.float64)
        self._check(self.lib.hpr_set_vector(self.h, _abi.VEC[name], _abi.dptr(a), len(a)))

    def solution(self):
        m, n = self.model.m, self.model.n
        x, y, z, w = np.zeros(n), np.zeros(m), np.zeros(n), np.zeros(n)
        self._check(self.lib.hpr_get_solution(self.h, _abi.dptr(x), _abi.dptr(y), _abi.dptr(z), _abi.dptr(w)))
        return x, y, z, w

    def set_schedule(self, mode: str):
        """'auto' (timed choice per size class), 'engine' or 'fused'."""
        self._check(self.lib.hpr_set_schedule(self.h, _abi.HPR_SCHEDULE[mode]))

    def set_precision(self, mode: str):
        self._check(self.lib.hpr_set_precision(self.h, _abi.HPR_PREC[mode]))

    def solve(self, params: Optional[HPRSOCP_parameters] = None) -> HPRSOCP_results:
        params = params or HPRSOCP_parameters()
        p = params.to_c()
        m, n = self.model.m, self.model.n
        x, y, z, w = np.zeros(n), np.zeros(m), np.zeros(n), np.zeros(n)
        r = _abi.hpr_results()
        r.x, r.y, r.z, r.w = _abi.dptr(x), _abi.dptr(y), _abi.dptr(z), _abi.dptr(w)
        self._check(self.lib.hpr_solve(self.h, C.byref(p), C.byref(r)))
        return results_from_c(r, x, y, z, w)


def optimize(model: SOCPModel, params: Optional[HPRSOCP_parameters] = None) -> HPRSOCP_results:
    """optimize (src/algorithm.jl:2538-2581): scaling, power iteration and the
    HPR loop on one B200.  ``warm_up`` is accepted and ignored: the kernels
    are compiled ahead of time, so there is no JIT to warm."""
    params = params or HPRSOCP_parameters()
    if not params.use_gpu:
        raise ValueError("this build has no CPU path: use_gpu must be true")
    with Context(model, device=params.device_number) as ctx:
        return ctx.solve(params)

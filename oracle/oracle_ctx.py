"""Python binding of the CPU oracle (TEST INFRASTRUCTURE ONLY).

``OracleContext`` mirrors ``hprsocp_b200.Context`` method for method so a test
can run the same call sequence on the oracle and on the CUDA library.  Only
tests/, the smoke check and the benchmark's CPU-baseline / reference arm use
this module; the product never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, os.path.join(ROOT, "hpr-socp_b200"))
from hprsocp_b200 import _abi  # noqa: E402
from hprsocp_b200.solver import HPRSOCP_parameters, results_from_c  # noqa: E402

LIB = os.path.join(HERE, "_build", "libhpr_oracle.so")
_lib = None


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        try:
            build()  # no-op when up to date
        except (OSError, subprocess.CalledProcessError):
            if not os.path.exists(LIB):
                raise
        L = C.CDLL(LIB)
        vp, dp, lp = C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_int64)
        sig = {
            "oracle_create": (C.c_int, [C.POINTER(_abi.hpr_problem), C.c_int, C.POINTER(vp)]),
            "oracle_destroy": (None, [vp]),
            "oracle_last_error": (C.c_char_p, [vp]),
            "oracle_scale": (C.c_int, [vp, C.POINTER(_abi.hpr_params), C.POINTER(_abi.hpr_scale_info)]),
            "oracle_power_A": (C.c_int, [vp, C.c_int, C.c_double, dp]),
            "oracle_power_Q": (C.c_int, [vp, C.c_int, C.c_double, dp]),
            "oracle_set_sigma_lambda": (C.c_int, [vp, C.c_double, C.c_double, C.c_double]),
            "oracle_set_inner": (C.c_int, [vp, C.c_int64]),
            "oracle_get_scalars": (C.c_int, [vp, dp, dp, dp, lp]),
            "oracle_iterate": (C.c_int, [vp, C.c_int64, C.c_int]),
            "oracle_residuals": (C.c_int, [vp, C.c_int, C.POINTER(_abi.hpr_residuals)]),
            "oracle_mnorm": (C.c_int, [vp, dp]),
            "oracle_sigma_terms": (C.c_int, [vp, dp, dp, dp, dp]),
            "oracle_sigma_golden_diag": (C.c_int, [vp, C.c_double, C.c_double, C.c_double, C.c_double,
                                                   C.c_double, dp]),
            "oracle_restart": (C.c_int, [vp]),
            "oracle_get_vector": (C.c_int, [vp, C.c_int, dp, C.c_size_t]),
            "oracle_set_vector": (C.c_int, [vp, C.c_int, dp, C.c_size_t]),
            "oracle_get_solution": (C.c_int, [vp, dp, dp, dp, dp]),
            "oracle_solve": (C.c_int, [vp, C.POINTER(_abi.hpr_params), C.POINTER(_abi.hpr_results)]),
            "oracle_golden": (C.c_double, [C.c_double] * 7 + [C.c_int]),
            "oracle_print_step": (C.c_double, [C.c_int64]),
        }
        for k, (r, a) in sig.items():
            f = getattr(L, k)
            f.restype = r
            f.argtypes = a
        _lib = L
    return _lib


class OracleContext:
    def __init__(self, model, threads: int = 0):
        self.lib = lib()
        self.model = model
        self._prob = model.to_c()
        h = C.c_void_p()
        rc = self.lib.oracle_create(C.byref(self._prob), threads, C.byref(h))
        if rc != 0:
            raise _abi.HPRError(rc, "oracle_create failed")
        self.h = h

    def _check(self, rc):
        if rc != 0:
            raise _abi.HPRError(rc, self.lib.oracle_last_error(self.h).decode())

    def close(self):
        if getattr(self, "h", None):
            self.lib.oracle_destroy(self.h)
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

    def scale(self, params=None):
        p = (params or HPRSOCP_parameters()).to_c()
        info = _abi.hpr_scale_info()
        self._check(self.lib.oracle_scale(self.h, C.byref(p), C.byref(info)))
        return {k: getattr(info, k) for k, _ in info._fields_}

    def power_A(self, maxit=5000, tol=1e-4):
        v = C.c_double()
        self._check(self.lib.oracle_power_A(self.h, maxit, tol, C.byref(v)))
        return v.value

    def power_Q(self, maxit=5000, tol=1e-4):
        v = C.c_double()
        self._check(self.lib.oracle_power_Q(self.h, maxit, tol, C.byref(v)))
        return v.value

    def set_sigma_lambda(self, sigma, lamA, lamQ=0.0):
        self._check(self.lib.oracle_set_sigma_lambda(self.h, sigma, lamA, lamQ))

    def set_inner(self, inner):
        self._check(self.lib.oracle_set_inner(self.h, inner))

    def scalars(self):
        s, a, q = C.c_double(), C.c_double(), C.c_double()
        k = C.c_int64()
        self._check(self.lib.oracle_get_scalars(self.h, C.byref(s), C.byref(a), C.byref(q), C.byref(k)))
        return s.value, a.value, q.value, k.value

    def iterate(self, k, full_last=True):
        self._check(self.lib.oracle_iterate(self.h, k, int(full_last)))

    def residuals(self, include_bounds=False):
        r = _abi.hpr_residuals()
        self._check(self.lib.oracle_residuals(self.h, int(include_bounds), C.byref(r)))
        return r.as_dict()

    def mnorm(self):
        v = C.c_double()
        self._check(self.lib.oracle_mnorm(self.h, C.byref(v)))
        return v.value

    def sigma_terms(self):
        a, b, c, d = C.c_double(), C.c_double(), C.c_double(), C.c_double()
        self._check(self.lib.oracle_sigma_terms(self.h, C.byref(a), C.byref(b), C.byref(c), C.byref(d)))
        return a.value, b.value, c.value, d.value

    def golden_diag(self, a, b, lo=1e-12, hi=1e12, tol=1e-13):
        v = C.c_double()
        self._check(self.lib.oracle_sigma_golden_diag(self.h, a, b, lo, hi, tol, C.byref(v)))
        return v.value

    def restart(self):
        self._check(self.lib.oracle_restart(self.h))

    def _len(self, name):
        m, n = self.model.m, self.model.n
        if name in ("y", "y_bar", "last_y", "s", "dy", "row_norm", "AL", "AU"):
            return m
        if name == "soc_rhs":
            return m - self.model.number_linear_con
        if name in ("A_values", "AT_values"):
            return self.model.A.nnz
        return n

    def get(self, name):
        out = np.zeros(self._len(name))
        self._check(self.lib.oracle_get_vector(self.h, _abi.VEC[name], _abi.dptr(out), len(out)))
        return out

    def set(self, name, arr):
        a = np.ascontiguousarray(arr, dtype=np.float64)
        self._check(self.lib.oracle_set_vector(self.h, _abi.VEC[name], _abi.dptr(a), len(a)))

    def solution(self):
        m, n = self.model.m, self.model.n
        x, y, z, w = np.zeros(n), np.zeros(m), np.zeros(n), np.zeros(n)
        self._check(self.lib.oracle_get_solution(self.h, _abi.dptr(x), _abi.dptr(y), _abi.dptr(z), _abi.dptr(w)))
        return x, y, z, w

    def solve(self, params=None):
        params = params or HPRSOCP_parameters()
        p = params.to_c()
        m, n = self.model.m, self.model.n
        x, y, z, w = np.zeros(n), np.zeros(m), np.zeros(n), np.zeros(n)
        r = _abi.hpr_results()
        r.x, r.y, r.z, r.w = _abi.dptr(x), _abi.dptr(y), _abi.dptr(z), _abi.dptr(w)
        self._check(self.lib.oracle_solve(self.h, C.byref(p), C.byref(r)))
        return results_from_c(r, x, y, z, w)


def golden(a, b, c, d, lo=1e-12, hi=1e12, tol=1e-13, maxiter=200):
    return lib().oracle_golden(a, b, c, d, lo, hi, tol, maxiter)


def print_step(it):
    return lib().oracle_print_step(it)

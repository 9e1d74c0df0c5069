"""Canonical SOCP model, the builder of the reference, and its C-ABI view.

Canonical ordering (src/utils/builders.jl:8-22 of the reference): linear rows
of A first (equalities, then inequalities), cone rows last; boxed variables
first, cone variables last with every cone contiguous.  Indices are stored
0-based here; ``build_from_SOCP_data`` accepts the reference's 1-based cone
index vectors by default.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import Optional

import numpy as np
import scipy.sparse as sp

from . import _abi


def _csr32(M, shape=None) -> sp.csr_matrix:
    if M is None:
        return sp.csr_matrix(shape, dtype=np.float64)
    if isinstance(M, np.ndarray):
        M = sp.csr_matrix(M)
    M = sp.csr_matrix(M, dtype=np.float64)
    M.sum_duplicates()
    M.sort_indices()
    M.indptr = M.indptr.astype(np.int32)
    M.indices = M.indices.astype(np.int32)
    return M


@dataclass
class SOCPModel:
    """QP_info_cpu (src/structs.jl:97-150) with 0-based cone indices."""

    A: sp.csr_matrix
    c: np.ndarray
    AL: np.ndarray
    AU: np.ndarray
    l: np.ndarray
    u: np.ndarray
    soc_rhs: np.ndarray
    SOC_con_idx: np.ndarray  # 0-based starts + end sentinel
    SOC_var_idx: np.ndarray
    number_linear_con: int
    number_lu_x: int
    Q: Optional[sp.csr_matrix] = None        # explicit Q (HPR_Q_CSR)
    q_diag: Optional[np.ndarray] = None      # operator diag(q_diag) + F'F
    F: Optional[sp.csr_matrix] = None
    obj_constant: float = 0.0
    AT: Optional[sp.csr_matrix] = None
    _keep: list = field(default_factory=list, repr=False)

    def __post_init__(self):
        self.A = _csr32(self.A)
        m, n = self.A.shape
        for name in ("c", "AL", "AU", "l", "u", "soc_rhs"):
            setattr(self, name, np.ascontiguousarray(getattr(self, name), dtype=np.float64))
        self.SOC_con_idx = np.ascontiguousarray(self.SOC_con_idx, dtype=np.int64)
        self.SOC_var_idx = np.ascontiguousarray(self.SOC_var_idx, dtype=np.int64)
        if self.Q is not None:
            self.Q = _csr32(self.Q)
            if self.Q.nnz == 0:
                self.Q = None
        if self.F is not None:
            self.F = _csr32(self.F)
            self.q_diag = np.ascontiguousarray(self.q_diag, dtype=np.float64)
        if self.AT is None:
            self.AT = _csr32(self.A.T.tocsr())
        else:
            self.AT = _csr32(self.AT)

    @property
    def m(self) -> int:
        return self.A.shape[0]

    @property
    def n(self) -> int:
        return self.A.shape[1]

    @property
    def soc_rhs_full(self) -> np.ndarray:
        full = np.zeros(self.m)
        full[self.number_linear_con:] = self.soc_rhs
        return full

    @property
    def has_quadratic_terms(self) -> bool:
        """has_quadratic_terms (Q_operators/Q_operator_interface.jl:118-121)."""
        return self.F is not None or (self.Q is not None and self.Q.nnz > 0)

    def q_matvec(self, v: np.ndarray) -> np.ndarray:
        if self.F is not None:
            return self.q_diag * v + self.F.T @ (self.F @ v)
        if self.Q is not None:
            return self.Q @ v
        return np.zeros_like(v)

    # -- C ABI view -----------------------------------------------------------
    @staticmethod
    def _csr_struct(M: Optional[sp.csr_matrix], keep: list) -> _abi.hpr_csr:
        s = _abi.hpr_csr()
        if M is None:
            return s
        rp = np.ascontiguousarray(M.indptr, dtype=np.int32)
        ci = np.ascontiguousarray(M.indices, dtype=np.int32)
        v = np.ascontiguousarray(M.data, dtype=np.float64)
        keep += [rp, ci, v]
        s.nrows, s.ncols = M.shape
        s.nnz = M.nnz
        s.rowptr = _abi.iptr(rp)
        s.colind = _abi.iptr(ci)
        s.values = _abi.dptr(v)
        return s

    def to_c(self, with_transpose: bool = False) -> _abi.hpr_problem:
        """A struct pointing at this model's arrays (kept alive by the model).

        A' is formed on the device unless ``with_transpose`` passes the
        model's own copy (the reference's QP_info_cpu.AT)."""
        keep: list = []
        p = _abi.hpr_problem()
        p.m, p.n = self.A.shape
        p.m_lin = int(self.number_linear_con)
        p.n_box = int(self.number_lu_x)
        p.A = self._csr_struct(self.A, keep)
        if with_transpose:
            p.AT = self._csr_struct(self.AT, keep)
        for name in ("c", "l", "u", "AL", "AU", "soc_rhs"):
            arr = np.ascontiguousarray(getattr(self, name), dtype=np.float64)
            keep.append(arr)
            setattr(p, name, _abi.dptr(arr))
        ci = np.ascontiguousarray(self.SOC_con_idx, dtype=np.int64)
        vi = np.ascontiguousarray(self.SOC_var_idx, dtype=np.int64)
        keep += [ci, vi]
        p.soc_con_idx = _abi.lptr(ci)
        p.n_soc_con_idx = len(ci)
        p.soc_var_idx = _abi.lptr(vi)
        p.n_soc_var_idx = len(vi)
        p.index_base = 0
        if self.F is not None:
            p.q_kind = _abi.HPR_Q_DIAG_LOWRANK
            p.F = self._csr_struct(self.F, keep)
            qd = np.ascontiguousarray(self.q_diag, dtype=np.float64)
            keep.append(qd)
            p.q_diag = _abi.dptr(qd)
        elif self.Q is not None:
            p.q_kind = _abi.HPR_Q_CSR
            p.Q = self._csr_struct(self.Q, keep)
        else:
            p.q_kind = _abi.HPR_Q_NONE
        p.obj_constant = float(self.obj_constant)
        self._keep = keep
        return p

    def nbytes(self, with_transpose: bool = False) -> int:
        """Bytes ``to_c(with_transpose)`` hands to the library."""
        b = self.A.data.nbytes + self.A.indices.nbytes + self.A.indptr.nbytes
        if with_transpose:
            b += self.AT.data.nbytes + self.AT.indices.nbytes + self.AT.indptr.nbytes
        for name in ("c", "AL", "AU", "l", "u", "soc_rhs"):
            b += getattr(self, name).nbytes
        return b


def build_from_SOCP_data(Q, c, A, rhs, SOC_con_idx, number_eq, number_ineq, l, u,
                         SOC_var_idx, obj_constant: float = 0.0, verbose: bool = True,
                         index_base: int = 1) -> SOCPModel:
    """build_from_SOCP_data (src/utils/builders.jl:24-108).

    Equality rows get AL = AU = rhs, inequality rows are ``>= rhs``
    (AU = +Inf), cone rows keep rhs as ``soc_rhs``.  Cone index vectors use the
    reference's 1-based convention unless ``index_base=0``.  Raises
    ValueError with the reference's messages on malformed input.
    """
    A = _csr32(A)
    m, n = A.shape
    c = np.asarray(c, dtype=np.float64).copy()
    rhs = np.asarray(rhs, dtype=np.float64).copy()
    l = np.asarray(l, dtype=np.float64).copy()
    u = np.asarray(u, dtype=np.float64).copy()
    con = np.asarray(SOC_con_idx, dtype=np.int64) - index_base
    var = np.asarray(SOC_var_idx, dtype=np.int64) - index_base
    if len(c) != n:
        raise ValueError("Dimension mismatch: length(c) must equal number of columns of A.")
    if len(rhs) != m:
        raise ValueError("Dimension mismatch: length(rhs) must equal number of rows of A.")
    if len(l) != n:
        raise ValueError("Dimension mismatch: length(l) must equal number of variables.")
    if len(u) != n:
        raise ValueError("Dimension mismatch: length(u) must equal number of variables.")
    if number_eq < 0:
        raise ValueError("number_eq must be nonnegative.")
    if number_ineq < 0:
        raise ValueError("number_ineq must be nonnegative.")
    if number_eq + number_ineq > m:
        raise ValueError("number_eq + number_ineq cannot exceed the number of rows of A.")
    if len(con) == 0:
        raise ValueError("SOC_con_idx must contain at least one sentinel entry.")
    if len(var) == 0:
        raise ValueError("SOC_var_idx must contain at least one sentinel entry.")
    if con[0] != number_eq + number_ineq:
        raise ValueError("SOC_con_idx must start at number_eq + number_ineq + 1.")
    if con[-1] != m:
        raise ValueError("SOC_con_idx must end at m + 1.")
    nlin = number_eq + number_ineq
    soc_rhs = rhs[nlin:].copy()
    number_lu_x = int(var[0])
    if var[-1] != n:
        raise ValueError("SOC_var_idx must end at n + 1.")
    if not (0 <= number_lu_x <= n):
        raise ValueError("Invalid SOC_var_idx start.")
    AL = np.full(m, -np.inf)
    AU = np.full(m, np.inf)
    AL[:number_eq] = rhs[:number_eq]
    AU[:number_eq] = rhs[:number_eq]
    AL[number_eq:nlin] = rhs[number_eq:nlin]
    Qm = None if Q is None else _csr32(Q)
    return SOCPModel(A=A, c=c, AL=AL, AU=AU, l=l, u=u, soc_rhs=soc_rhs,
                     SOC_con_idx=con, SOC_var_idx=var, number_linear_con=nlin,
                     number_lu_x=number_lu_x, Q=Qm, obj_constant=float(obj_constant))

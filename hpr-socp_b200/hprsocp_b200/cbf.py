"""CBF (Conic Benchmark Format) ingest for SOCP instances.

``read_cbf`` returns the inputs of ``build_from_SOCP_data`` exactly as the
reference's reader does (read_cbf / _read_cbf_mmap / _cbf_prepare_layout,
src/utils/cbf_io.jl:1133-1455 and 493-634).  It runs the library's
multi-threaded C++ reader (``hpr_cbf_read``); ``read_cbf_py`` is a
line-by-line Python restatement of the same rules, kept to check it.

* constraint rows are reordered as equalities (L=), inequalities (L+ and L-,
  the latter negated so every inequality reads ``A x >= rhs``) and second
  order cone rows (Q); free rows (F) are dropped;
* CBF states ``A x + b`` in the cone, so ``rhs = -b`` on L=, L+ and Q rows
  and ``rhs = b`` on (negated) L- rows;
* variables are reordered as linear (L+ >= 0, L- <= 0, L= fixed at 0,
  F free) followed by cone variables (Q);
* ACOORD entries with value zero are skipped, duplicate (row, col) entries
  are summed in file order and sums equal to zero are dropped; BCOORD and
  OBJACOORD entries are assignments (a later entry for an index wins);
  entries read before both CON and VAR are applied after the others;
* ``OBJSENSE MAX`` (or ``SENSE max``) negates c and the offset;
* cone index vectors are 1-based, as the builder's default expects.

Only the conic-linear subset is accepted: PSD blocks, matrix variables,
integer variables (sections with a nonzero count) and other cones (for
example QR) raise ValueError with the reference's messages.
"""
from __future__ import annotations

import ctypes as C
import os
import re

import numpy as np
import scipy.sparse as sp

from . import _abi
from .model import SOCPModel, build_from_SOCP_data

_SUPPORTED = ("L+", "L-", "L=", "Q", "F")


def _check_extension(filename: str):
    if not (filename.endswith(".cbf") or filename.endswith(".CBF")):
        raise ValueError("Unsupported file format. Please provide a .cbf file.")


def read_cbf(filename: str, threads: int = 0):
    """(Q, c, A, rhs, SOC_con_idx, number_eq, number_ineq, l, u, SOC_var_idx,
    obj_constant) in the builder's layout, parsed by the library's C++ reader
    with `threads` host threads (0: all)."""
    _check_extension(filename)
    lib = _abi.load_library()
    h = C.c_void_p()
    rc = lib.hpr_cbf_read(os.fsencode(filename), int(threads), C.byref(h))
    if rc != _abi.HPR_OK:
        raise ValueError(lib.hpr_cbf_last_error().decode())
    try:
        d = _abi.hpr_cbf_data()
        if lib.hpr_cbf_data_get(h, C.byref(d)) != _abi.HPR_OK:
            raise RuntimeError("hpr_cbf_data_get failed")
        m, n, nnz = d.m, d.n, d.A.nnz

        def arr(ptr, k, dtype):
            if k == 0:
                return np.zeros(0, dtype=dtype)
            return np.ctypeslib.as_array(ptr, shape=(k,)).astype(dtype, copy=True)

        indptr = arr(d.A.rowptr, m + 1, np.int32)
        A = sp.csr_matrix((arr(d.A.values, nnz, np.float64), arr(d.A.colind, nnz, np.int32), indptr),
                          shape=(m, n))
        out = (sp.csr_matrix((n, n)), arr(d.c, n, np.float64), A, arr(d.rhs, m, np.float64),
               arr(d.soc_con_idx, d.n_soc_con_idx, np.int64), int(d.number_eq), int(d.number_ineq),
               arr(d.l, n, np.float64), arr(d.u, n, np.float64), arr(d.soc_var_idx, d.n_soc_var_idx, np.int64),
               float(d.obj_constant))
    finally:
        lib.hpr_cbf_free(h)
    return out


def read_cbf_model(filename: str, verbose: bool = False, threads: int = 0) -> SOCPModel:
    """read_cbf followed by build_from_SOCP_data (1-based cone indices)."""
    Q, c, A, rhs, con, n_eq, n_ineq, l, u, var, const = read_cbf(filename, threads)
    return build_from_SOCP_data(Q, c, A, rhs, con, n_eq, n_ineq, l, u, var, obj_constant=const, verbose=verbose)


# ---------------------------------------------------------------------------
# Python restatement (checks the C++ reader)
# ---------------------------------------------------------------------------
_TERM = re.compile(r"\r\n|\r|\n")
_FLOAT = re.compile(r"[+-]?(?:(?:\d+\.?\d*|\.\d+)(?:[eE][+-]?\d+)?|infinity|inf|nan)", re.IGNORECASE)
_SPACE = " \t\r"


class _Lines:
    """_cbf_next_line_bounds / _cbf_next_data_line over the file's lines."""

    def __init__(self, text: str):
        self.lines = _TERM.split(text) if text else []
        if text and text[-1] in "\r\n":
            self.lines.pop()
        self.i = 0

    def raw(self):
        if self.i >= len(self.lines):
            return None
        self.i += 1
        return self.lines[self.i - 1]

    def data(self):
        while True:
            s = self.raw()
            if s is None:
                return None
            t = s.strip(_SPACE)
            if t and t[0] != "#":
                return t


def _int(s: str, i: int):
    n = len(s)
    while i < n and s[i] in _SPACE:
        i += 1
    if i >= n:
        raise ValueError("Invalid CBF line: expected integer token.")
    sign = 1
    if s[i] == "-":
        sign, i = -1, i + 1
    elif s[i] == "+":
        i += 1
    j = i
    while j < n and "0" <= s[j] <= "9":
        j += 1
    if j == i:
        raise ValueError("Invalid CBF line: expected integer token.")
    return sign * int(s[i:j]), j


def _float(s: str, i: int):
    n = len(s)
    while i < n and s[i] in _SPACE:
        i += 1
    if i >= n:
        raise ValueError("Invalid CBF line: expected floating-point token.")
    mt = _FLOAT.match(s, i)
    if not mt:
        raise ValueError("Invalid CBF line: expected floating-point token.")
    return float(mt.group(0)), mt.end()


def _group(s: str):
    i, n = 0, len(s)
    while i < n and s[i] in _SPACE:
        i += 1
    if i >= n:
        raise ValueError("Invalid CBF line: expected a cone tag and length.")
    j = i
    while j < n and s[j] not in " \t":
        j += 1
    return s[i:j], _int(s, j)[0]


def _prepare_layout(con, var, nconstr, nvar):
    """_cbf_prepare_layout (src/utils/cbf_io.jl:493-634), 0-based."""
    if not con:
        raise ValueError("Invalid CBF file: missing CON section.")
    if not var:
        raise ValueError("Invalid CBF file: missing VAR section.")
    for t, _ in con:
        if t not in _SUPPORTED:
            raise ValueError(f"Unsupported constraint cone type {t}.")
    for t, _ in var:
        if t not in _SUPPORTED:
            raise ValueError(f"Unsupported variable cone type {t}.")
    m = sum(k for _, k in con)
    n = sum(k for _, k in var)
    if nconstr not in (-1, m):
        raise ValueError(f"CBF CON size mismatch: declared nconstr={nconstr} but group sum is {m}.")
    if nvar not in (-1, n):
        raise ValueError(f"CBF VAR size mismatch: declared nvar={nvar} but group sum is {n}.")
    n_eq = sum(k for t, k in con if t == "L=")
    n_ineq = sum(k for t, k in con if t in ("L+", "L-"))
    soc_lens = [k for t, k in con if t == "Q"]
    row_new = np.full(m, -1, dtype=np.int64)
    a_sign = np.ones(m)
    b_sign = -np.ones(m)
    ptr = {"L=": 0, "ineq": n_eq, "Q": n_eq + n_ineq}
    r = 0
    for t, k in con:
        if t != "F":
            key = "ineq" if t in ("L+", "L-") else t
            row_new[r:r + k] = np.arange(ptr[key], ptr[key] + k)
            ptr[key] += k
            if t == "L-":
                a_sign[r:r + k] = -1.0
                b_sign[r:r + k] = 1.0
        r += k
    n_soc_vars = sum(k for t, k in var if t == "Q")
    n_lin = n - n_soc_vars
    col_new = np.zeros(n, dtype=np.int64)
    l = np.empty(n)
    u = np.empty(n)
    var_idx = [n_lin + 1]
    lp, sq, c0 = 0, n_lin, 0
    for t, k in var:
        if t == "Q":
            col_new[c0:c0 + k] = np.arange(sq, sq + k)
            l[sq:sq + k] = -np.inf
            u[sq:sq + k] = np.inf
            sq += k
            var_idx.append(sq + 1)
        else:
            col_new[c0:c0 + k] = np.arange(lp, lp + k)
            l[lp:lp + k] = 0.0 if t in ("L+", "L=") else -np.inf
            u[lp:lp + k] = 0.0 if t in ("L-", "L=") else np.inf
            lp += k
        c0 += k
    con_idx = [n_eq + n_ineq + 1]
    for k in soc_lens:
        con_idx.append(con_idx[-1] + k)
    return dict(m=m, n=n, rows=n_eq + n_ineq + sum(soc_lens), n_eq=n_eq, n_ineq=n_ineq, row_new=row_new,
                a_sign=a_sign, b_sign=b_sign, col_new=col_new, l=l, u=u, con_idx=con_idx, var_idx=var_idx)


def _sum_duplicates_in_order(rows, cols, vals, shape):
    """sparse!(I, J, V) + dropzeros!: duplicates summed in input order."""
    order = np.lexsort((cols, rows))  # stable: input order within a (row, col)
    r, c, v = rows[order], cols[order], vals[order]
    if len(v):
        new = np.ones(len(v), dtype=bool)
        new[1:] = (r[1:] != r[:-1]) | (c[1:] != c[:-1])
        starts = np.flatnonzero(new)
        sums = v[starts].copy()
        ends = np.append(starts[1:], len(v))
        for g in np.flatnonzero(ends - starts > 1):
            s = v[starts[g]]
            for k in range(starts[g] + 1, ends[g]):
                s = s + v[k]
            sums[g] = s
        keep = sums != 0.0
        r, c, v = r[starts][keep], c[starts][keep], sums[keep]
    indptr = np.zeros(shape[0] + 1, dtype=np.int64)
    np.add.at(indptr, r + 1, 1)
    return sp.csr_matrix((v, c.astype(np.int32), np.cumsum(indptr).astype(np.int32)), shape=shape)


def read_cbf_py(filename: str):
    """The Python restatement of the reference's reader; same return values
    as read_cbf."""
    _check_extension(filename)
    with open(filename, "r", newline="") as f:
        lines = _Lines(f.read())
    con, var = [], []
    nconstr = nvar = -1
    sense, objoffset = "min", 0.0
    ready = False
    blocks = {"ACOORD": [], "BCOORD": [], "OBJACOORD": []}

    def need(what, after=True):
        s = lines.raw()
        if s is None:
            raise ValueError(f"Invalid CBF file: unexpected EOF {'after' if after else 'inside'} {what}.")
        return s

    while True:
        key = lines.data()
        if key is None:
            break
        if key in ("CON", "VAR"):
            head = need(key)
            total, i = _int(head, 0)
            ng, _ = _int(head, i)
            grp = [_group(need(key, after=False)) for _ in range(max(ng, 0))]
            if key == "CON":
                con, nconstr = grp, total
            else:
                var, nvar = grp, total
            ready = ready or (bool(con) and bool(var))
        elif key in blocks:
            k, _ = _int(need(key), 0)
            rows = [need(key, after=False) for _ in range(max(k, 0))]
            ents = []
            for s in rows:
                a, i = _int(s, 0)
                if key == "ACOORD":
                    b, i = _int(s, i)
                    v, _ = _float(s, i)
                    ents.append((a, b, v))
                else:
                    v, _ = _float(s, i)
                    ents.append((a, v))
            blocks[key].append((ready, ents))
        elif key == "OBJBCOORD":
            objoffset, _ = _float(need(key), 0)
        elif key in ("OBJSENSE", "SENSE"):
            raw = need("objective sense section")
            t = raw.strip().lower()
            if t in ("min", "minimize", "minimise"):
                sense = "min"
            elif t in ("max", "maximize", "maximise"):
                sense = "max"
            else:
                raise ValueError(f"Unsupported CBF objective sense: \"{raw}\".")
        elif key in ("DCOORD", "HCOORD", "hCOORD", "PSDCON", "FCOORD", "OBJFCOORD", "PSDVAR", "INT"):
            k, _ = _int(need("section header"), 0)
            if k != 0:
                if key in ("DCOORD", "HCOORD", "hCOORD", "PSDCON"):
                    raise ValueError("PSD constraints are not supported.")
                if key in ("FCOORD", "OBJFCOORD", "PSDVAR"):
                    raise ValueError("Matrix variables are not supported.")
                raise ValueError("Integer variables are not supported.")
    L = _prepare_layout(con, var, nconstr, nvar)

    def ordered(bl):
        return [e for r, e in bl if r] + [e for r, e in bl if not r]

    c = np.zeros(L["n"])
    for ents in ordered(blocks["OBJACOORD"]):
        for j, v in ents:
            if not 0 <= j < L["n"]:
                raise ValueError("Invalid CBF file: OBJACOORD index out of range.")
            c[L["col_new"][j]] = v
    rhs = np.zeros(L["rows"])
    for ents in ordered(blocks["BCOORD"]):
        for i, v in ents:
            if not 0 <= i < L["m"]:
                raise ValueError("Invalid CBF file: BCOORD index out of range.")
            if L["row_new"][i] >= 0:
                rhs[L["row_new"][i]] = L["b_sign"][i] * v
    ents = [e for blk in ordered(blocks["ACOORD"]) for e in blk]
    ac = np.array(ents, dtype=object).reshape(-1, 3) if ents else np.zeros((0, 3), dtype=object)
    ri = ac[:, 0].astype(np.int64)
    ci = ac[:, 1].astype(np.int64)
    vals = ac[:, 2].astype(np.float64)
    if len(ri) and (ri.min() < 0 or ri.max() >= L["m"] or ci.min() < 0 or ci.max() >= L["n"]):
        raise ValueError("Invalid CBF file: ACOORD index out of range.")
    rn = L["row_new"][ri]
    av = L["a_sign"][ri] * vals
    keep = (rn >= 0) & (av != 0.0)
    A = _sum_duplicates_in_order(rn[keep], L["col_new"][ci[keep]], av[keep], (L["rows"], L["n"]))
    if sense == "max":
        c = -c
        objoffset = -objoffset
    Q = sp.csr_matrix((L["n"], L["n"]))
    return (Q, c, A, rhs, np.array(L["con_idx"], dtype=np.int64), L["n_eq"], L["n_ineq"], L["l"], L["u"],
            np.array(L["var_idx"], dtype=np.int64), float(objoffset))


def write_cbf(filename: str, con, var, acoord, bcoord=(), objacoord=(), objoffset: float = 0.0,
              sense: str = "min"):
    """Write a conic-linear CBF file: `con` / `var` are (cone, size) groups,
    `acoord` (row, col, value), `bcoord` (row, value) and `objacoord`
    (col, value) use 0-based indices; the constraint is A x + b in cone."""
    m = sum(k for _, k in con)
    n = sum(k for _, k in var)
    out = ["VER", "3", "", "OBJSENSE", sense.upper(), ""]
    out += ["VAR", f"{n} {len(var)}"] + [f"{t} {k}" for t, k in var] + [""]
    out += ["CON", f"{m} {len(con)}"] + [f"{t} {k}" for t, k in con] + [""]
    if len(objacoord):
        out += ["OBJACOORD", str(len(objacoord))] + [f"{int(j)} {float(v)!r}" for j, v in objacoord] + [""]
    if objoffset:
        out += ["OBJBCOORD", repr(float(objoffset)), ""]
    if len(acoord):
        out += ["ACOORD", str(len(acoord))] + [f"{int(i)} {int(j)} {float(v)!r}" for i, j, v in acoord] + [""]
    if len(bcoord):
        out += ["BCOORD", str(len(bcoord))] + [f"{int(i)} {float(v)!r}" for i, v in bcoord] + [""]
    with open(filename, "w") as f:
        f.write("\n".join(out) + "\n")

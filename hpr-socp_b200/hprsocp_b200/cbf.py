"""CBF (Conic Benchmark Format) reader for SOCP instances.

``read_cbf`` returns the inputs of ``build_from_SOCP_data`` exactly as the
reference's reader does (read_cbf / _cbf_prepare_layout,
src/utils/cbf_io.jl:1438-1455 and 493-634):

* constraint rows are reordered as equalities (L=), inequalities (L+ and L-,
  the latter negated so every inequality reads ``A x >= rhs``) and second
  order cone rows (Q); free rows (F) are dropped;
* CBF states ``A x + b`` in the cone, so ``rhs = -b`` on L=, L+ and Q rows
  and ``rhs = b`` on (negated) L- rows;
* variables are reordered as linear (L+ >= 0, L- <= 0, L= fixed at 0,
  F free) followed by cone variables (Q);
* ``OBJSENSE MAX`` (or ``SENSE max``) negates c and the offset;
* cone index vectors are 1-based, as the builder's default expects.

Only the conic-linear subset is accepted: PSD blocks, matrix variables,
integer variables and other cones (for example QR) raise ValueError with
the reference's messages.  Duplicate (row, col) entries are summed.
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp

from .model import SOCPModel, build_from_SOCP_data

_SUPPORTED = ("L+", "L-", "L=", "Q", "F")


def _data_lines(text: str):
    out = []
    for raw in text.splitlines():
        s = raw.strip()
        if s and not s.startswith("#"):
            out.append(s)
    return out


def _block(lines, i, k, cols, dtype=float):
    """k lines of `cols` numbers starting at lines[i] as a (k, cols) array."""
    if k == 0:
        return np.zeros((0, cols))
    if i + k > len(lines):
        raise ValueError("Invalid CBF file: truncated coordinate block.")
    arr = np.array(" ".join(lines[i:i + k]).split(), dtype=dtype)
    if arr.size != k * cols:
        raise ValueError("Invalid CBF file: malformed coordinate block.")
    return arr.reshape(k, cols)


def _sense(token: str) -> str:
    t = token.strip().lower()
    if t in ("min", "minimize"):
        return "min"
    if t in ("max", "maximize"):
        return "max"
    raise ValueError(f"Unsupported objective sense {token}.")


def read_cbf_raw(filename: str) -> dict:
    """The sections of a CBF file (0-based indices, as stored)."""
    with open(filename, "r") as f:
        lines = _data_lines(f.read())
    d = {"con": [], "var": [], "nconstr": -1, "nvar": -1, "objacoord": np.zeros((0, 2)),
         "acoord": np.zeros((0, 3)), "bcoord": np.zeros((0, 2)), "objoffset": 0.0, "sense": "min",
         "psd": False, "matvar": False, "int": False}
    i = 0
    while i < len(lines):
        key = lines[i]
        if key in ("CON", "VAR"):
            total, groups = (int(v) for v in lines[i + 1].split()[:2])
            grp = []
            for j in range(groups):
                parts = lines[i + 2 + j].split()
                grp.append((parts[0], int(parts[1])))
            d[key.lower()] = grp
            d["nconstr" if key == "CON" else "nvar"] = total
            i += 2 + groups
        elif key in ("ACOORD", "BCOORD", "OBJACOORD"):
            k = int(lines[i + 1].split()[0])
            cols = 3 if key == "ACOORD" else 2
            d[key.lower()] = _block(lines, i + 2, k, cols)
            i += 2 + k
        elif key == "OBJBCOORD":
            d["objoffset"] = float(lines[i + 1].split()[0])
            i += 2
        elif key in ("OBJSENSE", "SENSE"):
            d["sense"] = _sense(lines[i + 1])
            i += 2
        elif key in ("PSDCON", "DCOORD", "HCOORD", "hCOORD"):
            d["psd"] = True
            k = int(lines[i + 1].split()[0])
            i += 2 + k
        elif key in ("PSDVAR", "FCOORD", "OBJFCOORD"):
            d["matvar"] = True
            k = int(lines[i + 1].split()[0])
            i += 2 + k
        elif key == "INT":
            k = int(lines[i + 1].split()[0])
            d["int"] = k > 0
            i += 2 + k
        else:
            i += 1  # VER, POWCONES, ... and their values: nothing to keep
    return d


def read_cbf(filename: str):
    """(Q, c, A, rhs, SOC_con_idx, number_eq, number_ineq, l, u, SOC_var_idx,
    obj_constant) in the builder's layout (see the module docstring)."""
    if not (filename.endswith(".cbf") or filename.endswith(".CBF")):
        raise ValueError("Unsupported file format. Please provide a .cbf file.")
    d = read_cbf_raw(filename)
    if d["psd"]:
        raise ValueError("PSD constraints are not supported.")
    if d["matvar"]:
        raise ValueError("Matrix variables are not supported.")
    if d["int"]:
        raise ValueError("Integer variables are not supported.")
    con, var = d["con"], d["var"]
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
    if d["nconstr"] not in (-1, m):
        raise ValueError(f"CBF CON size mismatch: declared nconstr={d['nconstr']} but group sum is {m}.")
    if d["nvar"] not in (-1, n):
        raise ValueError(f"CBF VAR size mismatch: declared nvar={d['nvar']} but group sum is {n}.")

    # rows: equalities, inequalities (L- negated), cone rows; F rows dropped
    n_eq = sum(k for t, k in con if t == "L=")
    n_ineq = sum(k for t, k in con if t in ("L+", "L-"))
    row_new = np.full(m, -1, dtype=np.int64)
    a_sign = np.ones(m)
    b_sign = -np.ones(m)
    nxt = {"L=": 0, "ineq": n_eq, "Q": n_eq + n_ineq}
    soc_con_lens = []
    r = 0
    for t, k in con:
        if t != "F":
            key = "ineq" if t in ("L+", "L-") else t
            row_new[r:r + k] = np.arange(nxt[key], nxt[key] + k)
            nxt[key] += k
            if t == "L-":
                a_sign[r:r + k] = -1.0
                b_sign[r:r + k] = 1.0
        if t == "Q":
            soc_con_lens.append(k)
        r += k
    rows_total = n_eq + n_ineq + sum(soc_con_lens)

    # columns: linear blocks first, then cone blocks
    n_soc_vars = sum(k for t, k in var if t == "Q")
    n_lin = n - n_soc_vars
    col_new = np.zeros(n, dtype=np.int64)
    l = np.empty(n)
    u = np.empty(n)
    soc_var_idx = [n_lin + 1]
    lp, sp_ = 0, n_lin
    c0 = 0
    for t, k in var:
        if t == "Q":
            col_new[c0:c0 + k] = np.arange(sp_, sp_ + k)
            l[sp_:sp_ + k] = -np.inf
            u[sp_:sp_ + k] = np.inf
            sp_ += k
            soc_var_idx.append(sp_ + 1)
        else:
            col_new[c0:c0 + k] = np.arange(lp, lp + k)
            l[lp:lp + k] = 0.0 if t in ("L+", "L=") else -np.inf
            u[lp:lp + k] = 0.0 if t in ("L-", "L=") else np.inf
            lp += k
        c0 += k

    ac = d["acoord"]
    ri = ac[:, 0].astype(np.int64)
    ci = ac[:, 1].astype(np.int64)
    if ac.shape[0] and (ri.min() < 0 or ri.max() >= m or ci.min() < 0 or ci.max() >= n):
        raise ValueError("Invalid CBF file: ACOORD index out of range.")
    keep = row_new[ri] >= 0
    A = sp.csr_matrix((ac[keep, 2] * a_sign[ri[keep]], (row_new[ri[keep]], col_new[ci[keep]])),
                      shape=(rows_total, n))
    A.sum_duplicates()
    b = np.zeros(m)
    bc = d["bcoord"]
    if bc.shape[0]:
        np.add.at(b, bc[:, 0].astype(np.int64), bc[:, 1])
    rhs = np.zeros(rows_total)
    kept = row_new >= 0
    rhs[row_new[kept]] = b_sign[kept] * b[kept]
    c = np.zeros(n)
    oc = d["objacoord"]
    if oc.shape[0]:
        np.add.at(c, col_new[oc[:, 0].astype(np.int64)], oc[:, 1])
    obj_constant = float(d["objoffset"])
    if d["sense"] == "max":
        c = -c
        obj_constant = -obj_constant
    soc_con_idx = [n_eq + n_ineq + 1]
    for k in soc_con_lens:
        soc_con_idx.append(soc_con_idx[-1] + k)
    Q = sp.csr_matrix((n, n))
    return Q, c, A, rhs, soc_con_idx, n_eq, n_ineq, l, u, soc_var_idx, obj_constant


def read_cbf_model(filename: str, verbose: bool = False) -> SOCPModel:
    """read_cbf followed by build_from_SOCP_data (1-based cone indices)."""
    Q, c, A, rhs, con, n_eq, n_ineq, l, u, var, const = read_cbf(filename)
    return build_from_SOCP_data(Q, c, A, rhs, con, n_eq, n_ineq, l, u, var, obj_constant=const, verbose=verbose)


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

"""Two-sided linear rows: the MOI row mapping of the reference, and its
merge back into single rows.

The reference's MOI wrapper turns an ``Interval`` constraint l <= a'x <= u
(l < u) into two inequality rows, a'x >= l and -a'x >= -u, and a
``LessThan`` row into a negated >= row (_moi_add_scalar_affine_rows!,
src/MOI_wrapper.jl:492-526).  The library takes two-sided rows
AL <= Ax <= AU natively, so each such pair can be one row: fewer rows, half
the pair's nonzeros in A and A', and fewer bytes in every iteration.

* ``merge_interval_rows`` finds the pairs in a built model (a >= row and a
  >= row with exactly the negated coefficients) and merges each into one
  two-sided row; it returns the merged model and a ``RowMap``.
* ``expand_interval_duals`` maps the merged model's y back to the rows the
  caller built: a merged row's y >= 0 means its lower bound is active, so
  the pair's duals are max(y, 0) and max(-y, 0), and A'y is unchanged.
* ``split_interval_rows`` is the mapping itself (what the MOI wrapper
  builds from a two-sided model), for tests and comparisons.
"""
from __future__ import annotations

import dataclasses
from dataclasses import dataclass

import numpy as np
import scipy.sparse as sp

from .model import SOCPModel


@dataclass
class RowMap:
    """How the rows of a merged model relate to the rows of the original."""

    m_orig: int
    kept: np.ndarray     # original index of every merged-model row
    lower: np.ndarray    # original rows merged as the lower bound (a'x >= l)
    upper: np.ndarray    # their partners (-a'x >= -u), dropped
    merged: np.ndarray   # merged-model index of each pair


def _with_rows(model: SOCPModel, A: sp.csr_matrix, AL, AU, n_lin: int) -> SOCPModel:
    shift = n_lin - model.number_linear_con
    con = np.asarray(model.SOC_con_idx, dtype=np.int64) + shift
    return dataclasses.replace(model, A=A, AL=np.asarray(AL, dtype=np.float64), AU=np.asarray(AU, dtype=np.float64),
                               SOC_con_idx=con, number_linear_con=n_lin, AT=None, _keep=[])


def merge_interval_rows(model: SOCPModel):
    """(merged model, RowMap): every pair of linear >= rows whose
    coefficients are exact negatives of each other, with -AL[j] >= AL[i],
    becomes the single row AL[i] <= a_i'x <= -AL[j]."""
    A = model.A.tocsr()
    AL, AU = model.AL, model.AU
    nl = int(model.number_linear_con)
    m = A.shape[0]
    cand = [i for i in range(nl) if np.isinf(AU[i]) and AU[i] > 0 and np.isfinite(AL[i])]
    rows = {}
    for i in cand:
        s, e = A.indptr[i], A.indptr[i + 1]
        rows.setdefault((A.indices[s:e].tobytes(), A.data[s:e].tobytes()), []).append(i)
    used = np.zeros(m, dtype=bool)
    partner = {}
    for i in cand:
        if used[i]:
            continue
        s, e = A.indptr[i], A.indptr[i + 1]
        if e == s:
            continue
        for j in rows.get((A.indices[s:e].tobytes(), (-A.data[s:e]).tobytes()), ()):
            if j != i and not used[j] and -AL[j] >= AL[i]:
                used[i] = used[j] = True
                partner[i] = j
                break
    drop = np.zeros(m, dtype=bool)
    for j in partner.values():
        drop[j] = True
    kept = np.flatnonzero(~drop)
    new_of = np.full(m, -1, dtype=np.int64)
    new_of[kept] = np.arange(len(kept))
    AL2, AU2 = AL.copy(), AU.copy()
    for i, j in partner.items():
        AU2[i] = -AL[j]
    merged = _with_rows(model, A[kept], AL2[kept], AU2[kept], nl - len(partner))
    lower = np.array(sorted(partner), dtype=np.int64)
    upper = np.array([partner[i] for i in lower], dtype=np.int64)
    return merged, RowMap(m_orig=m, kept=kept, lower=lower, upper=upper, merged=new_of[lower])


def expand_interval_duals(y: np.ndarray, rmap: RowMap) -> np.ndarray:
    """y of the merged model in the original model's rows."""
    y = np.asarray(y, dtype=np.float64)
    out = np.zeros(rmap.m_orig)
    out[rmap.kept] = y
    ym = y[rmap.merged]
    out[rmap.lower] = np.maximum(ym, 0.0)
    out[rmap.upper] = np.maximum(-ym, 0.0)
    return out


def split_interval_rows(model: SOCPModel) -> SOCPModel:
    """The MOI wrapper's rows for a model with two-sided linear rows:
    equalities first, then per row a >= l (when l is finite) and -a >= -u
    (when u is finite), in row order; cone rows unchanged."""
    A = model.A.tocsr()
    AL, AU = model.AL, model.AU
    nl = int(model.number_linear_con)
    eq = [i for i in range(nl) if AL[i] == AU[i]]
    blocks, lo, hi = [A[eq]], [AL[eq]], [AU[eq]]
    rows, signs, rhs = [], [], []
    for i in range(nl):
        if AL[i] == AU[i]:
            continue
        if np.isfinite(AL[i]):
            rows.append(i)
            signs.append(1.0)
            rhs.append(AL[i])
        if np.isfinite(AU[i]):
            rows.append(i)
            signs.append(-1.0)
            rhs.append(-AU[i])
    if rows:
        blocks.append(sp.diags(np.array(signs)) @ A[rows])
        lo.append(np.array(rhs))
        hi.append(np.full(len(rows), np.inf))
    blocks.append(A[nl:])
    lo.append(AL[nl:])
    hi.append(AU[nl:])
    A2 = sp.vstack(blocks, format="csr")
    return _with_rows(model, A2, np.concatenate(lo), np.concatenate(hi), len(eq) + len(rows))

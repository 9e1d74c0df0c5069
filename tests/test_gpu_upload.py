"""Device-side ingest of the problem (hpr_upload): A' formed on the device,
1-based indices, rows with unsorted columns and malformed input.

The reference builds its GPU matrices from a validated SparseMatrixCSC
(src/algorithm.jl:2318-2352, src/utils/builders.jl:24-108); every accepted
variant of the same matrix must lead to bit-identical iterates.
"""
import ctypes as C
import functools

import numpy as np
import pytest
import scipy.sparse as sp

from hprsocp_b200 import Context, HPRSOCP_parameters, _abi, instances
from helpers import stress_model

pytestmark = pytest.mark.gpu

VECS = ["x", "y", "z_bar", "y_bar", "s"]


@pytest.fixture(scope="module")
def model():
    return stress_model(5)


def _run(ctx, k=150):
    info = ctx.scale(HPRSOCP_parameters(verbose=False))
    lam = ctx.power_A() * 1.05
    ctx.set_sigma_lambda(info["norm_b"] / info["norm_c"], lam, 0.0)
    ctx.set_inner(0)
    ctx.iterate(k, True)
    return {v: ctx.get(v) for v in VECS}


def _with_A(model, rp, ci, v, base=0):
    """The model's problem struct with A replaced (arrays kept on the struct)."""
    prob = model.to_c()
    keep = [np.ascontiguousarray(rp, dtype=np.int32), np.ascontiguousarray(ci, dtype=np.int32),
            np.ascontiguousarray(v, dtype=np.float64)]
    prob.A.rowptr, prob.A.colind, prob.A.values = _abi.iptr(keep[0]), _abi.iptr(keep[1]), _abi.dptr(keep[2])
    prob.A.nnz = len(keep[1])
    prob._keep_A = keep
    if base == 1:
        con = np.ascontiguousarray(np.asarray(model.SOC_con_idx, dtype=np.int64) + 1)
        var = np.ascontiguousarray(np.asarray(model.SOC_var_idx, dtype=np.int64) + 1)
        prob.soc_con_idx, prob.soc_var_idx = _abi.lptr(con), _abi.lptr(var)
        prob._keep_idx = [con, var]
        prob.index_base = 1
    return prob


def test_device_transpose_is_exact(model):
    ctx = Context(model)
    AT = sp.csr_matrix(model.A.T)
    AT.sort_indices()
    assert np.array_equal(ctx.get("AT_values"), AT.data)
    ref = _run(Context(model, with_transpose=True))
    got = _run(ctx)
    for v in VECS:
        assert np.array_equal(got[v], ref[v]), v


def test_one_based_indices(model):
    A = model.A
    ref = _run(Context(model))
    prob = _with_A(model, A.indptr + 1, A.indices + 1, A.data, base=1)
    got = _run(Context(model, problem=prob))
    for v in VECS:
        assert np.array_equal(got[v], ref[v]), v


def test_unsorted_rows_are_ordered(model):
    A = model.A
    rng = np.random.default_rng(3)
    ci, v = A.indices.copy(), A.data.copy()
    for r in range(A.shape[0]):
        a, b = A.indptr[r], A.indptr[r + 1]
        p = rng.permutation(b - a)
        ci[a:b], v[a:b] = ci[a:b][p], v[a:b][p]
    ref = _run(Context(model))
    got = _run(Context(model, problem=_with_A(model, A.indptr, ci, v)))
    for k in VECS:
        assert np.array_equal(got[k], ref[k]), k


@pytest.mark.parametrize("defect, message", [
    ("column", "column index out of range"),
    ("negative", "column index out of range"),
    ("nan", "non-finite value"),
    ("inf", "non-finite value"),
    ("rowptr", "rowptr decreases"),
    ("span", "rowptr does not span nnz"),
])
def test_malformed_matrix_is_rejected(defect, message):
    model = instances.config0(0)
    A = model.A
    rp, ci, v = A.indptr.copy(), A.indices.copy(), A.data.copy()
    k = len(ci) // 2
    if defect == "column":
        ci[k] = A.shape[1]
    elif defect == "negative":
        ci[k] = -1
    elif defect == "nan":
        v[k] = np.nan
    elif defect == "inf":
        v[k] = -np.inf
    elif defect == "rowptr":
        r = np.searchsorted(rp, k)
        rp[r] = rp[r + 1] + 1
    elif defect == "span":
        rp[-1] -= 1
    with pytest.raises(_abi.HPRError, match=message):
        Context(model, problem=_with_A(model, rp, ci, v))


@functools.lru_cache(maxsize=None)
def _vector_case(size):
    return instances.config0(0) if size == "small" else instances.config1(1, scale=0.3)


@pytest.mark.parametrize("field, value, message", [
    ("c", np.inf, "c has non-finite entries"),
    ("l", np.nan, "NaN in bounds"),
    ("AU", np.nan, "NaN in bounds"),
    ("soc_rhs", np.inf, "soc_rhs has non-finite entries"),
])
@pytest.mark.parametrize("size", ["small", "large"])
def test_bad_problem_vector_is_rejected(field, value, message, size):
    """c, the bounds and soc_rhs are checked while they are copied to the
    device: a small array on the way to a plain copy, a large one (above the
    4 MB staging threshold) chunk by chunk in the pinned staging buffers,
    with the bad value in a late chunk.  Infinite bounds stay allowed."""
    import dataclasses
    model = _vector_case(size)
    arr = np.array(getattr(model, field), dtype=np.float64)
    arr[len(arr) - 3] = value
    bad = dataclasses.replace(model, **{field: arr})
    with pytest.raises(_abi.HPRError, match=message):
        Context(bad)
    if field == "l":
        arr[len(arr) - 3] = -np.inf  # an infinite bound is not an error
        with Context(dataclasses.replace(model, l=arr)):
            pass

"""Two-sided rows (hprsocp_b200/rows.py): the reference's MOI row mapping
(_moi_add_scalar_affine_rows!, src/MOI_wrapper.jl:492-526) and its merge
back into single rows."""
import numpy as np
import pytest
import scipy.sparse as sp

from hprsocp_b200 import HPRSOCP_parameters, instances
from hprsocp_b200.model import build_from_SOCP_data
from hprsocp_b200.rows import expand_interval_duals, merge_interval_rows, split_interval_rows


def _same_model(a, b):
    assert a.A.shape == b.A.shape
    assert np.array_equal(a.A.indptr, b.A.indptr) and np.array_equal(a.A.indices, b.A.indices)
    assert np.array_equal(a.A.data.view(np.uint64), b.A.data.view(np.uint64))
    assert np.array_equal(a.AL, b.AL) and np.array_equal(a.AU, b.AU)
    assert a.number_linear_con == b.number_linear_con
    assert np.array_equal(a.SOC_con_idx, b.SOC_con_idx)
    assert np.array_equal(a.soc_rhs, b.soc_rhs)


def test_split_then_merge_is_the_original_model():
    model = instances.config0(0)  # 1000 two-sided rows, 25 constraint cones
    split = split_interval_rows(model)
    assert split.A.shape[0] == model.A.shape[0] + 1000
    assert np.all(np.isinf(split.AU[:split.number_linear_con]))
    merged, rmap = merge_interval_rows(split)
    _same_model(merged, model)
    assert len(rmap.lower) == 1000 and np.array_equal(rmap.upper, rmap.lower + 1)


def test_dual_expansion_keeps_A_transpose_y():
    model = instances.config0(0)
    split = split_interval_rows(model)
    merged, rmap = merge_interval_rows(split)
    rng = np.random.default_rng(3)
    y = rng.standard_normal(merged.A.shape[0])
    ys = expand_interval_duals(y, rmap)
    assert np.all(ys[rmap.lower] >= 0) and np.all(ys[rmap.upper] >= 0)
    assert np.all(np.minimum(ys[rmap.lower], ys[rmap.upper]) == 0)
    np.testing.assert_allclose(split.A.T @ ys, merged.A.T @ y, rtol=1e-12, atol=1e-12)


def test_only_matching_pairs_merge():
    # rows: x0 + x1 >= 1, -x0 - x1 >= -3 (a pair), 2 x0 >= 0.5, -x0 - x1 >= -0.5
    # (negation of row 0 but u < l: left alone), x0 - x1 = 0.25 (equality)
    A = sp.csr_matrix(np.array([[0.0, 0.0], [1.0, 1.0], [-1.0, -1.0], [2.0, 0.0]]))
    Q, c = None, np.array([1.0, 2.0])
    model = build_from_SOCP_data(Q, c, sp.vstack([sp.csr_matrix([[1.0, -1.0]]), A[1:], sp.csr_matrix([[-1.0, -1.0]])]),
                                 np.array([0.25, 1.0, -3.0, 0.5, -0.5]), [6], 1, 4, np.zeros(2), np.full(2, 10.0), [3],
                                 verbose=False)
    merged, rmap = merge_interval_rows(model)
    assert merged.A.shape[0] == 4 and merged.number_linear_con == 4
    assert list(rmap.lower) == [1] and list(rmap.upper) == [2]
    assert merged.AL[1] == 1.0 and merged.AU[1] == 3.0
    # the second negated row (u = 0.5 < l = 1) keeps its own >= form
    assert merged.AL[3] == -0.5 and np.isinf(merged.AU[3])


@pytest.mark.gpu
def test_moi_pairs_and_two_sided_rows_solve_alike():
    from hprsocp_b200 import Context
    model = instances.config0(0)
    split = split_interval_rows(model)
    merged, rmap = merge_interval_rows(split)
    p = HPRSOCP_parameters(verbose=False, stoptol=1e-6)
    with Context(model) as ctx:
        r0 = ctx.solve(p)
    with Context(split) as ctx:
        r1 = ctx.solve(p)
    with Context(merged) as ctx:
        r2 = ctx.solve(p)
    assert r0.status == r1.status == r2.status == "OPTIMAL"
    # merging restores the two-sided model exactly, so the solve is the same
    assert r2.iter == r0.iter and np.array_equal(r2.x, r0.x) and np.array_equal(r2.y, r0.y)
    # the pair form reaches the same optimum
    assert abs(r1.primal_obj - r0.primal_obj) <= 1e-5 * max(1.0, abs(r0.primal_obj))
    ys = expand_interval_duals(r0.y, rmap)
    assert ys.shape == r1.y.shape
    np.testing.assert_allclose(split.A.T @ ys, model.A.T @ r0.y, rtol=1e-10, atol=1e-10)

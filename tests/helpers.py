"""Shared helpers of the test suite: KAT loading and array comparison."""
import json
import os

import numpy as np
import scipy.sparse as sp

from hprsocp_b200 import build_from_SOCP_data

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _inf(v):
    a = np.asarray(v, dtype=np.float64)
    a[a >= 1e308] = np.inf
    a[a <= -1e308] = -np.inf
    return a


def load_kats():
    with open(os.path.join(GOLDEN, "reference_kats.json")) as f:
        return json.load(f)


def kat_model(case):
    n = len(case["c"])
    A = sp.csr_matrix(np.array(case["A"], dtype=float).reshape(-1, n)) if case["A"] else sp.csr_matrix((0, n))
    Q = None if case["Q"] is None else sp.csr_matrix(np.array(case["Q"], dtype=float))
    return build_from_SOCP_data(Q, np.array(case["c"], dtype=float), A, np.array(case["rhs"], dtype=float),
                                case["SOC_con_idx"], case["number_eq"], case["number_ineq"], _inf(case["l"]),
                                _inf(case["u"]), case["SOC_var_idx"], verbose=False)


def rel_err(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    if a.size == 0:
        return 0.0
    return float(np.max(np.abs(a - b)) / max(1.0, float(np.max(np.abs(b)))))


def stress_model(seed=5, with_long_rows=True):
    """Small instance that exercises every engine path: linear rows longer
    than one tile (multi-CTA row slices), small cones packed per tile, cones
    larger than kSmallConeMax and kRowCap (multi-CTA cone slices), a cone
    containing a long row, and empty rows."""
    from hprsocp_b200 import instances
    rng = np.random.default_rng(seed)
    var_dims = [3] * 400 + [50] * 40 + [300] * 3 + [2500] * 2
    n_box = 8000
    n = n_box + int(np.sum(var_dims))
    m1 = 6000
    len1 = np.clip(np.rint(np.exp(np.log(10.0) + 1.1 * rng.standard_normal(m1))), 0, 1500).astype(np.int64)
    if with_long_rows:
        len1[[7, 1000, 4321]] = [3000, 5000, 2049]
    len1[[11, 12]] = 0
    con_dims = [3] * 300 + [40] * 20 + [200] * 3 + [1500]
    m2 = int(np.sum(con_dims))
    len2 = rng.integers(3, 12, size=m2)
    if with_long_rows:
        len2[m2 - 10] = 4500  # a long row inside the last (large) cone
    A1 = instances._random_rows(rng, m1, n, len1)
    A2 = instances._random_rows(rng, m2, n, len2)
    return instances._assemble(rng, A1, A2, n_box, var_dims, con_dims)


def tall_model(seed=3):
    """More constraint rows than variables (m > n), with boxed and cone
    variables and linear and cone rows: every length-m buffer is exercised
    beyond n."""
    import scipy.sparse as sp
    from hprsocp_b200 import instances
    rng = np.random.default_rng(seed)
    n, n_box = 300, 200
    var_dims = [5] * 20
    con_dims = [4] * 50 + [40] * 2
    m1 = 420
    A1 = sp.random(m1, n, density=0.03, random_state=rng, data_rvs=rng.standard_normal, format="csr")
    A2 = sp.random(int(np.sum(con_dims)), n, density=0.03, random_state=rng, data_rvs=rng.standard_normal,
                   format="csr")
    return instances._assemble(rng, A1, A2, n_box, var_dims, con_dims)


def cone_branches(bar, dual, starts):
    """Projection branch of every cone from a full iteration's outputs: 0 when
    the projection is the origin (bar block all zero), 1 when the raw point
    was inside the cone (dual block all zero: bar = raw exactly), 2 for a
    projection onto the boundary.  Variable cones: (x_bar, z_bar); constraint
    cones: (s, y_bar).  The branches set these blocks to exact zeros, so the
    test is exact."""
    starts = np.asarray(starts, dtype=np.int64)
    if len(starts) < 2 or starts[-1] <= starts[0]:
        return np.zeros(0, dtype=np.int8)
    lo, hi = int(starts[0]), int(starts[-1])
    idx = starts[:-1] - lo
    nb = np.add.reduceat(np.abs(bar[lo:hi]) > 0, idx)
    nd = np.add.reduceat(np.abs(dual[lo:hi]) > 0, idx)
    return np.where(nb == 0, 0, np.where(nd == 0, 1, 2)).astype(np.int8)


def branch_disagreements(g, o, model):
    """Cones whose projection branch differs between the CUDA path (g) and
    the oracle (o) after a full iteration: (variable cones, constraint cones)."""
    vx = np.sum(cone_branches(g.get("x_bar"), g.get("z_bar"), model.SOC_var_idx) !=
                cone_branches(o.get("x_bar"), o.get("z_bar"), model.SOC_var_idx))
    cy = np.sum(cone_branches(g.get("s"), g.get("y_bar"), model.SOC_con_idx) !=
                cone_branches(o.get("s"), o.get("y_bar"), model.SOC_con_idx))
    return int(vx), int(cy)


def edge_model(kind, seed=7):
    """Degenerate shapes of the problem data, each a bounded problem with a
    planted primal-dual point (instances._assemble):
      lp_box     linear rows and boxed variables only, no cone anywhere;
      one_cone   every variable in one cone of 300 (no boxed variable);
      cones_only no linear row: every row of A in a constraint cone;
      dim_one    cones of dimension 1 and 2 on both sides;
      sparse     empty rows and empty columns in A;
      no_rows    m = 0: boxes and cones only."""
    from hprsocp_b200.instances import _assemble
    rng = np.random.default_rng(seed)

    def rnd(m, n, d):
        return sp.random(m, n, density=d, random_state=rng, data_rvs=rng.standard_normal, format="csr")

    if kind == "lp_box":
        return _assemble(rng, rnd(150, 300, 0.03), sp.csr_matrix((0, 300)), 300, [], [])
    if kind == "one_cone":
        return _assemble(rng, rnd(100, 300, 0.03), rnd(100, 300, 0.03), 0, [300], [5] * 20)
    if kind == "cones_only":
        return _assemble(rng, sp.csr_matrix((0, 200)), rnd(120, 200, 0.04), 100, [10] * 10, [4] * 30)
    if kind == "dim_one":
        return _assemble(rng, rnd(60, 200, 0.04), rnd(30, 200, 0.04), 100, [1] * 50 + [2] * 25, [1] * 20 + [2] * 5)
    if kind == "sparse":
        A1 = rnd(120, 250, 0.02).tolil()
        A1[10:20, :] = 0.0          # empty rows
        A1[:, 200:230] = 0.0        # empty columns
        A2 = rnd(40, 250, 0.02).tolil()
        A2[:, 200:230] = 0.0
        return _assemble(rng, A1.tocsr(), A2.tocsr(), 150, [10] * 10, [4] * 10)
    if kind == "no_rows":
        return _assemble(rng, sp.csr_matrix((0, 200)), sp.csr_matrix((0, 200)), 100, [10] * 10, [])
    raise ValueError(kind)

"""CBF reader (read_cbf, src/utils/cbf_io.jl:1438-1455, 493-634): the
builder layout of the reference, round trips and the rejected inputs."""
import json
import os

import numpy as np
import pytest
import scipy.sparse as sp

from hprsocp_b200 import instances
from hprsocp_b200.cbf import read_cbf, read_cbf_model, write_cbf
from helpers import GOLDEN

S2 = np.sqrt(2.0)


def _model_cbf(path):
    """min -3x - 5y + z  s.t.  x + 2y <= 10,  3x + y <= 12,
    (0.5z + 1, 0.5z - 1, sqrt2 x, sqrt2 y) in Q^4,  x, y, z >= 0 — written
    in CBF's `A x + b in K` form."""
    write_cbf(path, con=[("L-", 2), ("Q", 4)], var=[("L+", 3)],
              acoord=[(0, 0, 1.0), (0, 1, 2.0), (1, 0, 3.0), (1, 1, 1.0), (2, 2, 0.5), (3, 2, 0.5),
                      (4, 0, S2), (5, 1, S2)],
              bcoord=[(0, -10.0), (1, -12.0), (2, 1.0), (3, -1.0)],
              objacoord=[(0, -3.0), (1, -5.0), (2, 1.0)])


def test_layout_matches_the_reference_builder_inputs(tmp_path):
    path = str(tmp_path / "model.cbf")
    _model_cbf(path)
    Q, c, A, rhs, con, n_eq, n_ineq, l, u, var, const = read_cbf(path)
    with open(os.path.join(GOLDEN, "reference_kats.json")) as f:
        kat = json.load(f)["solves"]["model_cbf"]
    assert np.allclose(A.toarray(), np.array(kat["A"]), rtol=0, atol=1e-15)
    assert np.allclose(rhs, kat["rhs"]) and np.allclose(c, kat["c"])
    assert list(con) == kat["SOC_con_idx"] and list(var) == kat["SOC_var_idx"]
    assert (n_eq, n_ineq) == (kat["number_eq"], kat["number_ineq"])
    assert np.array_equal(l, np.zeros(3)) and np.all(np.isinf(u))
    assert Q.nnz == 0 and const == 0.0


def test_model_cbf_solves_to_the_known_optimum(tmp_path):
    import sys
    sys.path.insert(0, os.path.join(os.path.dirname(GOLDEN), "..", "oracle"))
    from oracle_ctx import OracleContext
    from hprsocp_b200 import HPRSOCP_parameters
    path = str(tmp_path / "model.cbf")
    _model_cbf(path)
    model = read_cbf_model(path)
    with OracleContext(model, threads=1) as o:
        r = o.solve(HPRSOCP_parameters(verbose=False, stoptol=1e-8, max_iter=200000))
    assert r.status == "OPTIMAL"
    assert np.allclose(r.x, [1.5, 2.5, 8.5], atol=1e-4)
    assert abs(r.primal_obj + 8.5) <= 1e-4


def test_round_trip_of_a_generated_instance(tmp_path):
    """Every cone family (L=, L+, L-, F rows; L+, L-, L=, F, Q variables), a
    maximisation with an offset and duplicate entries."""
    rng = np.random.default_rng(4)
    con = [("L=", 3), ("F", 2), ("L+", 4), ("Q", 3), ("L-", 2), ("Q", 5)]
    var = [("Q", 4), ("L+", 3), ("F", 2), ("Q", 3), ("L-", 2), ("L=", 1)]
    m, n = sum(k for _, k in con), sum(k for _, k in var)
    Ad = rng.standard_normal((m, n)) * (rng.random((m, n)) < 0.4)
    ac = [(i, j, Ad[i, j]) for i, j in zip(*np.nonzero(Ad))]
    ac.append((0, 0, 0.25))  # a duplicate of (0, 0) (or a new entry): summed
    Ad[0, 0] += 0.25
    b = rng.standard_normal(m)
    cobj = rng.standard_normal(n)
    path = str(tmp_path / "gen.cbf")
    write_cbf(path, con, var, ac, [(i, b[i]) for i in range(m)], [(j, cobj[j]) for j in range(n)],
              objoffset=2.5, sense="max")
    Q, c, A, rhs, conidx, n_eq, n_ineq, l, u, varidx, const = read_cbf(path)
    # expected layout built independently
    rows = {"L=": [], "ineq": [], "Q": []}
    r = 0
    for t, k in con:
        for i in range(r, r + k):
            if t == "L=":
                rows["L="].append((Ad[i], -b[i]))
            elif t == "L+":
                rows["ineq"].append((Ad[i], -b[i]))
            elif t == "L-":
                rows["ineq"].append((-Ad[i], b[i]))
            elif t == "Q":
                rows["Q"].append((Ad[i], -b[i]))
        r += k
    allrows = rows["L="] + rows["ineq"] + rows["Q"]
    cols_lin, cols_q, j = [], [], 0
    for t, k in var:
        (cols_q if t == "Q" else cols_lin).extend(range(j, j + k))
        j += k
    perm = cols_lin + cols_q
    Aexp = np.array([a for a, _ in allrows])[:, perm]
    assert np.allclose(A.toarray(), Aexp, rtol=0, atol=1e-14)
    assert np.allclose(rhs, [v for _, v in allrows])
    assert np.allclose(c, -cobj[perm]) and const == -2.5
    assert (n_eq, n_ineq) == (3, 6)
    assert list(conidx) == [10, 13, 18] and list(varidx) == [9, 13, 16]
    assert np.array_equal(l[:8], [0, 0, 0, -np.inf, -np.inf, -np.inf, -np.inf, 0])
    assert np.array_equal(u[:8], [np.inf] * 5 + [0, 0, 0])
    model = read_cbf_model(path)
    assert model.A.shape == (m - 2, n)


@pytest.mark.parametrize("body, message", [
    ("VAR\n1 1\nL+ 1\nCON\n1 1\nQR 1\n", "Unsupported constraint cone type QR."),
    ("VAR\n1 1\nEXP 1\nCON\n1 1\nL+ 1\n", "Unsupported variable cone type EXP."),
    ("VAR\n1 1\nL+ 1\nCON\n1 1\nL+ 1\nPSDCON\n1\n2\n", "PSD constraints are not supported."),
    ("VAR\n1 1\nL+ 1\nCON\n1 1\nL+ 1\nPSDVAR\n1\n2\n", "Matrix variables are not supported."),
    ("VAR\n1 1\nL+ 1\nCON\n1 1\nL+ 1\nINT\n1\n0\n", "Integer variables are not supported."),
    ("VAR\n1 1\nL+ 1\n", "missing CON section"),
    ("VAR\n2 1\nL+ 1\nCON\n1 1\nL+ 1\n", "CBF VAR size mismatch"),
])
def test_rejected_inputs(tmp_path, body, message):
    path = str(tmp_path / "bad.cbf")
    with open(path, "w") as f:
        f.write(body)
    with pytest.raises(ValueError, match=message.replace(".", r"\.")):
        read_cbf(path)


def test_extension_is_checked(tmp_path):
    path = str(tmp_path / "x.txt")
    open(path, "w").write("VAR\n1 1\nF 1\n")
    with pytest.raises(ValueError, match="Please provide a .cbf file"):
        read_cbf(path)


@pytest.mark.gpu
def test_model_cbf_on_the_gpu(tmp_path):
    from hprsocp_b200 import HPRSOCP_parameters, optimize
    path = str(tmp_path / "model.cbf")
    _model_cbf(path)
    r = optimize(read_cbf_model(path), HPRSOCP_parameters(verbose=False, stoptol=1e-8, max_iter=200000))
    assert r.status == "OPTIMAL"
    assert np.allclose(r.x, [1.5, 2.5, 8.5], atol=1e-4)
    assert abs(r.primal_obj + 8.5) <= 1e-4

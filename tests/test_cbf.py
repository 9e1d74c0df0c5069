"""CBF reader (read_cbf, src/utils/cbf_io.jl:1438-1455, 493-634): the
builder layout of the reference, round trips and the rejected inputs."""
import json
import os
import re

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


# ---------------------------------------------------------------------------
# The library's C++ reader against the Python restatement of the reference's
# rules (read_cbf_py): identical arrays, bit for bit, on every case below.
# ---------------------------------------------------------------------------
from hprsocp_b200.cbf import read_cbf_py  # noqa: E402


def _same(a, b):
    Qa, ca, Aa, ra, cona, eqa, ina, la, ua, vara, ka = a
    Qb, cb, Ab, rb, conb, eqb, inb, lb, ub, varb, kb = b
    assert Aa.shape == Ab.shape and Qa.shape == Qb.shape and Qa.nnz == Qb.nnz == 0
    assert np.array_equal(Aa.indptr, Ab.indptr) and np.array_equal(Aa.indices, Ab.indices)
    assert np.array_equal(Aa.data.view(np.uint64), Ab.data.view(np.uint64))
    for x, y in ((ca, cb), (ra, rb), (la, lb), (ua, ub)):
        assert np.array_equal(np.asarray(x).view(np.uint64), np.asarray(y).view(np.uint64))
    assert list(cona) == list(conb) and list(vara) == list(varb)
    assert (eqa, ina) == (eqb, inb) and ka == kb


def _write(tmp_path, name, text, newline="\n"):
    path = str(tmp_path / name)
    with open(path, "w", newline="") as f:
        f.write(text.replace("\n", newline))
    return path


TRICKY = """# comment before the header
VER
3

OBJSENSE
  maximise
ACOORD
3
0 0 2.0
1 1 -1.5e-3
0 0 1.0
VAR
5 3
L+ 2
Q 2
F 1
CON
4 3
L- 1
Q 2
F 1
   # comments between sections are skipped
ACOORD
9
0 1 0.0
0 2 4.0
0 2 -4.0
1 3 1.25
1 3 2.5
1 3 -0.75
2 4 3.0
3 0 9.0
2 0 -0.0
BCOORD
4
0 1.0
1 -2.0
1 3.0
3 7.0
OBJACOORD
3
4 1.0
4 -2.0
0 0.5
OBJBCOORD
1.5
PSDCON
0
INT
0
"""


@pytest.mark.parametrize("newline", ["\n", "\r\n", "\r"])
def test_native_reader_matches_the_restatement_on_edge_rules(tmp_path, newline):
    """Duplicates (three in a row) summed in file order, zero entries and
    zero sums dropped, later BCOORD/OBJACOORD entries winning, a block read
    before CON/VAR applied after the others, F rows dropped, MAX, empty PSD
    and INT sections, comments, and every line ending."""
    path = _write(tmp_path, "tricky.cbf", TRICKY, newline)
    py = read_cbf_py(path)
    for threads in (1, 3, 8):
        _same(read_cbf(path, threads=threads), py)
    Q, c, A, rhs, con, n_eq, n_ineq, l, u, var, const = py
    # new columns: L+ vars 0, 1 and the F var 4 -> 0, 1, 2; Q vars 2, 3 -> 3, 4.
    # The (0, 0) entries come from the block read before CON/VAR: applied
    # after the later block, so A[0, 0] = -(2 + 1) on the negated L- row
    assert A.shape == (3, 5) and A[0, 0] == -3.0
    assert 3 not in A[0].indices  # 4 - 4 dropped
    assert A[1, 4] == (1.25 + 2.5) + (-0.75)
    assert A.nnz == 4  # the F row's entry and the zeros are gone
    assert rhs[1] == -3.0  # the later BCOORD entry for row 1 wins
    assert c[2] == 2.0 and c[0] == -0.5 and const == -1.5  # max: negated


def test_native_reader_handles_a_file_without_final_newline(tmp_path):
    path = _write(tmp_path, "nofinal.cbf", "VAR\n2 1\nL+ 2\nCON\n1 1\nL+ 1\nACOORD\n2\n0 0 1.0\n0 1 2.0")
    _same(read_cbf(path), read_cbf_py(path))
    assert read_cbf(path)[2].nnz == 2


def test_native_reader_is_thread_invariant_on_a_large_file(tmp_path):
    rng = np.random.default_rng(7)
    m, n, nnz = 3000, 2500, 300_000
    rows = rng.integers(0, m, nnz)
    cols = rng.integers(0, n, nnz)
    vals = np.round(rng.standard_normal(nnz), 3)
    vals[rng.random(nnz) < 0.01] = 0.0
    con = [("L=", 500), ("L-", 700), ("F", 300), ("L+", 500), ("Q", 1000)]
    var = [("L+", 1000), ("Q", 1000), ("F", 300), ("L-", 200)]
    path = str(tmp_path / "big.cbf")
    write_cbf(path, con, var, list(zip(rows, cols, vals)), [(i, 0.5 * i) for i in range(0, m, 3)],
              [(j, 1.0) for j in range(0, n, 5)], objoffset=1.0)
    ref = read_cbf(path, threads=1)
    for threads in (2, 5, 8):
        _same(read_cbf(path, threads=threads), ref)
    _same(ref, read_cbf_py(path))


@pytest.mark.parametrize("body, message", [
    ("VAR\n1 1\nL+ 1\nCON\n1 1\nL+ 1\nACOORD\n2\n0 0 1.0\n", "unexpected EOF inside ACOORD"),
    ("VAR\n1 1\nL+ 1\nCON\n1 1\nL+ 1\nACOORD\n1\n\n", "expected integer token"),
    ("VAR\n1 1\nL+ 1\nCON\n1 1\nL+ 1\nACOORD\n1\n0 0 x\n", "expected floating-point token"),
    ("VAR\n1 1\nL+ 1\nCON\n1 1\nL+ 1\nACOORD\n1\n0 3 1.0\n", "ACOORD index out of range"),
    ("VAR\n1 1\nL+ 1\nCON\n1 1\nL+ 1\nBCOORD\n1\n4 1.0\n", "BCOORD index out of range"),
    ("VAR\n1 1\nL+ 1\nCON\n1 1\nL+ 1\nOBJSENSE\nsideways\n", "Unsupported CBF objective sense"),
    ("VAR\n1 1\nL+ 1\nCON\n1 1\nL+ 1\nDCOORD\n2\n", "PSD constraints are not supported."),
    ("VAR\n1 1\nL+ 1\nCON\n", "unexpected EOF after CON"),
])
def test_native_and_restatement_reject_alike(tmp_path, body, message):
    path = _write(tmp_path, "bad.cbf", body)
    for reader in (read_cbf, read_cbf_py):
        with pytest.raises(ValueError, match=re.escape(message)):
            reader(path)

"""Dataset runner (run_dataset, src/utils/dataset.jl:4-122): the result table,
its SGM10 and solved rows, and resuming an interrupted run."""
import csv
import math
import os
import sys

import numpy as np
import pytest

from hprsocp_b200 import HPRSOCP_parameters
from hprsocp_b200.cbf import write_cbf
from hprsocp_b200.dataset import COLUMNS, run_dataset, sgm10

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
S2 = np.sqrt(2.0)


def _oracle_solve(model, params):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from oracle_ctx import OracleContext
    with OracleContext(model, threads=1) as o:
        return o.solve(params)


def _write_instances(folder):
    os.makedirs(folder, exist_ok=True)
    # min -3x - 5y + z, two linear rows, one cone of 4 (known optimum -8.5)
    write_cbf(os.path.join(folder, "a_model.cbf"), con=[("L-", 2), ("Q", 4)], var=[("L+", 3)],
              acoord=[(0, 0, 1.0), (0, 1, 2.0), (1, 0, 3.0), (1, 1, 1.0), (2, 2, 0.5), (3, 2, 0.5),
                      (4, 0, S2), (5, 1, S2)],
              bcoord=[(0, -10.0), (1, -12.0), (2, 1.0), (3, -1.0)], objacoord=[(0, -3.0), (1, -5.0), (2, 1.0)])
    # min x + y s.t. x + y >= 1, x, y >= 0 (optimum 1)
    write_cbf(os.path.join(folder, "b_lp.cbf"), con=[("L+", 1)], var=[("L+", 2)],
              acoord=[(0, 0, 1.0), (0, 1, 1.0)], bcoord=[(0, -1.0)], objacoord=[(0, 1.0), (1, 1.0)])
    with open(os.path.join(folder, "notes.txt"), "w") as f:
        f.write("not an instance\n")


def _table(path):
    with open(os.path.join(path, "HPRSOCP_result.csv"), newline="") as f:
        return list(csv.DictReader(f))


def test_sgm10():
    assert sgm10([0, 0]) == pytest.approx(0.0)
    assert sgm10([90]) == pytest.approx(90.0)
    assert sgm10([10, 30]) == pytest.approx(math.sqrt(20 * 40) - 10)


def test_table_summary_rows_and_resume(tmp_path):
    data, out = str(tmp_path / "data"), str(tmp_path / "out")
    _write_instances(data)
    p = HPRSOCP_parameters(verbose=False, stoptol=1e-6, max_iter=200000)
    rows = run_dataset(data, out, p, solve=_oracle_solve)
    assert [r["name"] for r in rows] == ["a_model.cbf", "b_lp.cbf"]
    t = _table(out)
    assert list(t[0].keys()) == COLUMNS
    assert [r["name"] for r in t] == ["a_model.cbf", "b_lp.cbf", "SGM10", "solved"]
    assert all(r["status"] == "OPTIMAL" for r in t[:2])
    assert float(t[0]["primal_obj"]) == pytest.approx(-8.5, abs=1e-4)
    assert float(t[1]["primal_obj"]) == pytest.approx(1.0, abs=1e-4)
    assert float(t[2]["iter"]) == pytest.approx(sgm10([float(r["iter"]) for r in t[:2]]))
    assert t[3]["alg_time"] == "2"
    assert os.path.getsize(os.path.join(out, "HPRSOCP_log.txt")) > 0
    # a rerun solves nothing new; a new file is solved and appended
    calls = []

    def counting(model, params):
        calls.append(model.n)
        return _oracle_solve(model, params)

    run_dataset(data, out, p, solve=counting)
    assert calls == []
    write_cbf(os.path.join(data, "c_lp.cbf"), con=[("L+", 1)], var=[("L+", 1)], acoord=[(0, 0, 1.0)],
              bcoord=[(0, -2.0)], objacoord=[(0, 1.0)])
    run_dataset(data, out, p, solve=counting)
    assert calls == [1]
    assert [r["name"] for r in _table(out)] == ["a_model.cbf", "b_lp.cbf", "c_lp.cbf", "SGM10", "solved"]


@pytest.mark.gpu
def test_sequential_and_batched_runs_agree(tmp_path):
    data = str(tmp_path / "data")
    _write_instances(data)
    p = HPRSOCP_parameters(verbose=False, stoptol=1e-6, max_iter=200000)
    seq = run_dataset(data, str(tmp_path / "seq"), p)
    bat = run_dataset(data, str(tmp_path / "bat"), p, slots=2)
    assert [r["name"] for r in seq] == [r["name"] for r in bat]
    for a, b in zip(seq, bat):
        assert a["status"] == b["status"] == "OPTIMAL"
        assert a["iter"] == b["iter"] and a["primal_obj"] == b["primal_obj"]

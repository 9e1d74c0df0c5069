"""The pins in configs/*.json describe what the seeded generators build (CPU).

The benchmark configurations leave choices open (which cones are variable
cones, the lognormal parameter, the portfolio's cone structure, ...); the
generators in hprsocp_b200.instances make them and configs/*.json records
them.  These tests keep the two in step.
"""
import json
import os

import numpy as np
import pytest

from hprsocp_b200 import instances

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _cfg(name):
    with open(os.path.join(ROOT, "configs", f"{name}.json")) as f:
        return json.load(f)


def _cone_counts(starts):
    d = np.diff(np.asarray(starts))
    vals, counts = np.unique(d, return_counts=True)
    return sorted([[int(c), int(v)] for v, c in zip(vals, counts)], key=lambda x: x[1])


def test_config0_pins():
    c = _cfg("config0")
    m = instances.config0(c["seed"])
    assert m.n == c["n"] and m.number_lu_x == c["n_box"]
    assert m.number_linear_con == c["A1"]["rows"] and m.m == c["A1"]["rows"] + c["A2"]["rows"]
    assert _cone_counts(m.SOC_var_idx) == c["variable_cones"]
    assert _cone_counts(m.SOC_con_idx) == c["constraint_cones"]
    assert np.all(m.l[:m.number_lu_x] == c["box"][0]) and np.all(m.u[:m.number_lu_x] == c["box"][1])
    assert m.Q is None and m.F is None


def test_config1_pins():
    c = _cfg("config1")
    m = instances.config1(c["seed"], scale=c["scale"])
    assert (m.n, m.m, m.A.nnz) == (c["n"], c["m"], c["nnz_A"])
    assert _cone_counts(m.SOC_var_idx) == sorted(c["variable_cones"], key=lambda x: x[1])
    assert _cone_counts(m.SOC_con_idx) == sorted(c["constraint_cones"], key=lambda x: x[1])
    assert m.number_linear_con == c["A1"]["rows"]
    rows = np.diff(m.A.indptr[: m.number_linear_con + 1])
    assert rows.max() <= 2000 and 8 <= np.median(rows) <= 12


@pytest.mark.parametrize("scale", [0.01])
def test_config2_pins(scale):
    c = _cfg("config2")
    m = instances.config2(c["seed"], scale=scale)
    assert m.n == int(round(c["n"] * scale))
    assert m.F is not None and m.F.shape[0] == 50 and m.q_diag is not None
    assert np.all(m.l == c["box"][0]) and np.all(m.u == c["box"][1])
    assert set(np.diff(m.SOC_con_idx).tolist()) == {101}


def test_config4_pins():
    c = _cfg("config4")
    stream = instances.serving_stream(c["seed"], 40)
    for model, tol, t in stream:
        assert 50 <= model.n <= 20000 and model.m == max(1, model.n // 2)
        assert tol in (1e-4, 1e-6) and t == 0.0
        dims = np.diff(model.SOC_var_idx)
        assert dims.size >= 1 and dims.min() >= 3 and dims.max() <= 64
    assert 0 < sum(m.Q is not None for m, _, _ in stream) < len(stream)

"""The CPU oracle against the reference's own known answers (CPU only)."""
import math

import numpy as np
import pytest

from kat_checks import KATS, run_kat, run_solve_kat
from oracle_ctx import OracleContext, golden, print_step


@pytest.mark.parametrize("name", sorted(KATS["kats"]))
def test_oracle_kat(name):
    run_kat(OracleContext, name)


@pytest.mark.parametrize("name", sorted(KATS["solves"]))
def test_oracle_solve_kat(name):
    run_solve_kat(OracleContext, name)


def test_print_step_schedule():
    # print_step (algorithm.jl:1906-1908): every 10 below 1000, then /10
    assert [print_step(i) for i in (0, 1, 99, 100, 999, 1000, 9999, 10000, 123456)] == \
        [10, 10, 10, 10, 10, 100, 100, 1000, 10000]


def test_golden_matches_closed_form():
    # golden (kernels.jl:6268-6305) with c = 0 minimises a x + b/x -> sqrt(b/a)
    for a, b in ((1.0, 4.0), (3.0, 1e-4), (1e-6, 10.0)):
        x = golden(a, b, 0.0, 0.0)
        assert abs(x - math.sqrt(b / a)) <= 1e-6 * math.sqrt(b / a)


def test_golden_with_quadratic_term():
    a, b, c, d = 1.0, 2.0, 0.5, 3.0
    f = lambda x: a * x + b / x + c * x * x / (1 + d * x)
    xs = np.exp(np.linspace(np.log(1e-3), np.log(1e3), 200001))
    x_grid = xs[np.argmin(f(xs))]
    x = golden(a, b, c, d)
    assert abs(x - x_grid) <= 1e-3 * x_grid

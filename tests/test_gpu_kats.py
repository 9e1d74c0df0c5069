"""The CUDA library against the reference's own known answers."""
import pytest

from kat_checks import KATS, run_kat, run_solve_kat

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def Ctx():
    from hprsocp_b200 import Context
    return Context


@pytest.mark.parametrize("name", sorted(KATS["kats"]))
def test_gpu_kat(Ctx, name):
    run_kat(Ctx, name)


@pytest.mark.parametrize("name", sorted(KATS["solves"]))
def test_gpu_solve_kat(Ctx, name):
    run_solve_kat(Ctx, name)

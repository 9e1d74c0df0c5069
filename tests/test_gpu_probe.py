"""Random-gather probe (hpr_probe_gather): runs, reports a positive rate and
rejects malformed sizes."""
import ctypes as C

import pytest

from hprsocp_b200 import _abi

pytestmark = pytest.mark.gpu


def test_probe_reports_a_rate():
    lib = _abi.load_library()
    ms, rate = C.c_double(), C.c_double()
    assert lib.hpr_probe_gather(0, 1 << 22, 1 << 20, C.byref(ms), C.byref(rate)) == _abi.HPR_OK
    assert ms.value > 0 and rate.value > 1e9


@pytest.mark.parametrize("n, nx", [(0, 1), (100, 0), (100, 200)])
def test_probe_rejects_bad_sizes(n, nx):
    lib = _abi.load_library()
    ms = C.c_double()
    assert lib.hpr_probe_gather(0, n, nx, C.byref(ms), None) == _abi.HPR_E_BAD_INPUT

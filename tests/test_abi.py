"""The C ABI library: builds, loads, exports every declared symbol (CPU)."""
import ctypes as C
import os
import re

import pytest

from hprsocp_b200 import _abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "hprsocp_b200.h")


def declared_symbols():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(hpr_[A-Za-z0-9_]+)\s*\(", text)))


def test_header_declares_the_abi():
    syms = declared_symbols()
    assert "hpr_create" in syms and "hpr_iterate" in syms and "hpr_solve" in syms
    assert set(syms) == set(_abi.PROTOTYPES), set(syms) ^ set(_abi.PROTOTYPES)


def test_library_exports_every_declared_symbol():
    lib = C.CDLL(_abi.LIB_PATH)
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing


def test_library_binds_and_reports_version():
    lib = _abi.load_library()
    assert lib.hpr_version() >= 10000
    assert lib.hpr_status_string(_abi.HPR_E_BUDGET).decode() == "HBM budget exceeded"


def test_default_params_match_reference_defaults():
    lib = _abi.load_library()
    p = _abi.hpr_params()
    lib.hpr_default_params(C.byref(p))
    # HPRSOCP_parameters() (src/structs.jl:277)
    assert p.stoptol == 1e-6 and p.sigma == -1 and p.check_iter == 150
    assert p.max_iter == 2**31 - 1 and p.time_limit == 3600.0 and p.print_frequency == -1
    assert p.use_Ruiz_scaling == 1 and p.ruiz_iterations == 10 and p.use_Pock_Chambolle_scaling == 1
    assert p.use_bc_scaling == 1 and p.bc_scaling_norm_type == 0
    assert p.soc_block_scaling_strategy == _abi.SOC_SCALE_STRATEGIES["phase_taper"]


def test_no_device_is_an_error_not_a_fallback():
    """Without a usable GPU hpr_create reports HPR_E_CUDA (there is no CPU
    path).  Skipped where a GPU is present."""
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    lib = _abi.load_library()
    h = C.c_void_p()
    assert lib.hpr_create(0, 0, C.byref(h)) == _abi.HPR_E_CUDA
    assert not h.value


def test_struct_layouts_match_the_header(tmp_path):
    """Every ctypes struct has the C struct's size and field offsets
    (compiled here from include/hprsocp_b200.h)."""
    import shutil
    import subprocess
    cxx = shutil.which("g++") or shutil.which("cc")
    if cxx is None:
        pytest.skip("no C compiler")
    structs = [_abi.hpr_csr, _abi.hpr_problem, _abi.hpr_params, _abi.hpr_residuals, _abi.hpr_results,
               _abi.hpr_scale_info, _abi.hpr_cbf_data]
    lines = ['#include <cstdio>', '#include <cstddef>', f'#include "{HEADER}"', "int main() {"]
    for st in structs:
        name = st.__name__
        lines.append(f'  std::printf("{name} size %zu\\n", sizeof({name}));')
        for field, _ in st._fields_:
            lines.append(f'  std::printf("{name} {field} %zu\\n", offsetof({name}, {field}));')
    lines.append("  return 0;\n}")
    src = tmp_path / "layout.cpp"
    src.write_text("\n".join(lines))
    exe = str(tmp_path / "layout")
    subprocess.run([cxx, "-o", exe, str(src)], check=True)
    got = {}
    for line in subprocess.run([exe], check=True, capture_output=True, text=True).stdout.splitlines():
        name, field, value = line.split()
        got[(name, field)] = int(value)
    for st in structs:
        name = st.__name__
        assert got[(name, "size")] == C.sizeof(st), name
        for field, _ in st._fields_:
            assert got[(name, field)] == getattr(st, field).offset, (name, field)

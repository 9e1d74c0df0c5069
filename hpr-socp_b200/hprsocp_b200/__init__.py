"""hprsocp_b200 — B200-native dual HPR iteration for SOCPs behind the
reference HPR-SOCP solver interface (build_from_SOCP_data / optimize)."""
from ._abi import HPRError, load_library, LIB_PATH
from .model import SOCPModel, build_from_SOCP_data
from .solver import Context, HPRSOCP_parameters, HPRSOCP_results, optimize
from .cbf import read_cbf, read_cbf_model

__all__ = [
    "HPRError", "load_library", "LIB_PATH", "SOCPModel", "build_from_SOCP_data",
    "Context", "HPRSOCP_parameters", "HPRSOCP_results", "optimize", "read_cbf", "read_cbf_model",
]

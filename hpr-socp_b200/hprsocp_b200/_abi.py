"""ctypes mirror of include/hprsocp_b200.h and the loader of the CUDA library.

The library is built in-tree (``hpr-socp_b200/lib/libhprsocp_b200.so``).
There is no CPU fallback: if the shared object is missing this module raises
ImportError-like errors on first use instead of silently degrading.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
PKG_ROOT = os.path.dirname(HERE)
LIB_PATH = os.path.join(PKG_ROOT, "lib", "libhprsocp_b200.so")

# status codes
HPR_OK = 0
HPR_E_CUDA = 1
HPR_E_BUDGET = 2
HPR_E_BAD_INPUT = 3
HPR_E_NUMERIC = 4
HPR_E_TIMEOUT = 5
HPR_E_STATE = 6
HPR_E_UNSUPPORTED = 7

HPR_Q_NONE = 0
HPR_Q_CSR = 1
HPR_Q_DIAG_LOWRANK = 2
HPR_Q_OPERATOR = 3

HPR_BC_NORM = {"l2": 0, "rms": 1, "linf": 2, "l_inf": 2, "inf": 2}

SOC_SCALE_STRATEGIES = {
    "max": 1, "rms": 2, "geom": 3, "adaptive": 4, "hybrid": 5, "ruiz_geom": 6,
    "role_split": 7, "pock_safe_role_split": 8, "size_split_role_split": 9,
    "pre_pock_size_split": 10, "pre_pock_huge_var_taper": 11,
    "pre_pock_huge_var_taper_pock_geom": 12, "pre_pock_band_split": 13,
    "pre_pock_constraint_rms": 14, "pre_pock_constraint_max": 15,
    "pre_pock_constraint_taper": 16, "small_cone_constraint_max": 17,
    "count_aware_small_cone_bias": 18, "phase_blend": 19, "phase_taper": 20,
}

HPR_PREC = {"fp64": 0, "fp32": 1, "bf16": 2}

HPR_SCHEDULE = {"auto": 0, "engine": 1, "fused": 2}

HPR_STATUS = {0: "OPTIMAL", 1: "MAX_ITER", 2: "TIME_LIMIT"}

VEC = {
    "x": 0, "x_bar": 1, "x_hat": 2, "last_x": 3, "z_bar": 4, "y": 5,
    "y_bar": 6, "last_y": 7, "s": 8, "w": 9, "w_bar": 10, "last_w": 11,
    "ATy": 12, "last_ATy": 13, "dx": 14, "dy": 15, "row_norm": 16,
    "col_norm": 17, "c": 18, "AL": 19, "AU": 20, "l": 21, "u": 22,
    "soc_rhs": 23, "A_values": 24, "AT_values": 25, "dw": 26,
}

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int32)
_lp = C.POINTER(C.c_int64)


class hpr_csr(C.Structure):
    _fields_ = [("nrows", C.c_int64), ("ncols", C.c_int64), ("nnz", C.c_int64),
                ("rowptr", _ip), ("colind", _ip), ("values", _dp)]


class hpr_problem(C.Structure):
    _fields_ = [("m", C.c_int64), ("n", C.c_int64), ("m_lin", C.c_int64),
                ("n_box", C.c_int64), ("A", hpr_csr), ("AT", hpr_csr),
                ("c", _dp), ("l", _dp), ("u", _dp), ("AL", _dp), ("AU", _dp),
                ("soc_rhs", _dp), ("soc_con_idx", _lp), ("n_soc_con_idx", C.c_int64),
                ("soc_var_idx", _lp), ("n_soc_var_idx", C.c_int64),
                ("index_base", C.c_int32), ("q_kind", C.c_int32), ("Q", hpr_csr),
                ("q_diag", _dp), ("F", hpr_csr), ("obj_constant", C.c_double)]


class hpr_params(C.Structure):
    _fields_ = [("stoptol", C.c_double), ("sigma", C.c_double), ("max_iter", C.c_int64),
                ("time_limit", C.c_double), ("check_iter", C.c_int64),
                ("print_frequency", C.c_int64), ("device_number", C.c_int32),
                ("use_Ruiz_scaling", C.c_int32), ("ruiz_iterations", C.c_int32),
                ("use_bc_scaling", C.c_int32), ("bc_scaling_norm_type", C.c_int32),
                ("use_Pock_Chambolle_scaling", C.c_int32),
                ("soc_block_scaling_strategy", C.c_int32), ("verbose", C.c_int32),
                ("initial_x", _dp), ("initial_y", _dp), ("lambda_max_A", C.c_double),
                ("lambda_max_Q", C.c_double), ("precision", C.c_int32), ("refine", C.c_int32),
                ("auto_save", C.c_int32), ("save_filename", C.c_char_p)]


class hpr_residuals(C.Structure):
    _fields_ = [("err_Rp_org_bar", C.c_double), ("err_Rp_linear_org_bar", C.c_double),
                ("err_Rp_soc_org_bar", C.c_double), ("err_Rd_org_bar", C.c_double),
                ("KKTx_and_gap_org_bar", C.c_double), ("primal_obj_bar", C.c_double),
                ("rel_gap_bar", C.c_double), ("dual_obj_bar", C.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class hpr_results(C.Structure):
    _fields_ = [("iter", C.c_int64), ("iter_4", C.c_int64), ("iter_6", C.c_int64),
                ("time", C.c_double), ("time_4", C.c_double), ("time_6", C.c_double),
                ("power_time", C.c_double), ("primal_obj", C.c_double),
                ("residuals", C.c_double), ("gap", C.c_double), ("status", C.c_int32),
                ("restarts", C.c_int32), ("sigma_final", C.c_double),
                ("lambda_max_A", C.c_double), ("lambda_max_Q", C.c_double),
                ("last", hpr_residuals), ("x", _dp), ("y", _dp), ("z", _dp), ("w", _dp)]


class hpr_scale_info(C.Structure):
    _fields_ = [("b_scale", C.c_double), ("c_scale", C.c_double), ("norm_b", C.c_double),
                ("norm_c", C.c_double), ("norm_b_org", C.c_double),
                ("norm_c_org", C.c_double), ("Q_is_diag", C.c_int32)]


class hpr_cbf_data(C.Structure):
    _fields_ = [("m", C.c_int64), ("n", C.c_int64), ("number_eq", C.c_int64),
                ("number_ineq", C.c_int64), ("A", hpr_csr), ("rhs", _dp), ("c", _dp),
                ("l", _dp), ("u", _dp), ("soc_con_idx", _lp), ("n_soc_con_idx", C.c_int64),
                ("soc_var_idx", _lp), ("n_soc_var_idx", C.c_int64), ("obj_constant", C.c_double)]


# Every entry point of include/hprsocp_b200.h with its ctypes signature.
PROTOTYPES = {
    "hpr_version": (C.c_int, []),
    "hpr_status_string": (C.c_char_p, [C.c_int]),
    "hpr_default_params": (None, [C.POINTER(hpr_params)]),
    "hpr_create": (C.c_int, [C.c_int, C.c_size_t, C.POINTER(C.c_void_p)]),
    "hpr_destroy": (C.c_int, [C.c_void_p]),
    "hpr_last_error": (C.c_char_p, [C.c_void_p]),
    "hpr_upload": (C.c_int, [C.c_void_p, C.POINTER(hpr_problem)]),
    "hpr_scale": (C.c_int, [C.c_void_p, C.POINTER(hpr_params), C.POINTER(hpr_scale_info)]),
    "hpr_power_A": (C.c_int, [C.c_void_p, C.c_int, C.c_double, _dp]),
    "hpr_power_Q": (C.c_int, [C.c_void_p, C.c_int, C.c_double, _dp]),
    "hpr_set_sigma_lambda": (C.c_int, [C.c_void_p, C.c_double, C.c_double, C.c_double]),
    "hpr_set_inner": (C.c_int, [C.c_void_p, C.c_int64]),
    "hpr_get_scalars": (C.c_int, [C.c_void_p, _dp, _dp, _dp, _lp]),
    "hpr_iterate": (C.c_int, [C.c_void_p, C.c_int64, C.c_int]),
    "hpr_compute_residuals": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(hpr_residuals)]),
    "hpr_compute_residuals_noalloc": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(hpr_residuals)]),
    "hpr_mnorm": (C.c_int, [C.c_void_p, _dp]),
    "hpr_sigma_terms": (C.c_int, [C.c_void_p, _dp, _dp, _dp, _dp]),
    "hpr_sigma_golden_diag": (C.c_int, [C.c_void_p, C.c_double, C.c_double, C.c_double,
                                        C.c_double, C.c_double, _dp]),
    "hpr_restart": (C.c_int, [C.c_void_p]),
    "hpr_get_vector": (C.c_int, [C.c_void_p, C.c_int, _dp, C.c_size_t]),
    "hpr_set_vector": (C.c_int, [C.c_void_p, C.c_int, _dp, C.c_size_t]),
    "hpr_get_solution": (C.c_int, [C.c_void_p, _dp, _dp, _dp, _dp]),
    "hpr_set_precision": (C.c_int, [C.c_void_p, C.c_int]),
    "hpr_set_q_operator": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_double]),
    "hpr_device_memory": (C.c_int, [C.c_void_p, C.POINTER(C.c_size_t), _lp]),
    "hpr_set_schedule": (C.c_int, [C.c_void_p, C.c_int]),
    "hpr_solve": (C.c_int, [C.c_void_p, C.POINTER(hpr_params), C.POINTER(hpr_results)]),
    "hpr_optimize": (C.c_int, [C.POINTER(hpr_problem), C.POINTER(hpr_params),
                               C.POINTER(hpr_results)]),
    "hpr_last_iterate_ms": (C.c_int, [C.c_void_p, _dp, _lp]),
    "hpr_iteration_bytes": (C.c_int, [C.c_void_p, _dp]),
    "hpr_serve_create": (C.c_int, [C.c_int, C.c_int, C.c_size_t, C.POINTER(C.c_void_p)]),
    "hpr_serve_submit": (C.c_int, [C.c_void_p, C.POINTER(hpr_problem), C.POINTER(hpr_params), _lp]),
    "hpr_serve_poll": (C.c_int, [C.c_void_p, C.c_int64, C.c_int, C.POINTER(hpr_results), _dp]),
    "hpr_serve_set_resident": (C.c_int, [C.c_void_p, C.c_int]),
    "hpr_serve_stats": (C.c_int, [C.c_void_p, _lp, _lp, C.POINTER(C.c_size_t)]),
    "hpr_serve_phase_times": (C.c_int, [C.c_void_p, _dp, _lp]),
    "hpr_serve_last_error": (C.c_char_p, [C.c_void_p]),
    "hpr_serve_destroy": (C.c_int, [C.c_void_p]),
    "hpr_cbf_read": (C.c_int, [C.c_char_p, C.c_int, C.POINTER(C.c_void_p)]),
    "hpr_cbf_last_error": (C.c_char_p, []),
    "hpr_cbf_data_get": (C.c_int, [C.c_void_p, C.POINTER(hpr_cbf_data)]),
    "hpr_cbf_problem": (C.c_int, [C.c_void_p, C.POINTER(hpr_problem)]),
    "hpr_cbf_free": (None, [C.c_void_p]),
}

_LIB = None


def load_library(path: str | None = None):
    """Load libhprsocp_b200.so and bind every prototype; fails loudly."""
    global _LIB
    if _LIB is not None and path is None:
        return _LIB
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise RuntimeError(
            f"CUDA library not built: {p} is missing (run `make -C hpr-socp_b200` "
            "or __graft_entry__.build()); there is no CPU fallback")
    lib = C.CDLL(p)
    for name, (res, args) in PROTOTYPES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _LIB = lib
    return lib


class HPRError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"[{code}] {msg}")
        self.code = code


def dptr(a):
    return a.ctypes.data_as(_dp) if a is not None else None


def iptr(a):
    return a.ctypes.data_as(_ip) if a is not None else None


def lptr(a):
    return a.ctypes.data_as(_lp) if a is not None else None

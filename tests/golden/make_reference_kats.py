"""Writes reference_kats.json: the known-answer cases of the reference's own
test suite (PolyU-IOR/HPR-SOCP test/runtests.jl, read as text) and of its
bundled instance data/model.cbf, re-encoded as plain data.

The reference is Julia and cannot run in this environment, so these cases are
transcribed, not generated: every entry names the runtests.jl lines it comes
from.  Indices are 1-based as in the reference (cone index vectors and CSR
coordinates below are given as dense matrices).

Run:  python tests/golden/make_reference_kats.py
"""
import json
import math
import os

S2 = math.sqrt(2.0)

KATS = {
    # runtests.jl:297-322 — SOC variable projection through the x update
    "soc_var_projection": {
        "source": "test/runtests.jl:297-322",
        "Q": [[0, 0, 0], [0, 0, 0], [0, 0, 0]], "c": [0, 0, 0], "A": [], "rhs": [],
        "SOC_con_idx": [1], "number_eq": 0, "number_ineq": 0,
        "l": [-1e308] * 3, "u": [1e308] * 3, "SOC_var_idx": [1, 4],
        "sigma": 1.0, "lambda_max_A": 0.0,
        "set": {"x": [0.0, 1.0, 0.0]},
        "expect": {"x_bar": [0.5, 0.5, 0.0], "z_bar": [0.5, -0.5, 0.0]},
    },
    # runtests.jl:324-351 — SOC constraint projection through the y update
    "soc_con_projection": {
        "source": "test/runtests.jl:324-351",
        "Q": None, "c": [0, 0, 0], "A": [[1, 0, 0], [0, 1, 0], [0, 0, 1]], "rhs": [0, 0, 0],
        "SOC_con_idx": [1, 4], "number_eq": 0, "number_ineq": 0,
        "l": [-1e308] * 3, "u": [1e308] * 3, "SOC_var_idx": [4],
        "sigma": 1.0, "lambda_max_A": 1.0,
        "set": {"x": [0.0, 1.0, 0.0]},  # x_hat = x when y = c = 0 and no bounds
        "expect": {"x_hat": [0.0, 1.0, 0.0], "s": [0.5, 0.5, 0.0], "y_bar": [0.5, -0.5, 0.0]},
    },
    # runtests.jl:353-391 — bound/cone violation 0.5 and Rp = [0.5,-0.5,0]
    "soc_violation": {
        "source": "test/runtests.jl:353-373",
        "Q": None, "c": [0, 0, 0], "A": [], "rhs": [],
        "SOC_con_idx": [1], "number_eq": 0, "number_ineq": 0,
        "l": [-1e308] * 3, "u": [1e308] * 3, "SOC_var_idx": [1, 4],
        "set": {"x_bar": [0.0, 1.0, 0.0]},
        "expect_residuals": {"bounds_violation": 0.5},
    },
    "soc_con_rp": {
        "source": "test/runtests.jl:375-391",
        "Q": None, "c": [0, 0, 0], "A": [[1, 0, 0], [0, 1, 0], [0, 0, 1]], "rhs": [0, 0, 0],
        "SOC_con_idx": [1, 4], "number_eq": 0, "number_ineq": 0,
        "l": [-1e308] * 3, "u": [1e308] * 3, "SOC_var_idx": [4],
        "set": {"x_bar": [0.0, 1.0, 0.0]},
        # Rp = [0.5,-0.5,0], |Ax| = 1, norm_b_org = 0 -> err = 0.5/(1+1)
        "expect_residuals": {"err_Rp_org_bar": 0.25, "err_Rp_soc_org_bar": 0.25, "err_Rp_linear_org_bar": 0.0},
    },
    # runtests.jl:405-433 — split primal residual, mixed rows
    "split_rp_mixed": {
        "source": "test/runtests.jl:405-433",
        "Q": None, "c": [0, 0, 0, 0], "A": [[1, 0, 0, 0], [0, 1, 0, 0], [0, 0, 1, 0], [0, 0, 0, 1]],
        "rhs": [0, 0, 0, 0], "SOC_con_idx": [2, 5], "number_eq": 0, "number_ineq": 1,
        "l": [-1e308] * 4, "u": [1e308] * 4, "SOC_var_idx": [5],
        "set": {"x_bar": [-2.0, 0.0, 1.0, 0.0]},
        # linear Rp = 2, cone Rp = [0.5,-0.5,0]; denominator 1 + max(0, 2) = 3
        "expect_residuals": {"err_Rp_linear_org_bar": 2.0 / 3.0, "err_Rp_soc_org_bar": 0.5 / 3.0,
                             "err_Rp_org_bar": 2.0 / 3.0},
    },
    # runtests.jl:435-460 — pure linear model: SOC part exactly zero
    "split_rp_linear": {
        "source": "test/runtests.jl:435-460",
        "Q": None, "c": [0, 0], "A": [[1, 0]], "rhs": [0], "SOC_con_idx": [2],
        "number_eq": 0, "number_ineq": 1, "l": [-1e308] * 2, "u": [1e308] * 2, "SOC_var_idx": [3],
        "set": {"x_bar": [-1.0, 0.0]},
        "expect_residuals": {"err_Rp_linear_org_bar": 0.5, "err_Rp_soc_org_bar": 0.0, "err_Rp_org_bar": 0.5},
    },
    # runtests.jl:462-486 — pure SOC model: linear part exactly zero
    "split_rp_soc": {
        "source": "test/runtests.jl:462-486",
        "Q": None, "c": [0, 0, 0], "A": [[1, 0, 0], [0, 1, 0], [0, 0, 1]], "rhs": [0, 0, 0],
        "SOC_con_idx": [1, 4], "number_eq": 0, "number_ineq": 0,
        "l": [-1e308] * 3, "u": [1e308] * 3, "SOC_var_idx": [4],
        "set": {"x_bar": [0.0, 1.0, 0.0]},
        "expect_residuals": {"err_Rp_linear_org_bar": 0.0, "err_Rp_soc_org_bar": 0.25, "err_Rp_org_bar": 0.25},
    },
    # runtests.jl:607-638 — dual objective includes the SOC rhs shift
    "dual_objective_rhs_shift": {
        "source": "test/runtests.jl:607-638",
        "Q": None, "c": [0, 0, 0], "A": [[0, 0, 0], [0, 0, 0], [0, 0, 0]], "rhs": [1, 0, 0],
        "SOC_con_idx": [1, 4], "number_eq": 0, "number_ineq": 0,
        "l": [-1e308] * 3, "u": [1e308] * 3, "SOC_var_idx": [4],
        "set": {"x_bar": [0, 0, 0], "z_bar": [0, 0, 0], "y_bar": [1, 0, 0], "s": [0, 0, 0]},
        "expect_residuals": {"dual_obj_bar": 1.0},
    },
    # runtests.jl:701-723 — M-norm finite and non-negative (Q = I, m = 0)
    "mnorm_q_identity": {
        "source": "test/runtests.jl:701-723",
        "Q": [[1, 0, 0], [0, 1, 0], [0, 0, 1]], "c": [0, 0, 0], "A": [], "rhs": [],
        "SOC_con_idx": [1], "number_eq": 0, "number_ineq": 0,
        "l": [-1e308] * 3, "u": [1e308] * 3, "SOC_var_idx": [1, 4],
        "sigma": 1.0, "lambda_max_A": 0.0, "lambda_max_Q": 1.0,
        "set": {"dw": [0.05, -0.05, 0.1]},
        "expect_mnorm_finite_nonnegative": True,
    },
}

# End-to-end known answers.
SOLVES = {
    # runtests.jl:260-282 (JuMP x == 5, y == 1, [t, y] in SOC, min t), in the
    # canonical layout the MOI wrapper produces: x boxed (free), then (t, y).
    "jump_soc": {
        "source": "test/runtests.jl:260-282",
        "Q": None, "c": [0, 1, 0], "A": [[1, 0, 0], [0, 0, 1]], "rhs": [5, 1],
        "SOC_con_idx": [3], "number_eq": 2, "number_ineq": 0,
        "l": [-1e308] * 3, "u": [1e308] * 3, "SOC_var_idx": [2, 4],
        "stoptol": 1e-5, "max_iter": 5000,
        "expect_x": [5.0, 1.0, 1.0], "atol": 1e-3,
    },
    # runtests.jl:544-561 — SOC variables only, Q = I, no rows: x = 0
    "soc_vars_only": {
        "source": "test/runtests.jl:544-561",
        "Q": [[1, 0, 0], [0, 1, 0], [0, 0, 1]], "c": [0, 0, 0], "A": [], "rhs": [],
        "SOC_con_idx": [1], "number_eq": 0, "number_ineq": 0,
        "l": [-1e308] * 3, "u": [1e308] * 3, "SOC_var_idx": [1, 4],
        "stoptol": 1e-5, "max_iter": 2000, "expect_x_norm_le": 1e-3,
    },
    # runtests.jl:563-581 — pure SOC constraints, Q = I: x = 0
    "pure_soc_cons": {
        "source": "test/runtests.jl:563-581",
        "Q": [[1, 0, 0], [0, 1, 0], [0, 0, 1]], "c": [0, 0, 0], "A": [[1, 0, 0], [0, 1, 0], [0, 0, 1]],
        "rhs": [0, 0, 0], "SOC_con_idx": [1, 4], "number_eq": 0, "number_ineq": 0,
        "l": [-1e308] * 3, "u": [1e308] * 3, "SOC_var_idx": [4],
        "stoptol": 1e-5, "max_iter": 2000, "expect_x_norm_le": 1e-3,
    },
    # runtests.jl:583-604 — mixed linear and SOC constraints, Q = I: x = 0
    "mixed_lin_soc": {
        "source": "test/runtests.jl:583-604",
        "Q": [[1, 0, 0, 0], [0, 1, 0, 0], [0, 0, 1, 0], [0, 0, 0, 1]], "c": [0, 0, 0, 0],
        "A": [[1, 0, 0, 0], [0, 1, 0, 0], [0, 0, 1, 0], [0, 0, 0, 1]], "rhs": [0, 0, 0, 0],
        "SOC_con_idx": [2, 5], "number_eq": 0, "number_ineq": 1,
        "l": [-1e308] * 4, "u": [1e308] * 4, "SOC_var_idx": [5],
        "stoptol": 1e-5, "max_iter": 2000, "expect_x_norm_le": 1e-3,
    },
    # runtests.jl:656-680 — trust-region SOC with equality (GPU test in the
    # reference): OPTIMAL, |Ax-b| <= 1e-5, x1 >= |x2:4|
    "trust_region": {
        "source": "test/runtests.jl:656-680",
        "Q": [[0, 0, 0, 0], [0, 1, 0, 0], [0, 0, 2, 0], [0, 0, 0, 3]], "c": [0, -1, 0.5, 0.25],
        "A": [[1, 0, 0, 0]], "rhs": [1], "SOC_con_idx": [2], "number_eq": 1, "number_ineq": 0,
        "l": [-1e308] * 4, "u": [1e308] * 4, "SOC_var_idx": [1, 5],
        "stoptol": 1e-6, "max_iter": 4000, "expect_feas_atol": 1e-5,
    },
    # data/model.cbf (+ demo/demo_JuMP.jl:4-19): min -3x-5y+z s.t.
    # x+2y <= 10, 3x+y <= 12, (0.5z+1, 0.5z-1, sqrt2 x, sqrt2 y) in Q^4,
    # x,y,z >= 0.  Optimum x=1.5, y=2.5, z=8.5, objective -8.5 (derived by
    # hand: z = x^2+y^2 at the optimum and both linear rows are slack).
    "model_cbf": {
        "source": "data/model.cbf",
        "Q": None, "c": [-3, -5, 1],
        "A": [[-1, -2, 0], [-3, -1, 0], [0, 0, 0.5], [0, 0, 0.5], [S2, 0, 0], [0, S2, 0]],
        "rhs": [-10, -12, -1, 1, 0, 0], "SOC_con_idx": [3, 7], "number_eq": 0, "number_ineq": 2,
        "l": [0, 0, 0], "u": [1e308] * 3, "SOC_var_idx": [4],
        "stoptol": 1e-8, "max_iter": 200000,
        "expect_x": [1.5, 2.5, 8.5], "expect_obj": -8.5, "atol": 1e-4,
    },
}

if __name__ == "__main__":
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_kats.json")
    with open(out, "w") as f:
        json.dump({"kats": KATS, "solves": SOLVES}, f, indent=1, sort_keys=True)
    print("wrote", out)

"""Auto-save (HPRSOCP_parameters.auto_save / save_filename): the current and
best iterates in original coordinates, their residuals and the parameters,
written on every print iteration and at termination
(src/algorithm.jl:2871-2880, save_state_to_hdf5! 306-421; the best iterate
is kept at residual checks as in compute_residuals!, 176-195).

The archive is .npz with the reference's HDF5 paths as member names.  The
final file's current iterate must be the returned solution bit for bit, and
its best iterate must be the solution of the same solve stopped at the best
iteration.
"""
import os

import numpy as np
import pytest

from hprsocp_b200 import Context, HPRSOCP_parameters, instances
from helpers import stress_model

pytestmark = pytest.mark.gpu

SCALARS = ["sigma", "err_Rp", "err_Rd", "primal_obj", "dual_obj", "rel_gap", "KKTx_and_gap"]
PARAMS = ["stoptol", "sigma", "max_iter", "time_limit", "check_iter", "warm_up", "print_frequency",
          "device_number", "use_Ruiz_scaling", "ruiz_iterations", "use_bc_scaling", "bc_scaling_norm_type",
          "use_l2_scaling", "use_Pock_Chambolle_scaling", "soc_block_scaling_strategy", "auto_save"]


def expected_members(m):
    vec = ["x_org", "w_org", "z_org"] + (["y_org"] if m > 0 else [])
    cur = ["current/" + k for k in ["iteration", "time_elapsed", "timestamp"] + vec + SCALARS]
    best = ["best/" + k for k in vec + SCALARS + ["iteration"]]
    return set(cur + best + ["parameters/" + k for k in PARAMS])


def solve(model, **kw):
    with Context(model) as ctx:
        return ctx.solve(HPRSOCP_parameters(verbose=False, **kw))


def test_final_file_is_the_returned_solution(tmp_path):
    model = instances.config0(0)
    path = str(tmp_path / "ck.npz")
    r = solve(model, stoptol=1e-6, auto_save=True, save_filename=path, print_frequency=100)
    assert r.status == "OPTIMAL"
    d = np.load(path)
    assert set(d.files) == expected_members(model.m)
    assert int(d["current/iteration"]) == r.iter
    # same unscaling expression as the returned solution: bit-identical
    assert np.array_equal(d["current/x_org"], r.x)
    assert np.array_equal(d["current/y_org"], r.y)
    assert np.array_equal(d["current/z_org"], r.z)
    assert np.array_equal(d["current/w_org"], r.x)  # no quadratic term: w = x
    assert float(d["current/KKTx_and_gap"]) == r.residuals
    assert float(d["current/err_Rp"]) == r.last["err_Rp_org_bar"]
    assert float(d["current/err_Rd"]) == r.last["err_Rd_org_bar"]
    assert float(d["current/primal_obj"]) == r.primal_obj
    assert float(d["current/sigma"]) == r.sigma
    assert float(d["current/time_elapsed"]) > 0.0
    assert str(d["current/timestamp"]).count("T") == 1
    # the best iterate is the final one when the solve ends below tolerance
    assert float(d["best/KKTx_and_gap"]) <= float(d["current/KKTx_and_gap"])
    assert int(d["best/iteration"]) == r.iter
    assert np.array_equal(d["best/x_org"], r.x)
    assert float(d["parameters/stoptol"]) == 1e-6
    assert int(d["parameters/print_frequency"]) == 100
    assert bool(d["parameters/auto_save"])
    assert str(d["parameters/soc_block_scaling_strategy"]) == "phase_taper"
    assert str(d["parameters/bc_scaling_norm_type"]) == "l2"
    assert [f for f in os.listdir(tmp_path) if ".tmp" in f] == []


def test_best_iterate_is_the_solve_stopped_there(tmp_path):
    """With a fixed iteration budget the last iterate is not always the
    best; the file's best iterate must equal a rerun stopped at best/iteration."""
    model = stress_model(3)
    path = str(tmp_path / "ck.npz")
    kw = dict(stoptol=0.0, check_iter=150, print_frequency=50)
    r = solve(model, max_iter=1200, auto_save=True, save_filename=path, **kw)
    d = np.load(path)
    bi = int(d["best/iteration"])
    assert bi % 50 == 0 and 0 <= bi <= r.iter
    assert float(d["best/KKTx_and_gap"]) <= float(d["current/KKTx_and_gap"])
    rb = solve(model, max_iter=bi, **kw)
    assert rb.iter == bi
    assert np.array_equal(d["best/x_org"], rb.x)
    assert np.array_equal(d["best/y_org"], rb.y)
    assert np.array_equal(d["best/z_org"], rb.z)
    assert float(d["best/KKTx_and_gap"]) == rb.residuals


def test_quadratic_term_writes_w(tmp_path):
    model = instances.small_socp(11, n=300, diag_q=True)
    path = str(tmp_path / "q.npz")
    r = solve(model, stoptol=1e-6, auto_save=True, save_filename=path)
    d = np.load(path)
    assert np.array_equal(d["current/x_org"], r.x)
    assert np.array_equal(d["current/w_org"], r.w)


def test_warm_start_vectors_are_recorded(tmp_path):
    model = instances.config0(0)
    ref = solve(model, stoptol=1e-4)
    path = str(tmp_path / "w.npz")
    solve(model, stoptol=1e-6, initial_x=ref.x, initial_y=ref.y, auto_save=True, save_filename=path)
    d = np.load(path)
    assert np.array_equal(d["parameters/initial_x"], ref.x)
    assert np.array_equal(d["parameters/initial_y"], ref.y)


def test_unwritable_path_does_not_fail_the_solve(tmp_path):
    model = instances.config0(0)
    path = str(tmp_path / "no_such_dir" / "ck.npz")
    ref = solve(model, stoptol=1e-6)
    r = solve(model, stoptol=1e-6, auto_save=True, save_filename=path)
    assert r.status == "OPTIMAL" and r.iter == ref.iter
    assert np.array_equal(r.x, ref.x)
    assert not os.path.exists(path)


def test_auto_save_leaves_the_iterates_unchanged(tmp_path):
    # (print iterations are also residual checks, so both runs print alike)
    model = stress_model(4)
    ref = solve(model, stoptol=1e-6, print_frequency=30)
    r = solve(model, stoptol=1e-6, auto_save=True, save_filename=str(tmp_path / "s.npz"), print_frequency=30)
    assert r.iter == ref.iter
    assert np.array_equal(r.x, ref.x) and np.array_equal(r.y, ref.y)

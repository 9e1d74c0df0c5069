"""The engine's tile planner (hpr-socp_b200/csrc/hpr_plan.cpp) on the host,
built here from its source with a small driver (plan_selftest.cpp): random
row lengths (empty rows, rows longer than a tile), linear rows and cones of
1 to 364 rows, full and capped tiles.  Every plan must cover each row
exactly once, keep tiles within their nonzero and row caps, keep small cones
whole, number the slices of split cones and long rows, queue apply tiles
last, and carry run descriptors (row starts, ordinals, non-empty masks,
slot offsets) that match the row pointers."""
import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CUDA_INC = "/usr/local/cuda/include"


@pytest.fixture(scope="module")
def driver(tmp_path_factory):
    cxx = shutil.which("g++") or shutil.which("c++")
    if cxx is None or not os.path.isdir(CUDA_INC):
        pytest.skip("no C++ compiler or CUDA headers")
    exe = str(tmp_path_factory.mktemp("plan") / "plan_selftest")
    subprocess.run([cxx, "-std=c++17", "-O2", "-I", CUDA_INC, "-o", exe, os.path.join(HERE, "plan_selftest.cpp"),
                    os.path.join(ROOT, "hpr-socp_b200", "csrc", "hpr_plan.cpp")], check=True)
    return exe


@pytest.mark.parametrize("seed", [1, 2, 3, 4])
def test_random_plans_keep_the_engine_invariants(driver, seed):
    out = subprocess.run([driver, str(seed), "150"], capture_output=True, text=True)
    assert out.returncode == 0, out.stdout[-2000:]
    assert out.stdout.strip() == "ok 150"

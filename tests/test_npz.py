"""The auto-save archive writer (hpr-socp_b200/csrc/hpr_npz.cpp), built here
from its source with a small driver (npz_selftest.cpp): NumPy must read every
member back, zipfile must accept every CRC-32, and the CRC-32 itself must
match zlib's for every length and split point."""
import os
import shutil
import subprocess
import zipfile
import zlib

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


@pytest.fixture(scope="module")
def driver(tmp_path_factory):
    cxx = shutil.which("g++") or shutil.which("c++")
    if cxx is None:
        pytest.skip("no C++ compiler")
    exe = str(tmp_path_factory.mktemp("npz") / "npz_selftest")
    subprocess.run([cxx, "-std=c++17", "-O2", "-o", exe, os.path.join(HERE, "npz_selftest.cpp"),
                    os.path.join(ROOT, "hpr-socp_b200", "csrc", "hpr_npz.cpp")], check=True)
    return exe


@pytest.mark.parametrize("zip64", [0, 1])
def test_archive_reads_back(driver, tmp_path, zip64):
    path = str(tmp_path / f"t{zip64}.npz")
    out = subprocess.run([driver, path, str(zip64)], check=True, capture_output=True, text=True).stdout
    with zipfile.ZipFile(path) as z:
        assert z.testzip() is None  # every member's CRC-32 checks
        names = z.namelist()
    assert names == ["current/x_org.npy", "best/y_org.npy", "current/sigma.npy", "best/iteration.npy",
                     "parameters/auto_save.npy", "parameters/use_l2_scaling.npy", "current/timestamp.npy",
                     "empty.npy", "matrix.npy"]
    d = np.load(path, allow_pickle=False)
    x = d["current/x_org"]
    assert x.dtype == np.float64 and x.shape == (100003,)
    assert np.array_equal(x, 0.5 * np.arange(100003) - 3.25)
    assert d["best/y_org"].shape == (0,)
    assert d["current/sigma"].shape == () and float(d["current/sigma"]) == 1.25
    assert d["best/iteration"].dtype == np.int64 and int(d["best/iteration"]) == 150
    assert d["parameters/auto_save"].dtype == np.bool_ and bool(d["parameters/auto_save"])
    assert not bool(d["parameters/use_l2_scaling"])
    assert str(d["current/timestamp"]) == "2026-01-02T03:04:05.678"
    assert str(d["empty"]) == ""
    assert np.array_equal(d["matrix"], (np.arange(12, dtype=np.int64) * 7 - 20).reshape(3, 4))
    data = bytes((i * 37 + 11) & 0xFF for i in range(40))
    for line in out.splitlines():
        _, n, v = line.split()
        assert int(v) == zlib.crc32(data[:int(n)])

"""The C++17 drop-in header (include/qpp_b200.hpp) compiles against qpp's
signatures and passes the reference KATs through libqpp_b200.so."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _build(tmp_path):
    exe = str(tmp_path / "test_shim")
    subprocess.run(["g++", "-std=c++17", "-O1", "-I", os.path.join(ROOT, "include"),
                    "-I", "/usr/local/cuda/include",
                    os.path.join(ROOT, "tests", "cpp", "test_shim.cpp"),
                    "-L", os.path.join(ROOT, "qpp_b200"), "-lqpp_b200",
                    f"-Wl,-rpath,{os.path.join(ROOT, 'qpp_b200')}", "-o", exe], check=True)
    return exe


def test_shim_compiles(tmp_path):
    assert os.path.exists(_build(tmp_path))


@pytest.mark.gpu
def test_shim_runs_reference_kats(tmp_path):
    exe = _build(tmp_path)
    r = subprocess.run([exe], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "shim ok" in r.stdout

"""The Eigen-typed overloads of the C++ drop-in layer (include/qpp_b200.hpp):
compiled here against a minimal stand-in for Eigen's interface (Eigen itself
is not installed) and, on a GPU, run against the same calls on
qpp_b200::cmat, which must return identical matrices (tests/cpp/
test_eigen_shim.cpp)."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _build(tmp_path):
    exe = str(tmp_path / "test_eigen_shim")
    subprocess.run(["g++", "-std=c++17", "-O1",
                    "-I", os.path.join(ROOT, "tests", "cpp", "eigen_standin"),
                    "-I", os.path.join(ROOT, "include"), "-I", "/usr/local/cuda/include",
                    os.path.join(ROOT, "tests", "cpp", "test_eigen_shim.cpp"),
                    "-L", os.path.join(ROOT, "qpp_b200"), "-lqpp_b200",
                    f"-Wl,-rpath,{os.path.join(ROOT, 'qpp_b200')}", "-o", exe], check=True)
    return exe


def test_eigen_adapters_compile(tmp_path):
    assert os.path.exists(_build(tmp_path))


@pytest.mark.gpu
def test_eigen_adapters_match_cmat_calls(tmp_path):
    exe = _build(tmp_path)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "eigen adapters ok" in r.stdout

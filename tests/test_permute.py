"""Tiled bit permutation behind ptranspose / syspermute, checked on the CPU:
every output written once, every read inside the input, and the same source
element as the plain gather (tests/cpp/test_permute.cpp)."""
import os
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_tiled_permutation_addresses(tmp_path):
    exe = str(tmp_path / "test_permute")
    subprocess.run(["g++", "-std=c++17", "-O2", "-I", os.path.join(ROOT, "qpp_b200", "csrc"),
                    "-I", os.path.join(ROOT, "include"), "-I", "/usr/local/cuda/include",
                    os.path.join(ROOT, "tests", "cpp", "test_permute.cpp"),
                    "-L", os.path.join(ROOT, "qpp_b200"), "-lqpp_b200",
                    f"-Wl,-rpath,{os.path.join(ROOT, 'qpp_b200')}", "-o", exe], check=True)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "permute ok" in r.stdout

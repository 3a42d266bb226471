"""QFT pass plans behind qgpu_apply_qft, checked on the CPU: a host model of
k_qft_pass runs every planned pass and must reproduce the transform's
definition within 1e-12, reading and writing inside the state and writing
every element once (tests/cpp/test_qft.cpp)."""
import os
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_qft_pass_plans(tmp_path):
    exe = str(tmp_path / "test_qft")
    subprocess.run(["g++", "-std=c++17", "-O2", "-I", os.path.join(ROOT, "qpp_b200", "csrc"),
                    "-I", os.path.join(ROOT, "include"), "-I", "/usr/local/cuda/include",
                    os.path.join(ROOT, "tests", "cpp", "test_qft.cpp"),
                    "-L", os.path.join(ROOT, "qpp_b200"), "-lqpp_b200",
                    f"-Wl,-rpath,{os.path.join(ROOT, 'qpp_b200')}", "-o", exe], check=True)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "qft plans ok" in r.stdout

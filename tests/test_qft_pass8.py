"""Addressing of the register-round QFT passes (k_qft_pass8), checked on the
CPU on the plans of whole transforms of 22-30 qubits: both rounds cover the
tile once, the shared-memory swizzle is a bijection spreading every warp
access over the banks, loads and stores run over >= 128 contiguous bytes,
and every tile stays inside the state (tests/cpp/test_qft_pass8.cpp)."""
import os
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_qft_pass8_addressing(tmp_path):
    exe = str(tmp_path / "test_qft_pass8")
    subprocess.run(["g++", "-std=c++17", "-O2", "-I", os.path.join(ROOT, "qpp_b200", "csrc"),
                    "-I", os.path.join(ROOT, "include"), "-I", "/usr/local/cuda/include",
                    os.path.join(ROOT, "tests", "cpp", "test_qft_pass8.cpp"),
                    "-L", os.path.join(ROOT, "qpp_b200"), "-lqpp_b200",
                    f"-Wl,-rpath,{os.path.join(ROOT, 'qpp_b200')}", "-o", exe], check=True)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "qft pass8 ok" in r.stdout

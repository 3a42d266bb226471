"""Tile passes of the plain form (runs of 1- and 2-qubit gates applied in
shared memory, one read and one write of the state per run), checked on the
CPU: the planner and a host model of the kernel's addressing reproduce the
gate-by-gate result bit for bit (tests/cpp/test_gate_tiles.cpp)."""
import os
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_tile_passes_reproduce_gate_by_gate(tmp_path):
    exe = str(tmp_path / "test_gate_tiles")
    subprocess.run(["g++", "-std=c++17", "-O2", "-ffp-contract=off",
                    "-I", os.path.join(ROOT, "qpp_b200", "csrc"),
                    "-I", os.path.join(ROOT, "include"), "-I", "/usr/local/cuda/include",
                    os.path.join(ROOT, "tests", "cpp", "test_gate_tiles.cpp"),
                    "-L", os.path.join(ROOT, "qpp_b200"), "-lqpp_b200",
                    f"-Wl,-rpath,{os.path.join(ROOT, 'qpp_b200')}", "-o", exe], check=True)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "gate tiles ok" in r.stdout

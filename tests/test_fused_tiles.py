"""The fused complex128 form's tile-pass runs (blocks of <= 2 qubits from the
fusion planner, cut into runs of gate descriptors and steps run as they are),
checked on the CPU against the circuit's steps applied one by one, within
1e-12 (tests/cpp/test_fused_tiles.cpp)."""
import os
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_fused_tile_runs_reproduce_the_steps(tmp_path):
    exe = str(tmp_path / "test_fused_tiles")
    subprocess.run(["g++", "-std=c++17", "-O2",
                    "-I", os.path.join(ROOT, "qpp_b200", "csrc"),
                    "-I", os.path.join(ROOT, "include"), "-I", "/usr/local/cuda/include",
                    os.path.join(ROOT, "tests", "cpp", "test_fused_tiles.cpp"),
                    "-L", os.path.join(ROOT, "qpp_b200"), "-lqpp_b200",
                    f"-Wl,-rpath,{os.path.join(ROOT, 'qpp_b200')}", "-o", exe], check=True)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "fused tiles ok" in r.stdout

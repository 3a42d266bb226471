"""Cache blocking of the trajectory kernel, checked on the CPU: the planner's
tile passes reproduce the untiled programs bit for bit under a host
restatement of the kernel's gather / scatter addressing, and every address
stays inside the register (tests/cpp/test_tiles.cpp)."""
import os
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_tile_passes_match_untiled_programs(tmp_path):
    exe = str(tmp_path / "test_tiles")
    subprocess.run(["g++", "-std=c++17", "-O2", "-I", os.path.join(ROOT, "qpp_b200", "csrc"),
                    "-I", os.path.join(ROOT, "include"), "-I", "/usr/local/cuda/include",
                    os.path.join(ROOT, "tests", "cpp", "test_tiles.cpp"),
                    "-L", os.path.join(ROOT, "qpp_b200"), "-lqpp_b200",
                    f"-Wl,-rpath,{os.path.join(ROOT, 'qpp_b200')}", "-o", exe], check=True)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "tiles ok" in r.stdout

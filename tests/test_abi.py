"""The C-ABI library loads without a GPU and exports every symbol that
include/*.h declares (no compute call is made here)."""
import ctypes
import glob
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    syms = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"\b(qgpu_[a-z0-9_]+)\s*\(", src):
            syms.add(m.group(1))
    return syms


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(os.path.join(ROOT, "qpp_b200", "libqpp_b200.so"))
    syms = declared_symbols()
    assert len(syms) > 30
    missing = [s for s in sorted(syms) if not hasattr(lib, s)]
    assert not missing, missing


def test_status_names_without_gpu():
    import qpp_b200 as qb
    L = qb.lib()
    assert L.qgpu_status_name(9).decode() == "SubsysMismatchDims"
    assert b"sm_100a" in L.qgpu_version()

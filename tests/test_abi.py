"""The C-ABI library loads without a GPU and exports every function include/*.h declares."""
import ctypes
import glob
import os
import re

from vshe.abi import LIB_PATH

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"\b(vshe_[a-z0-9_]+)\s*\(", text):
            names.add(m.group(1))
    return names


def test_library_exports_every_declared_symbol():
    assert os.path.exists(LIB_PATH), "build the library first (__graft_entry__.build())"
    lib = ctypes.CDLL(LIB_PATH)
    names = declared_functions()
    assert len(names) >= 15
    missing = [n for n in sorted(names) if not hasattr(lib, n)]
    assert not missing, missing


def test_errstr_and_defaults_without_gpu():
    from vshe import gpu
    L = gpu.lib()
    assert L.vshe_errstr(-2).decode().startswith("solve(): Found empty row")
    o, _ = gpu.make_opts()
    assert o.precision == 1 and abs(o.tol - 1e-10) < 1e-24 and o.max_iters == 1000

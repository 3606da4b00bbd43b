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


def _c_layout(struct_names, tmp_path):
    """sizeof and the offset of every member of each struct, as g++ lays them out from the
    public headers."""
    import subprocess
    mirrors = _mirrors()
    lines = ['#include <cstdio>', '#include <cstddef>', '#include "vshe_gpu.h"', "int main() {"]
    for cname in struct_names:
        py = mirrors[cname]
        lines.append('  printf("%s %%zu\\n", sizeof(%s));' % (cname, cname))
        for fname, _ in py._fields_:
            lines.append('  printf("%s.%s %%zu\\n", offsetof(%s, %s));' % (cname, fname, cname, fname))
    lines.append("  return 0; }")
    src = tmp_path / "layout.cpp"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["g++", "-std=c++17", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout
    return dict((k, int(v)) for k, v in (ln.split() for ln in out.strip().splitlines()))


def _mirrors():
    from vshe import abi, gpu
    return {"vshe_solve_opts": abi.SolveOptsC, "vshe_solve_stats": abi.SolveStatsC, "vshe_she_info": gpu.SheInfoC,
            "vshe_server_opts": gpu.ServerOptsC, "vshe_server_result": gpu.ServerResultC,
            "vshe_device_desc": abi.DeviceDescC, "vshe_she_config": abi.SheConfigC, "vshe_coupling_tables": abi.CouplingC}


def test_ctypes_mirrors_match_the_c_layout(tmp_path):
    """Every struct the ctypes binding mirrors has the size and member offsets g++ gives the
    header's struct, so no field is read or written at the wrong place."""
    mirrors = _mirrors()
    got = _c_layout(list(mirrors), tmp_path)
    for cname, py in mirrors.items():
        assert got[cname] == ctypes.sizeof(py), cname
        for fname, _ in py._fields_:
            assert got["%s.%s" % (cname, fname)] == getattr(py, fname).offset, (cname, fname)

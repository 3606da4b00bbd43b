"""Extract the reference's tabulated spherical-harmonics coupling coefficients.

The reference ships a_{x,y,z} and b_{x,y,z} for L = 1, 3, 5, 7 as literal
assignments in viennashe/she/harmonics_coupling.hpp (fill_coupling_matrices_1,
_3, _5, _7 at :282, :309, :417, :644).  This script reads that file as text
and writes the values as golden fixtures (tests/golden/coupling_L{L}.json),
which the tests use to pin (a) the library's own quadrature of the coupling
integrals and (b) assembly parity when the reference's own tables are fed in.

Run from the repository root:  python tests/golden/make_coupling_golden.py [viennashe-dev root]
(the reference tree: the argument, else $VIENNASHE_REF_ROOT, else /root/reference; the fixtures
are committed).
"""
import json
import os
import re
import sys

REF_ROOT = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("VIENNASHE_REF_ROOT", "/root/reference")
REF = os.path.join(REF_ROOT, "viennashe", "she", "harmonics_coupling.hpp")
HERE = os.path.dirname(os.path.abspath(__file__))
NAMES = ["a_x", "a_y", "a_z", "b_x", "b_y", "b_z"]


def extract(text, L):
    m = re.search(r"void fill_coupling_matrices_%d\s*\(" % L, text)
    if not m:
        raise SystemExit("fill_coupling_matrices_%d not found" % L)
    start = text.index("{", m.end())
    depth, i = 0, start
    while True:
        if text[i] == "{":
            depth += 1
        elif text[i] == "}":
            depth -= 1
            if depth == 0:
                break
        i += 1
    body = text[start:i]
    out = {n: [] for n in NAMES}
    for name, r, c, val in re.findall(r"\b([ab]_[xyz])\((\d+),\s*(\d+)\)\s*=\s*([-+0-9.eE]+)\s*;", body):
        out[name].append([int(r), int(c), float(val)])
    return out


def main():
    if not os.path.exists(REF):
        sys.exit("reference tree not available: " + REF)
    text = open(REF).read()
    for L in (1, 3, 5, 7):
        tab = extract(text, L)
        doc = {
            "source": "viennashe/she/harmonics_coupling.hpp fill_coupling_matrices_%d" % L,
            "L": L,
            "dim": (L + 1) ** 2,
            "entries": tab,
        }
        path = os.path.join(HERE, "coupling_L%d.json" % L)
        with open(path, "w") as f:
            json.dump(doc, f, indent=0)
        print(path, {k: len(v) for k, v in tab.items()})


if __name__ == "__main__":
    main()

"""Writes tests/golden/bar200x50x160_reduced.json: the oracle's reduced, scaled and normalised
system of the benchmark's 2D bar (400 x 100 nm on a 200 x 50 mesh, contacts 1e25 / channel 1e22
m^-3, Gaussian doping edges jittered from seed 7, L = 3, 160 energies, 0.8 V; vshe.devices.config2),
the state vshe_she_assemble(3) produces on the device.  Stored: the sizes, SHA-256 of the row
offsets (int64, little endian) and of the column indices (int32, little endian), and the columns,
values and rhs of 96 rows drawn with seed 2024.  The oracle needs about 45 GB of host memory and a
few minutes for this size.

Usage: python tests/golden/make_bar_fixture.py [--nx 200 --ny 50 --ne 160 --L 3] [--out PATH]
"""
import argparse
import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "viennashe-dev_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

from vshe import devices as D  # noqa: E402
import oracle_api as O  # noqa: E402


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--nx", type=int, default=200)
    ap.add_argument("--ny", type=int, default=50)
    ap.add_argument("--ne", type=int, default=160)
    ap.add_argument("--L", type=int, default=3)
    ap.add_argument("--rows", type=int, default=96)
    ap.add_argument("--out", default=None)
    a = ap.parse_args()
    dev, cfg = D.config2(nx=a.nx, ny=a.ny, n_energies=a.ne, L=a.L)
    P = O.OracleProblem(dev, cfg, O.golden_coupling(a.L))
    A = P.matrix(3)
    sizes = dict(n_odd=P.n_odd, nnz_full=P.nnz[0])
    del P
    rng = np.random.default_rng(2024)
    rows = sorted(int(i) for i in rng.choice(A.n, size=a.rows, replace=False))
    out = {
        "workload": "nin_bar_2d_%dx%d_L%d_E%d_0.8V" % (a.nx, a.ny, a.L, a.ne),
        "nx": a.nx, "ny": a.ny, "n_energies": a.ne, "L": a.L,
        "n": int(A.n), "nnz": int(A.nnz), "n_odd": int(sizes["n_odd"]), "nnz_full": int(sizes["nnz_full"]),
        "sha256_row_ptr": hashlib.sha256(np.ascontiguousarray(A.rp, "<i8").tobytes()).hexdigest(),
        "sha256_col": hashlib.sha256(np.ascontiguousarray(A.ci, "<i4").tobytes()).hexdigest(),
        "rows": [{"row": i, "col": A.ci[A.rp[i]:A.rp[i + 1]].tolist(), "val": A.v[A.rp[i]:A.rp[i + 1]].tolist(),
                  "rhs": float(A.rhs[i])} for i in rows],
    }
    path = a.out or os.path.join(HERE, "bar%dx%dx%d_reduced.json" % (a.nx, a.ny, a.ne))
    with open(path, "w") as f:
        json.dump(out, f, indent=0)
    print("wrote", path, "n=%d nnz=%d" % (A.n, A.nnz))


if __name__ == "__main__":
    main()

"""Solves through the drop-in adapter compiled against the reference's headers
(tests/adapter/_build/libadapter_check.so, built by tests/adapter/build.sh): the reference's
sparse_matrix and linear_solver_config go in, the gpu-slot overload converts them to CSR and calls
vshe_solve_csr with the options it derives from the energy-slab bounds, and the result is the
oracle's solution within the bounds of a 1e-10 solve.  A second call on the same pattern (the
next Gummel step) reuses the resident schedule and gives the same x."""
import ctypes as C
import os

import numpy as np
import pytest

from vshe import devices as D
import oracle_api as O
import cases

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "tests", "adapter", "_build", "libadapter_check.so")


def _lib():
    assert os.path.exists(LIB), "build the adapter harness first (tests/adapter/build.sh, run by __graft_entry__.build())"
    L = C.CDLL(LIB)
    p64, p32, pd = C.POINTER(C.c_int64), C.POINTER(C.c_int32), C.POINTER(C.c_double)
    L.adapter_check_solve.argtypes = [C.c_int64, p64, p32, pd, pd, C.c_int64, p64, C.c_double, C.c_int64, pd, C.c_char_p, C.c_int]
    return L


def _solve(L, A, slabs, tol=1e-10):
    x = np.zeros(A.n)
    msg = C.create_string_buffer(512)
    s = np.ascontiguousarray(slabs, np.int64)
    rc = L.adapter_check_solve(A.n, A.rp.ctypes.data_as(C.POINTER(C.c_int64)), A.ci.ctypes.data_as(C.POINTER(C.c_int32)),
                               A.v.ctypes.data_as(C.POINTER(C.c_double)), A.rhs.ctypes.data_as(C.POINTER(C.c_double)),
                               len(s) - 1, s.ctypes.data_as(C.POINTER(C.c_int64)), tol, 20000,
                               x.ctypes.data_as(C.POINTER(C.c_double)), msg, 512)
    assert rc == 0, (rc, msg.value)
    return x


@pytest.mark.parametrize("case", ["bar_slabs", "diode"])
def test_adapter_solve_matches_oracle(case):
    if case == "bar_slabs":
        # slabs of up to 864 cells x 6 harmonics: wide enough for the per-slab block-ILU(1) path
        P = cases.oracle_problem(*D.config2(nx=70, ny=12, n_energies=60, L=3, bias=0.3))
    else:
        P = cases.oracle_problem(*cases.diode_small(L=1, boxes=60, bias=0.4))
    A = P.matrix(3)
    L = _lib()
    x = _solve(L, A, P.blocks())
    res = np.linalg.norm(O.spmv(A, x) - A.rhs) / np.linalg.norm(A.rhs)
    assert res < 1e-10
    xr, sr = O.csr_solve(A, A.rhs, precond=1, tol=1e-13, maxit=20000)
    assert sr["rc"] == 0
    assert np.max(np.abs(x - xr)) <= 5e-6 * np.max(np.abs(xr))
    # next Gummel step on the same pattern: the resident schedule is reused, same result
    x2 = _solve(L, A, P.blocks())
    assert np.array_equal(x, x2)

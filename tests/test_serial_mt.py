"""The reference arm's CPU solver (oracle/serial_solver_mt.cpp: serial_linear_solver's natural
ILU(0) + BiCGStab with r^ = r_0, level-scheduled over host threads) against the single-threaded
oracle.  With one thread every inner product sums in the serial order, so the iterates are
bitwise the oracle's; with several only the summation order of the inner products differs."""
import numpy as np
import pytest

import oracle_api as O
import cases


@pytest.fixture(scope="module", params=["diode_L1", "bar_L3"])
def system(request):
    if request.param == "diode_L1":
        P = cases.oracle_problem(*cases.diode_small(L=1, boxes=60, bias=0.4))
    else:
        P = cases.oracle_problem(*cases.bar_small(L=3, nx=12, ny=5, n_energies=30))
    return P.matrix(3)


def test_one_thread_is_the_serial_oracle(system):
    A = system
    x_ref, st_ref = O.csr_solve(A, A.rhs, precond=1, tol=1e-10, maxit=5000)
    x, st = O.serial_solve_mt(A, A.rhs, tol=1e-10, maxit=5000, threads=1)
    assert st["rc"] == 0 and st_ref["rc"] == 0
    assert st["iters"] == st_ref["iters"]
    assert st["relres"] == st_ref["relres"]
    assert np.array_equal(x, x_ref)


def test_threads_converge_like_the_serial_oracle(system):
    A = system
    x_ref, st_ref = O.csr_solve(A, A.rhs, precond=1, tol=1e-10, maxit=5000)
    x, st = O.serial_solve_mt(A, A.rhs, tol=1e-10, maxit=5000, threads=4, trace=True)
    assert st["rc"] == 0 and st["threads"] == 4
    assert abs(st["iters"] - st_ref["iters"]) <= max(2, st_ref["iters"] // 10)
    res = np.linalg.norm(O.spmv(A, x) - A.rhs) / np.linalg.norm(A.rhs)
    assert res < 1e-9
    xd = O.dense_solve(A, A.rhs) if A.n <= 4000 else x_ref
    assert np.linalg.norm(x - xd) / np.linalg.norm(xd) < 1e-6
    assert len(st["iter_s"]) == st["iters"] + 1 and np.all(np.diff(st["iter_s"]) >= 0)

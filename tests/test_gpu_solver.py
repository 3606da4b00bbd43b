"""CUDA solver path (through the C ABI) against the CPU oracle.

Tolerances: SpMV FP64 1e-13 relative (summation order differs), FP32 1e-6;
ILU(0) factor values 1e-11 relative to the row scale; solutions to the
stated FP64 residual 1e-10, and within 1e-7 of the oracle's direct solution.
"""
import numpy as np
import pytest

from vshe import devices as D
from vshe import gpu
import oracle_api as O
import cases

pytestmark = pytest.mark.gpu


def _problems():
    out = []
    dev, cfg = cases.diode_small(L=1, boxes=40)
    out.append(("diode_L1", dev, cfg))
    dev, cfg = cases.diode_small(L=3, boxes=30)
    out.append(("diode_L3", dev, cfg))
    dev, cfg = cases.bar_small(L=3, nx=12, ny=5, n_energies=30)
    out.append(("bar_L3", dev, cfg))
    return out


PROBLEMS = _problems()


@pytest.fixture(scope="module", params=PROBLEMS, ids=[p[0] for p in PROBLEMS])
def prob(request):
    name, dev, cfg = request.param
    P = cases.oracle_problem(dev, cfg)
    A = P.matrix(3)
    return name, P, A


def test_spmv_parity(gpu_ctx, prob):
    name, P, A = prob
    rng = np.random.default_rng(1)
    x = rng.standard_normal(A.n)
    S = gpu_ctx.system(A.rp, A.ci, A.v, A.rhs, precision="mixed")
    try:
        y_ref = O.spmv(A, x)
        y = S.spmv(x, "fp64")
        assert np.max(np.abs(y - y_ref)) <= 1e-13 * np.max(np.abs(y_ref))
        # the SpMV is FP64 in every mode; no FP32 copy of A exists
        with pytest.raises(gpu.VsheError):
            S.spmv(x, "mixed")
        # the solution vector is not used as scratch
        S.solve()
        x_sol = S.x()
        S.spmv(x, "fp64")
        assert np.array_equal(S.x(), x_sol)
    finally:
        S.free()


@pytest.mark.parametrize("block", [False, True])
def test_ilu0_factor_parity(gpu_ctx, prob, block):
    name, P, A = prob
    bl = P.blocks() if block else None
    S = gpu_ctx.system(A.rp, A.ci, A.v, A.rhs, precision="fp64", precond="block_ilu0" if block else "ilu0", blocks=bl)
    try:
        lu = S.factor_values()
        lu_ref = O.ilu0_values(A, blocks=bl)
        if block:
            blk = np.zeros(A.n, np.int64)
            for k in range(len(bl) - 1):
                blk[bl[k]:bl[k + 1]] = k
            rows = np.repeat(np.arange(A.n), np.diff(A.rp))
            lu_ref = np.where(blk[A.ci] == blk[rows], lu_ref, 0.0)
        scale = np.maximum(np.abs(lu_ref), 1.0)
        assert np.max(np.abs(lu - lu_ref) / scale) < 1e-11
    finally:
        S.free()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("precond,ordering", [("ilu0", "natural"), ("block_ilu0", "natural"), ("ilu0", "multicolor")])
def test_solve_parity(gpu_ctx, prob, precision, precond, ordering):
    name, P, A = prob
    xd = O.dense_solve(A, A.rhs) if A.n <= 4000 else O.csr_solve(A, A.rhs, tol=1e-14, maxit=20000)[0]
    bl = P.blocks() if precond == "block_ilu0" else None
    x, st = gpu_ctx.solve_csr(A.rp, A.ci, A.v, A.rhs, precision=precision, precond=precond, blocks=bl,
                              ordering=ordering, tol=1e-10, max_iters=4000)
    assert st["status"] == 0, st
    r = O.spmv(A, x) - A.rhs
    assert np.linalg.norm(r) / np.linalg.norm(A.rhs) < 1e-10
    assert st["rel_residual"] < 1e-10
    assert np.linalg.norm(x - xd) / np.linalg.norm(xd) < 1e-7


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_terminal_currents_at_tight_tolerance(gpu_ctx, prob, precision):
    """Terminal currents within 1e-8 of the oracle's direct solution when the solve is taken
    to a 1e-14 FP64 residual.  The current is the small anisotropic part of the solution: the
    oracle's own solve at 1e-12 still misses it by up to 2.6e-7, at 1e-14 by 2e-11."""
    name, P, A = prob
    xd = O.dense_solve(A, A.rhs) if A.n <= 4000 else O.csr_solve(A, A.rhs, tol=1e-15, maxit=20000)[0]
    x, st = gpu_ctx.solve_csr(A.rp, A.ci, A.v, A.rhs, precision=precision, precond="ilu0", tol=1e-14, max_iters=4000)
    assert st["status"] == 0 and st["rel_residual"] < 1e-14, st
    _, dens, cur, res = P.finish(x)
    _, dens_r, cur_r, _ = P.finish(xd)
    assert np.max(np.abs(cur - cur_r)) <= 1e-8 * np.max(np.abs(cur_r))
    assert np.max(np.abs(dens - dens_r) / dens_r) < 1e-8


def test_batch_equals_alone(gpu_ctx):
    probs = [cases.oracle_problem(*cases.diode_small(L=L, boxes=b, bias=v)) for L, b, v in ((1, 30, 0.2), (3, 24, 0.5), (1, 50, 0.8))]
    mats = [P.matrix(3) for P in probs]
    alone = []
    for A in mats:
        S = gpu_ctx.system(A.rp, A.ci, A.v, A.rhs, precision="mixed")
        x, st = S.solve()
        assert st["status"] == 0
        alone.append(x)
        S.free()
    systems = [gpu_ctx.system(A.rp, A.ci, A.v, A.rhs, precision="mixed") for A in mats]
    try:
        stats = gpu_ctx.batch_solve(systems)
        for S, st, xa, A in zip(systems, stats, alone, mats):
            assert st["status"] == 0 and st["rel_residual"] < 1e-10
            xb = S.x()
            assert np.array_equal(xb, xa), np.max(np.abs(xb - xa))
    finally:
        for S in systems:
            S.free()


def test_reference_error_behaviour(gpu_ctx):
    # empty row -> solve(): Found empty row (src/solvers/solve.hpp:54-58)
    rp = np.array([0, 1, 1, 2]); ci = np.array([0, 2]); v = np.array([1.0, 1.0])
    with pytest.raises(gpu.VsheError) as e:
        gpu_ctx.solve_csr(rp, ci, v, np.ones(3))
    assert e.value.code == -2
    # non-finite rhs -> error
    rp = np.array([0, 1, 2]); ci = np.array([0, 1]); v = np.array([2.0, 4.0])
    with pytest.raises(gpu.VsheError) as e:
        gpu_ctx.solve_csr(rp, ci, v, np.array([1.0, np.nan]))
    assert e.value.code == -3
    # ||b|| = 0 -> x = 0
    x, st = gpu_ctx.solve_csr(rp, ci, v, np.zeros(2))
    assert np.all(x == 0) and st["status"] == 0
    # diagonal system solves exactly
    x, st = gpu_ctx.solve_csr(rp, ci, v, np.array([1.0, 1.0]), precision="fp64")
    assert np.allclose(x, [0.5, 0.25], rtol=1e-14)


@pytest.mark.parametrize("ordering", ["natural", "multicolor"])
def test_iluk_factor_and_solve(gpu_ctx, prob, ordering):
    """ILU(1) (levels of fill, Saad Alg. 10.5): the factor values at A's entries match the
    oracle's ILU(1) (natural order), and the solve reaches 1e-10 in no more iterations than
    ILU(0) on the same ordering."""
    name, P, A = prob
    if ordering == "natural":
        S = gpu_ctx.system(A.rp, A.ci, A.v, A.rhs, precision="fp64", precond="ilu0", fill_level=1)
        try:
            lu = S.factor_values()
        finally:
            S.free()
        rp, ci, flu = O.iluk_csr(A, 1)
        ref = np.zeros(A.nnz)
        for i in range(A.n):
            cols = ci[rp[i]:rp[i + 1]]
            pos = np.searchsorted(cols, A.ci[A.rp[i]:A.rp[i + 1]])
            ref[A.rp[i]:A.rp[i + 1]] = flu[rp[i] + pos]
        assert np.max(np.abs(lu - ref) / np.maximum(np.abs(ref), 1.0)) < 1e-11
    xd = O.dense_solve(A, A.rhs) if A.n <= 4000 else O.csr_solve(A, A.rhs, tol=1e-14, maxit=20000)[0]
    its = {}
    for k in (0, 1):
        x, st = gpu_ctx.solve_csr(A.rp, A.ci, A.v, A.rhs, precision="mixed", precond="ilu0", ordering=ordering,
                                  fill_level=k, tol=1e-10, max_iters=4000)
        assert st["status"] == 0 and st["rel_residual"] < 1e-10, st
        assert np.linalg.norm(x - xd) / np.linalg.norm(xd) < 1e-7
        its[k] = st["iterations"]
    assert its[1] <= its[0], its


def test_ilut_factor_matches_oracle(gpu_ctx, prob):
    """VSHE_PRECOND_ILUT: the device factorisation (IKJ with ILUT's two dropping rules inside
    the host-analysed pattern) reproduces the oracle's ILUT(20, 1e-3) (Saad Alg. 10.6): factor
    values at A's entries to 1e-11 of the row scale (0 where ILUT dropped the entry)."""
    name, P, A = prob
    S = gpu_ctx.system(A.rp, A.ci, A.v, A.rhs, precision="fp64", precond="ilut", ilut_entries=20, ilut_drop=1e-3)
    try:
        lu = S.factor_values()
    finally:
        S.free()
    rp, ci, flu = O.ilut_csr(A, 20, 1e-3)
    ref = np.zeros(A.nnz)
    for i in range(A.n):
        cols = ci[rp[i]:rp[i + 1]]
        mine = A.ci[A.rp[i]:A.rp[i + 1]]
        pos = np.searchsorted(cols, mine)
        hit = (pos < len(cols)) & (cols[np.minimum(pos, len(cols) - 1)] == mine)
        ref[A.rp[i]:A.rp[i + 1]] = np.where(hit, flu[rp[i] + np.minimum(pos, len(cols) - 1)], 0.0)
    scale = np.maximum(np.abs(ref), 1.0)
    assert np.max(np.abs(lu - ref) / scale) < 1e-11


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_ilut_solve(gpu_ctx, prob, precision):
    """ILUT(20, 1e-3) reaches 1e-10 with x within the 1e-7 parity bar and in no more
    iterations than ILU(0)."""
    name, P, A = prob
    xd = O.dense_solve(A, A.rhs) if A.n <= 4000 else O.csr_solve(A, A.rhs, tol=1e-14, maxit=20000)[0]
    x, st = gpu_ctx.solve_csr(A.rp, A.ci, A.v, A.rhs, precision=precision, precond="ilut", ilut_entries=20, ilut_drop=1e-3,
                              tol=1e-10, max_iters=4000)
    assert st["status"] == 0 and st["rel_residual"] < 1e-10, st
    assert np.linalg.norm(x - xd) / np.linalg.norm(xd) < 1e-7
    _, st0 = gpu_ctx.solve_csr(A.rp, A.ci, A.v, A.rhs, precision=precision, precond="ilu0", tol=1e-10, max_iters=4000)
    assert st["iterations"] <= st0["iterations"], (st, st0)


def test_ilut_long_rows_match_oracle(gpu_ctx):
    """ILUT(20, 1e-6) on a system whose first row's U part and last row's L part hold about 1500
    entries: the device's p-largest selection keeps what the oracle's ILUT keeps (factor values
    at A's entries to 1e-11 of the row scale), and the solve reaches 1e-10 with x within 1e-7
    of the direct solution."""
    A = cases.arrow_csr()
    p, tau = 20, 1e-6
    S = gpu_ctx.system(A.rp, A.ci, A.v, A.rhs, precision="fp64", precond="ilut", ilut_entries=p, ilut_drop=tau)
    try:
        lu = S.factor_values()
    finally:
        S.free()
    rp, ci, flu = O.ilut_csr(A, p, tau)
    ref = np.zeros(A.nnz)
    for i in range(A.n):
        cols = ci[rp[i]:rp[i + 1]]
        mine = A.ci[A.rp[i]:A.rp[i + 1]]
        pos = np.minimum(np.searchsorted(cols, mine), len(cols) - 1)
        ref[A.rp[i]:A.rp[i + 1]] = np.where(cols[pos] == mine, flu[rp[i] + pos], 0.0)
    assert np.count_nonzero(ref[A.rp[0]:A.rp[1]]) == p + 1 and np.count_nonzero(ref[A.rp[-2]:A.rp[-1]]) == p + 1
    scale = np.maximum(np.abs(ref), 1.0)
    assert np.max(np.abs(lu - ref) / scale) < 1e-11
    xd = O.dense_solve(A, A.rhs)
    x, st = gpu_ctx.solve_csr(A.rp, A.ci, A.v, A.rhs, precision="fp64", precond="ilut", ilut_entries=p, ilut_drop=tau,
                              tol=1e-10, max_iters=2000)
    assert st["status"] == 0 and st["rel_residual"] < 1e-10, st
    assert np.linalg.norm(x - xd) / np.linalg.norm(xd) < 1e-7


def test_sweep_modes_bitwise_equal(gpu_ctx, prob):
    """The triangular-sweep schedules (grid barrier per level, one launch per level, one CTA per
    system, barrier-free flow, one CTA per block) compute every row in the same order, so the iterates, the
    iteration count and x are bitwise the same whichever one runs."""
    name, P, A = prob
    out = {}
    for mode in ("persistent", "per_level", "per_system", "flow", "per_block"):
        x, st = gpu_ctx.solve_csr(A.rp, A.ci, A.v, A.rhs, precision="mixed", precond="ilu0", trsv=mode, tol=1e-10, max_iters=4000)
        assert st["status"] == 0 and st["rel_residual"] < 1e-10, (mode, st)
        out[mode] = (x, st)
    assert out["flow"][1]["sweep_mode"] == 4 and out["persistent"][1]["sweep_mode"] == 1
    x0, st0 = out["persistent"]
    for mode, (x, st) in out.items():
        assert st["iterations"] == st0["iterations"], (mode, st["iterations"], st0["iterations"])
        assert np.array_equal(x, x0), (mode, np.max(np.abs(x - x0)))


def test_per_block_sweep_bitwise_equal():
    """Block-ILU per energy slab on a 2D bar: the per-block sweep (one CTA per slab, factor
    slices staged through shared memory) computes every row as the grid-wide sweep does, so x and
    the iteration count are bitwise the same; AUTO picks it for a slab-blocked system; and a
    batch of such systems gives each member the x it gets alone."""
    ctx = gpu.Context(0)
    try:
        out = {}
        P = cases.oracle_problem(*cases.bar_small(L=3, nx=12, ny=5, n_energies=30))
        A = P.matrix(3)
        blocks = P.blocks()
        for mode in ("persistent", "per_block", "auto", "per_system"):
            for precision in ("mixed", "fp64"):
                x, st = ctx.solve_csr(A.rp, A.ci, A.v, A.rhs, precision=precision, precond="block_ilu0", ordering="multicolor",
                                      blocks=blocks, fill_level=1, trsv=mode, tol=1e-10, max_iters=4000)
                assert st["status"] == 0 and st["rel_residual"] < 1e-10, (mode, precision, st)
                out[(mode, precision)] = (x, st)
        assert out[("auto", "mixed")][1]["sweep_mode"] == 5 and out[("per_block", "fp64")][1]["sweep_mode"] == 5
        assert out[("persistent", "mixed")][1]["sweep_mode"] == 1 and out[("per_system", "mixed")][1]["sweep_mode"] == 3
        # each task kernel forced: one staged CTA, clusters of 2, 4 and 8 CTAs
        for kern in (0, 2, 4, 8):
            ctx.set_task_sweep(kern)
            for precision in ("mixed", "fp64"):
                x, st = ctx.solve_csr(A.rp, A.ci, A.v, A.rhs, precision=precision, precond="block_ilu0", ordering="multicolor",
                                      blocks=blocks, fill_level=1, trsv="per_block", tol=1e-10, max_iters=4000)
                assert st["sweep_ctas"] == max(kern, 1)
                out[("kernel%d" % kern, precision)] = (x, st)
        ctx.set_task_sweep(-1)
        for precision in ("mixed", "fp64"):
            x0, st0 = out[("persistent", precision)]
            for mode in ("per_block", "auto", "per_system", "kernel0", "kernel2", "kernel4", "kernel8"):
                x, st = out[(mode, precision)]
                assert st["iterations"] == st0["iterations"], (mode, precision, st["iterations"], st0["iterations"])
                assert np.array_equal(x, x0), (mode, precision, np.max(np.abs(x - x0)))
        # a batch of two slab-blocked bars and a 1D diode (swept as one task per system)
        probs = [P, cases.oracle_problem(*cases.bar_small(L=1, nx=10, ny=4, n_energies=24)),
                 cases.oracle_problem(*cases.diode_small(L=1, boxes=40))]
        mats = [Q.matrix(3) for Q in probs]
        opts = [dict(precond="block_ilu0", ordering="multicolor", blocks=probs[0].blocks(), fill_level=1),
                dict(precond="block_ilu0", ordering="multicolor", blocks=probs[1].blocks(), fill_level=1),
                dict(precond="block_ilu0", ordering="natural", blocks=np.array([0, mats[2].n], np.int64))]
        alone = [ctx.solve_csr(M.rp, M.ci, M.v, M.rhs, precision="mixed", tol=1e-10, max_iters=4000, **o)[0] for M, o in zip(mats, opts)]
        systems = [ctx.system(M.rp, M.ci, M.v, M.rhs, precision="mixed", tol=1e-10, max_iters=4000, **o) for M, o in zip(mats, opts)]
        try:
            stats = ctx.batch_solve(systems)
            for S, st, xa in zip(systems, stats, alone):
                assert st["status"] == 0 and st["rel_residual"] < 1e-10, st
                assert np.array_equal(S.x(), xa)
        finally:
            for S in systems:
                S.free()
    finally:
        ctx.close()


def test_flow_sweep_batch_equals_alone(gpu_ctx):
    """A batch of systems of uneven size swept by the barrier-free kernel gives each member the
    x it gets alone."""
    probs = [cases.oracle_problem(*cases.diode_small(L=L, boxes=b, bias=v)) for L, b, v in ((1, 30, 0.2), (3, 24, 0.5))]
    probs.append(cases.oracle_problem(*cases.bar_small(L=3, nx=10, ny=4, n_energies=24)))
    mats = [P.matrix(3) for P in probs]
    alone = []
    for A in mats:
        x, st = gpu_ctx.solve_csr(A.rp, A.ci, A.v, A.rhs, precision="mixed", trsv="flow")
        assert st["status"] == 0
        alone.append(x)
    systems = [gpu_ctx.system(A.rp, A.ci, A.v, A.rhs, precision="mixed", trsv="flow") for A in mats]
    try:
        stats = gpu_ctx.batch_solve(systems)
        for S, st, xa in zip(systems, stats, alone):
            assert st["status"] == 0 and st["rel_residual"] < 1e-10 and st["sweep_mode"] == 4
            assert np.array_equal(S.x(), xa)
    finally:
        for S in systems:
            S.free()

"""Failure paths, triggered without faulting the GPU: a device-side wait made to run out (a poll
limit of one), a non-positive odd diagonal from a device description without scattering, a
BiCGStab breakdown on a host-built system, and HBM-budget refusals.  After each, the context is
still usable."""
import numpy as np
import pytest

from vshe import devices as D
from vshe import gpu
import oracle_api as O
import cases

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("trsv", ["persistent", "flow"])
def test_wait_timeout_reported_and_context_reusable(trsv):
    """With a poll limit of one, the first grid-barrier or flow-poll wait that is not already
    satisfied gives up: the solve returns VSHE_E_TIMEOUT.  With the default limit restored, the
    same context solves the same system to the same x as a fresh context."""
    A = cases.oracle_problem(*cases.bar_small(L=3, nx=12, ny=5, n_energies=30)).matrix(3)
    kw = dict(precision="mixed", precond="ilu0", ordering="multicolor", trsv=trsv, tol=1e-10, max_iters=4000)
    ctx = gpu.Context(0)
    try:
        ctx.set_spin_limit(1)
        with pytest.raises(gpu.VsheError) as ei:
            ctx.solve_csr(A.rp, A.ci, A.v, A.rhs, **kw)
        assert ei.value.code == -10
        ctx.set_spin_limit(0)
        x, st = ctx.solve_csr(A.rp, A.ci, A.v, A.rhs, **kw)
        assert st["status"] == 0 and st["rel_residual"] < 1e-10
    finally:
        ctx.close()
    ctx2 = gpu.Context(0)
    try:
        x2, _ = ctx2.solve_csr(A.rp, A.ci, A.v, A.rhs, **kw)
        assert np.array_equal(x, x2)
    finally:
        ctx2.close()


def test_odd_diagonal_without_scattering(gpu_ctx):
    """Without phonon scattering the odd rows have no diagonal entry: the reference's elimination
    throws (she/eliminate.hpp:262-270), the oracle raises, the device returns VSHE_E_ODD_DIAGONAL."""
    dev, cfg = cases.diode_small(L=1, boxes=20)
    cfg.acoustic_phonon = False
    cfg.optical_phonon = False
    with pytest.raises(RuntimeError, match="Diagonal entry not positive"):
        O.OracleProblem(dev, cfg, O.golden_coupling(1))
    with pytest.raises(gpu.VsheError) as ei:
        gpu.SheProblem(gpu_ctx, dev, cfg, coupling=O.golden_coupling(1), precision="fp64", precond="ilu0")
    assert ei.value.code == -4
    # the context still serves a valid problem
    dev2, cfg2 = cases.diode_small(L=1, boxes=20)
    P = gpu.SheProblem(gpu_ctx, dev2, cfg2, coupling=O.golden_coupling(1), precision="fp64", precond="ilu0")
    try:
        st, fres = P.run()
        assert st["status"] == 0 and fres < 1e-9
    finally:
        P.free()


def test_breakdown_on_skew_system(gpu_ctx):
    """A = [[0, 1], [-1, 0]], b = (1, 1), no preconditioner, r^ = r_0: (r^, A r_0) = 0 exactly,
    so BiCGStab breaks down in its first step: VSHE_E_BREAKDOWN."""
    rp = np.array([0, 1, 2], np.int64)
    ci = np.array([1, 0], np.int32)
    v = np.array([1.0, -1.0])
    b = np.array([1.0, 1.0])
    with pytest.raises(gpu.VsheError) as ei:
        gpu_ctx.solve_csr(rp, ci, v, b, precision="fp64", precond="none", shadow="r0", tol=1e-10, max_iters=50)
    assert ei.value.code == -5


def test_budget_refusal_leaves_nothing_allocated():
    """A system or SHE problem whose estimated footprint exceeds the context's HBM budget is
    refused with VSHE_E_BUDGET before any allocation; so is a served request alone above the
    server's budget, whose result carries the code while the server goes on serving."""
    A = cases.oracle_problem(*cases.bar_small(L=3, nx=12, ny=5, n_energies=30)).matrix(3)
    dev_big, cfg_big = D.config2(nx=40, ny=10, n_energies=160, L=3)
    ctx = gpu.Context(0, hbm_budget=1 << 20)
    try:
        assert ctx.bytes_in_use() == 0
        with pytest.raises(gpu.VsheError) as ei:
            ctx.system(A.rp, A.ci, A.v, A.rhs, precision="mixed")
        assert ei.value.code == -8
        with pytest.raises(gpu.VsheError) as ei:
            gpu.SheProblem(ctx, dev_big, cfg_big, coupling=O.golden_coupling(3), precision="mixed", precond="ilu0")
        assert ei.value.code == -8
        assert ctx.bytes_in_use() == 0
    finally:
        ctx.close()
    ctx = gpu.Context(0)
    try:
        dev_small, cfg_small = cases.diode_small(L=1, boxes=20)
        srv = gpu.Server(ctx, hbm_budget=64 << 20, precision="mixed", precond="ilu0", tol=1e-10, max_iters=2000)
        try:
            t_big = srv.submit(dev_big, cfg_big, coupling=O.golden_coupling(3), ordering="multicolor", precond="block_ilu0")
            t_small = srv.submit(dev_small, cfg_small, coupling=O.golden_coupling(1))
            with pytest.raises(gpu.VsheError) as ei:
                srv.wait(t_big)
            assert ei.value.code == -8
            res, dens, cur = srv.wait(t_small)
            assert res["status"] == 0 and res["rel_residual"] < 1e-10
        finally:
            srv.close()
        assert ctx.bytes_in_use() == 0
    finally:
        ctx.close()


def test_footprint_bound_covers_the_allocation(gpu_ctx):
    """The admission bound computed from the host set-up is not below what the problem then holds
    on the device (1D diode, 2D bars at L = 1, 3, 5)."""
    for dev, cfg, kw in [(*cases.diode_small(L=1, boxes=60), dict(precond="ilu0")),
                         (*cases.bar_small(L=1, nx=14, ny=6, n_energies=40), dict(precond="block_ilu0", ordering="multicolor")),
                         (*cases.bar_small(L=3, nx=12, ny=5, n_energies=30), dict(precond="block_ilu0", ordering="multicolor", fill_level=1)),
                         (*cases.bar_small(L=5, nx=8, ny=4, n_energies=24), dict(precond="ilut", ilut_entries=20, ilut_drop=1e-3))]:
        before = gpu_ctx.bytes_in_use()
        P = gpu.SheProblem(gpu_ctx, dev, cfg, coupling=O.golden_coupling(cfg.max_expansion_order), precision="mixed", **kw)
        try:
            P.run()
            held = gpu_ctx.bytes_in_use() - before
            assert 0 < held <= P.info["bytes_estimate"], (dev.name, held, P.info["bytes_estimate"])
        finally:
            P.free()

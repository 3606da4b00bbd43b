"""Served stream (vshe_server_*): requests that arrive while others are on the GPU are admitted
as slots and memory free up, iterate together with them, and leave as they converge.  Each
result must be the same served alone and served in the mix: the solve's reductions are per
system and in a fixed order, so the check is bitwise on iterations, residuals, densities and
currents.  The mix also has to meet the oracle like a single solve (1e-10 bounds of
test_gpu_she: x-derived densities 5e-6, currents 5e-4 of the flux scale)."""
import numpy as np
import pytest

from vshe import devices as D
from vshe import gpu
import oracle_api as O
import cases

pytestmark = pytest.mark.gpu


def _mix():
    # 1D diodes of both orders and biases (natural ILU(0)) and a small 2D bar (node-coloured)
    return [(cases.diode_small(L=1, boxes=40, bias=0.3), dict(ordering="natural")),
            (cases.diode_small(L=3, boxes=30, bias=0.5), dict(ordering="natural")),
            (cases.bar_small(L=3, nx=12, ny=5, n_energies=30), dict(ordering="multicolor", precond="block_ilu0")),
            (cases.diode_small(L=1, boxes=60, bias=0.8), dict(ordering="natural")),
            (cases.diode_small(L=3, boxes=24, bias=0.1), dict(ordering="natural"))]


def _serve(ctx, items, max_active=0):
    srv = gpu.Server(ctx, max_active=max_active, precision="mixed", precond="ilu0", tol=1e-10, max_iters=4000, check_every=4)
    try:
        tickets = [srv.submit(dev, cfg, coupling=O.golden_coupling(cfg.max_expansion_order), **kw) for (dev, cfg), kw in items]
        return [srv.wait(t, 120000.0) for t in tickets]
    finally:
        srv.close()


def test_served_results_equal_alone_and_meet_oracle(gpu_ctx):
    items = _mix()
    mixed = _serve(gpu_ctx, items)
    for k, item in enumerate(items):
        alone = _serve(gpu_ctx, [item])[0]
        (res_m, dens_m, cur_m), (res_a, dens_a, cur_a) = mixed[k], alone
        assert res_m["status"] == 0 and res_m["rel_residual"] < 1e-10, res_m
        assert res_m["iterations"] == res_a["iterations"] and res_m["rel_residual"] == res_a["rel_residual"], (k, res_m, res_a)
        assert np.array_equal(dens_m, dens_a) and np.array_equal(cur_m, cur_a), k
        (dev, cfg), _ = item
        P = cases.oracle_problem(dev, cfg)
        A = P.matrix(3)
        xr, _ = O.csr_solve(A, A.rhs, precond=1, tol=1e-13, maxit=20000)
        _, dens_r, cur_r, _ = P.finish(xr)
        assert np.max(np.abs(dens_m - dens_r)) < 5e-6 * np.max(np.abs(dens_r))
        if len(cur_r):
            assert np.max(np.abs(cur_m - cur_r)) <= 5e-4 * cases.current_scale(dens_r, cur_r)


def test_server_admits_as_slots_free(gpu_ctx):
    """With two slots the five requests are served two at a time; the later ones queue."""
    out = _serve(gpu_ctx, _mix(), max_active=2)
    assert all(r["status"] == 0 for r, _, _ in out)
    assert max(r["queue_ms"] for r, _, _ in out) > 0.0


def test_stagnation_stop_frees_the_slot(gpu_ctx):
    """A 2D bar at L = 5 with block-ILU(0) per slab, where BiCGStab stalls (the oracle: no
    convergence on a 25 x 10 x 60 bar), ends early as not converged once its residual has not
    halved in 100 iterations, far below its iteration cap; the request queued behind it is
    served."""
    dev5, cfg5 = cases.bar_small(L=5, nx=25, ny=10, n_energies=60)
    dev1, cfg1 = cases.diode_small(L=1, boxes=40, bias=0.3)
    srv = gpu.Server(gpu_ctx, max_active=1, stagnation_iters=100, precision="mixed", precond="ilu0", tol=1e-10,
                     max_iters=3000, check_every=8)
    try:
        t5 = srv.submit(dev5, cfg5, coupling=O.golden_coupling(5), ordering="multicolor", precond="block_ilu0")
        t1 = srv.submit(dev1, cfg1, coupling=O.golden_coupling(1), ordering="natural")
        try:
            res5, _, _ = srv.wait(t5)
            code = res5["status"]
        except gpu.VsheError as e:  # a diverging iterate ends as a breakdown, also early
            code, res5 = e.code, None
        assert code in (-6, -5)
        if res5 is not None:
            assert res5["iterations"] < 1500 and res5["rel_residual"] >= 1e-10
        res1, _, _ = srv.wait(t1)
        assert res1["status"] == 0 and res1["rel_residual"] < 1e-10
    finally:
        srv.close()

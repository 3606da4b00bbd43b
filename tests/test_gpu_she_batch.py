"""Bias sweep / many devices solved as one batch (vshe_she_run_batch).

Each system's reductions are finished per system in a fixed order, and the triangular-solve
chunks never mix systems, so every result of a batched run must be bit-identical to the same
problem run alone.  The batch also has to meet the oracle like a single run.
"""
import numpy as np
import pytest

from vshe import devices as D
from vshe import gpu
import oracle_api as O
import cases

pytestmark = pytest.mark.gpu


def _sweep():
    # uneven sizes, both expansion orders, several biases (a small version of the seeded sweep)
    return [cases.diode_small(L=1, boxes=40, bias=0.0), cases.diode_small(L=3, boxes=30, bias=0.4),
            cases.diode_small(L=1, boxes=60, bias=0.8), cases.diode_small(L=3, boxes=24, bias=0.2),
            cases.bar_small(L=1, nx=10, ny=4, n_energies=30)]


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_batch_bitwise_equals_alone(gpu_ctx, precision):
    items = _sweep()
    alone = []
    for dev, cfg in items:
        G = gpu.SheProblem(gpu_ctx, dev, cfg, coupling=O.golden_coupling(cfg.max_expansion_order), precision=precision, precond="ilu0")
        st, fr = G.run()
        assert st["status"] == 0, st
        alone.append((st, fr) + G.results())
        G.free()
    probs = [gpu.SheProblem(gpu_ctx, dev, cfg, coupling=O.golden_coupling(cfg.max_expansion_order), precision=precision, precond="ilu0")
             for dev, cfg in items]
    try:
        for rep in range(2):  # second call reuses the cached schedule
            stats, fres, ms = gpu.she_run_batch(gpu_ctx, probs)
            assert ms > 0
            for k, G in enumerate(probs):
                st_a, fr_a, x_a, d_a, c_a = alone[k]
                assert stats[k]["status"] == 0 and stats[k]["iterations"] == st_a["iterations"], (k, stats[k], st_a)
                assert stats[k]["rel_residual"] == st_a["rel_residual"]
                assert fres[k] == fr_a
                x, d, c = G.results()
                assert np.array_equal(x, x_a) and np.array_equal(d, d_a) and np.array_equal(c, c_a), k
    finally:
        for G in probs:
            G.free()


def test_batch_meets_oracle(gpu_ctx):
    items = _sweep()[:3]
    probs = [gpu.SheProblem(gpu_ctx, dev, cfg, coupling=O.golden_coupling(cfg.max_expansion_order), precision="mixed", precond="ilu0")
             for dev, cfg in items]
    try:
        stats, fres, _ = gpu.she_run_batch(gpu_ctx, probs)
        for (dev, cfg), G, st, fr in zip(items, probs, stats, fres):
            assert st["status"] == 0 and st["rel_residual"] < 1e-10, st
            assert fr < 1e-9
            P = cases.oracle_problem(dev, cfg)
            A = P.matrix(3)
            xr = O.dense_solve(A, A.rhs)
            xf_r, dens_r, cur_r, _ = P.finish(xr)
            x, dens, cur = G.results()
            # bounds of a 1e-10 solve (test_gpu_she.BOUNDS): ten times the oracle's own deviation
            assert np.max(np.abs(x - xf_r)) <= 5e-6 * np.max(np.abs(xf_r))
            assert np.max(np.abs(dens - dens_r)) < 5e-6 * np.max(np.abs(dens_r))
            assert np.max(np.abs(dens - dens_r) / np.abs(dens_r)) < 5e-4
            assert np.max(np.abs(cur - cur_r)) <= 5e-4 * cases.current_scale(dens_r, cur_r)
    finally:
        for G in probs:
            G.free()


def test_batch_rejects_bad_handles(gpu_ctx):
    dev, cfg = cases.diode_small(L=1, boxes=20)
    G = gpu.SheProblem(gpu_ctx, dev, cfg, coupling=O.golden_coupling(1), precision="mixed", precond="ilu0")
    try:
        with pytest.raises(gpu.VsheError):
            gpu.she_run_batch(gpu_ctx, [G, G])
    finally:
        G.free()
    with pytest.raises(gpu.VsheError):
        gpu.she_run_batch(gpu_ctx, [G])  # freed

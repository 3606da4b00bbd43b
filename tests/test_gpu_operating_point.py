"""GPU parity at the operating points the benchmark measures (through the C ABI, against the
CPU oracle fed the reference's coupling tables).

* The 2D bar of the headline workload at its own operating point (0.8 V, 160 energies, L = 3,
  contacts 1e25 / channel 1e22 m^-3, seed-7 doping edges) on a 40 x 10 mesh, solved with the
  headline's preconditioner (block-ILU(1) per energy slab, node distance-2 colouring): reduced
  system bit-identical in pattern and within 1e-12 in values, x, densities and terminal currents
  within the bounds of a 1e-10 solve.  At 0.8 V the terminal current is not a near-equilibrium
  cancellation; the oracle's own 1e-10 solve puts it within 2.7e-9 of its 1e-13 solve, and the
  device's is asserted within 1e-7 of the current.
* The full 200 x 50 x 160 reduced system the benchmark solves against an oracle-made fixture
  (tests/golden/bar200x50x160_reduced.json, made by tests/golden/make_bar_fixture.py): SHA-256
  of the row offsets and column indices, and the values and rhs of 96 seeded rows to 1e-12.
* Eight of the 64 seeded diodes of the batched sweep, solved in one batch with the other 56,
  and the served stream's requests at L <= 3 below 6000 cells, each against the oracle.
"""
import hashlib
import json
import os

import numpy as np
import pytest

from vshe import devices as D
from vshe import gpu
import oracle_api as O
import cases

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
TOL = 1e-10
BX, BD = 5e-6, 5e-6   # x and density bounds of a 1e-10 solve (relative to the largest entry)


def _assert_same(csr, gpu_tuple, rel=1e-12):
    rp, ci, v, b = gpu_tuple
    assert np.array_equal(rp, csr.rp), "row offsets differ"
    assert np.array_equal(ci, csr.ci), "column indices differ"
    assert np.all(np.abs(v - csr.v) <= rel * np.abs(csr.v)), np.max(np.abs(v - csr.v) / np.maximum(np.abs(csr.v), 1e-300))
    assert np.all(np.abs(b - csr.rhs) <= rel * np.abs(csr.rhs)), np.max(np.abs(b - csr.rhs))


def _oracle_reference(P):
    A = P.matrix(3)
    xr, sr = O.csr_solve(A, A.rhs, precond=1, tol=1e-13, maxit=20000)
    assert sr["rc"] == 0, sr
    xf, dens, cur, _ = P.finish(xr)
    return xf, dens, cur


def _check(P, x, dens, cur, cur_rel=None):
    xf_r, dens_r, cur_r = _oracle_reference(P)
    assert np.max(np.abs(x - xf_r)) <= BX * np.max(np.abs(xf_r))
    assert np.max(np.abs(dens - dens_r)) < BD * np.max(np.abs(dens_r))
    assert np.max(np.abs(dens - dens_r) / np.abs(dens_r)) < 100 * BD
    if len(cur_r):
        scale = cases.current_scale(dens_r, cur_r)
        assert np.max(np.abs(cur - cur_r[:len(cur)])) <= 5e-4 * scale
        if cur_rel is not None:
            assert np.max(np.abs(cur - cur_r[:len(cur)])) <= cur_rel * np.max(np.abs(cur_r)), (cur, cur_r)


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_bar_at_operating_point(gpu_ctx, precision):
    dev, cfg = D.config2(nx=40, ny=10, n_energies=160, L=3)
    cpl = O.golden_coupling(3)
    P = O.OracleProblem(dev, cfg, cpl)
    G = gpu.SheProblem(gpu_ctx, dev, cfg, coupling=cpl, precision=precision, precond="block_ilu0", ordering="multicolor",
                       fill_level=1, tol=TOL, max_iters=20000, check_every=16)
    try:
        assert G.info["n_energies"] == P.NH == 160
        assert G.info["n_even"] == P.n_even and G.info["n_odd"] == P.n_odd
        G.assemble(3)
        _assert_same(P.matrix(3), G.export("reduced"))
        assert np.array_equal(G.blocks(), P.blocks())
        st, full_res = G.run()
        assert st["status"] == 0 and st["rel_residual"] < TOL, st
        assert st["sweep_mode"] == 5, st  # one CTA per energy slab
        assert full_res < 10 * TOL
        x, dens, cur = G.results()
        _check(P, x, dens, cur, cur_rel=1e-7)
    finally:
        G.free()


def _sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def test_full_bar_reduced_system_matches_fixture(gpu_ctx):
    fx = json.load(open(os.path.join(HERE, "golden", "bar200x50x160_reduced.json")))
    dev, cfg = D.config2(nx=fx["nx"], ny=fx["ny"], n_energies=fx["n_energies"], L=fx["L"])
    G = gpu.SheProblem(gpu_ctx, dev, cfg, coupling=O.golden_coupling(fx["L"]), precision="mixed", precond="block_ilu0",
                       ordering="multicolor", fill_level=1)
    try:
        assert G.info["n_even"] == fx["n"] and G.info["nnz_reduced"] == fx["nnz"]
        assert G.info["n_odd"] == fx["n_odd"] and G.info["nnz_full"] == fx["nnz_full"]
        G.assemble(3)
        rp, ci, v, b = G.export("reduced")
        assert _sha(rp.astype("<i8")) == fx["sha256_row_ptr"]
        assert _sha(ci.astype("<i4")) == fx["sha256_col"]
        for row in fx["rows"]:
            i = row["row"]
            a, e = int(rp[i]), int(rp[i + 1])
            assert ci[a:e].tolist() == row["col"]
            ref = np.array(row["val"])
            assert np.all(np.abs(v[a:e] - ref) <= 1e-12 * np.abs(ref)), (i, np.max(np.abs(v[a:e] - ref) / np.abs(ref)))
            assert abs(b[i] - row["rhs"]) <= 1e-12 * abs(row["rhs"])
    finally:
        G.free()


def test_sweep_diodes_match_oracle(gpu_ctx):
    """The 64 seeded diodes of the batched sweep solved as one batch (vshe_she_run_batch); eight
    of them (every eighth) are checked against the oracle."""
    items = D.config3()
    probs = [gpu.SheProblem(gpu_ctx, dev, cfg, coupling=O.golden_coupling(cfg.max_expansion_order), precision="mixed",
                            precond="ilu0", ordering="natural", tol=TOL, max_iters=20000) for dev, cfg in items]
    try:
        stats, fres, _ = gpu.she_run_batch(gpu_ctx, probs)
        for k in range(0, 64, 8):
            dev, cfg = items[k]
            st = stats[k]
            assert st["status"] == 0 and st["rel_residual"] < TOL, (k, st)
            assert fres[k] < 10 * TOL
            P = O.OracleProblem(dev, cfg, O.golden_coupling(cfg.max_expansion_order))
            assert probs[k].info["n_even"] == P.n_even and probs[k].info["nnz_reduced"] == P.nnz[3]
            x, dens, cur = probs[k].results()
            _check(P, x, dens, cur)
    finally:
        for p in probs:
            p.free()


def test_served_requests_match_oracle(gpu_ctx):
    """The seed-23 served stream's requests at L <= 3 with fewer than 6000 cells (the 1D diodes
    and four 2D bars), submitted together to the continuous-batching server; each result against
    the oracle."""
    items = [(dev, cfg) for _, dev, cfg in D.config4(24, rate=200.0) if cfg.max_expansion_order <= 3 and dev.n_cells < 6000]
    assert len(items) >= 20
    cpl = {L: O.golden_coupling(L) for L in (1, 3)}
    srv = gpu.Server(gpu_ctx, precision="mixed", precond="ilu0", tol=TOL, max_iters=4000, check_every=8)
    try:
        tickets = []
        for dev, cfg in items:
            kw = dict(ordering="natural", precond="ilu0") if dev.dim == 1 else dict(ordering="multicolor", precond="block_ilu0")
            tickets.append(srv.submit(dev, cfg, coupling=cpl[cfg.max_expansion_order], **kw))
        results = [srv.wait(t) for t in tickets]
    finally:
        srv.close()
    for (dev, cfg), (res, dens, cur) in zip(items, results):
        assert res["status"] == 0 and res["rel_residual"] < TOL, (dev.name, res)
        P = O.OracleProblem(dev, cfg, cpl[cfg.max_expansion_order])
        xf_r, dens_r, cur_r = _oracle_reference(P)
        assert np.max(np.abs(dens - dens_r)) < BD * np.max(np.abs(dens_r)), dev.name
        assert np.max(np.abs(dens - dens_r) / np.abs(dens_r)) < 100 * BD, dev.name
        if len(cur_r):
            assert np.max(np.abs(cur - cur_r[:len(cur)])) <= 5e-4 * cases.current_scale(dens_r, cur_r), dev.name

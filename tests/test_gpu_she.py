"""Device-side SHE assembly, odd elimination, normalisation and post-processing
(through the C ABI) against the CPU oracle, fed the reference's own coupling tables.

Bar: the sparsity patterns (row offsets and column indices) are bit-identical;
values and right-hand sides agree to 1e-12 relative per entry.  Solutions are
compared with the oracle's 1e-13 solve; the bounds for a solve to a relative
residual `tol` are ten times what the oracle's own solve to that `tol` deviates
on these cases (x: 4.3e-7 at 1e-10, 3.1e-9 at 1e-12 of max|x|; currents: 3.8e-5
and 2.2e-7 of max|I|): the systems are ill-conditioned, so a 1e-10 residual
pins x to a few 1e-7 only.
"""
import numpy as np
import pytest

from vshe import devices as D
from vshe import gpu
import oracle_api as O
import cases

pytestmark = pytest.mark.gpu


def _cases():
    return [
        ("resistor2d", *cases.resistor_2d()),
        ("diode_L1", *cases.diode_small(L=1, boxes=40)),
        ("diode_L3", *cases.diode_small(L=3, boxes=30)),
        ("bar_L3", *cases.bar_small(L=3, nx=12, ny=5, n_energies=30)),
        ("bar_L5", *cases.bar_small(L=5, nx=8, ny=4, n_energies=24)),
        ("bar_L1", *cases.bar_small(L=1, nx=14, ny=6, n_energies=40)),
    ]


CASES = _cases()


@pytest.fixture(scope="module", params=CASES, ids=[c[0] for c in CASES])
def pair(request, gpu_ctx):
    name, dev, cfg = request.param
    cpl = O.golden_coupling(cfg.max_expansion_order)
    P = O.OracleProblem(dev, cfg, cpl)
    G = gpu.SheProblem(gpu_ctx, dev, cfg, coupling=cpl, precision="mixed", precond="ilu0")
    yield name, P, G
    G.free()


def _assert_same(csr, gpu_tuple, rel=1e-12):
    rp, ci, v, b = gpu_tuple
    assert np.array_equal(rp, csr.rp), "row offsets differ"
    assert np.array_equal(ci, csr.ci), "column indices differ"
    scale = np.abs(csr.v)
    assert np.all(np.abs(v - csr.v) <= rel * scale), np.max(np.abs(v - csr.v) / np.maximum(scale, 1e-300))
    bs = np.abs(csr.rhs)
    assert np.all(np.abs(b - csr.rhs) <= rel * np.maximum(bs, 1e-300 * 0 + bs)), np.max(np.abs(b - csr.rhs))


def test_sizes(pair):
    name, P, G = pair
    assert G.info["n_energies"] == P.NH
    assert G.info["n_even"] == P.n_even and G.info["n_odd"] == P.n_odd


def test_full_system_parity(pair):
    name, P, G = pair
    G.assemble(1)
    _assert_same(P.matrix(1), G.export("full"))


def test_eliminated_system_parity(pair):
    name, P, G = pair
    G.assemble(2)
    _assert_same(P.matrix(2), G.export("reduced"))


def test_normalised_system_parity(pair):
    name, P, G = pair
    G.assemble(3)
    _assert_same(P.matrix(3), G.export("reduced"))
    s, f = G.scaling()
    s_r, f_r = P.scaling()
    assert np.all(np.abs(s - s_r) <= 1e-12 * np.abs(s_r))
    assert np.all(np.abs(f - f_r) <= 1e-12 * np.abs(f_r))


def test_end_to_end(pair):
    name, P, G = pair
    st, full_res = G.run()
    _check_end_to_end(P, G, st, full_res, tol=1e-10)


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_end_to_end_tight(gpu_ctx, precision):
    """At a 1e-12 residual the distribution function, densities and currents pin down tightly."""
    dev, cfg = cases.bar_small(L=3, nx=12, ny=5, n_energies=30)
    cpl = O.golden_coupling(3)
    P = O.OracleProblem(dev, cfg, cpl)
    G = gpu.SheProblem(gpu_ctx, dev, cfg, coupling=cpl, precision=precision, precond="block_ilu0",
                       ordering="multicolor", tol=1e-12, max_iters=4000)
    try:
        st, full_res = G.run()
        _check_end_to_end(P, G, st, full_res, tol=1e-12)
    finally:
        G.free()


def test_end_to_end_multicolour(gpu_ctx):
    """The node-coloured ILU(0) ordering (2D) reaches the same solution."""
    dev, cfg = cases.bar_small(L=3, nx=12, ny=5, n_energies=30)
    cpl = O.golden_coupling(3)
    P = O.OracleProblem(dev, cfg, cpl)
    G = gpu.SheProblem(gpu_ctx, dev, cfg, coupling=cpl, precision="mixed", precond="ilu0", ordering="multicolor")
    try:
        st, full_res = G.run()
        _check_end_to_end(P, G, st, full_res, tol=1e-10)
    finally:
        G.free()


def test_end_to_end_ilut_L5(gpu_ctx):
    """A 2D bar at L = 5, where ILU(0) in any order stalls (the oracle: no convergence in 3000
    iterations on a 25 x 10 x 60 bar), solved with the ILUT-pattern preconditioner."""
    dev, cfg = cases.bar_small(L=5, nx=8, ny=4, n_energies=24)
    cpl = O.golden_coupling(5)
    P = O.OracleProblem(dev, cfg, cpl)
    G = gpu.SheProblem(gpu_ctx, dev, cfg, coupling=cpl, precision="mixed", precond="ilut", ilut_entries=20, ilut_drop=1e-3,
                       tol=1e-10, max_iters=4000)
    try:
        st, full_res = G.run()
        _check_end_to_end(P, G, st, full_res, tol=1e-10)
    finally:
        G.free()


# (x, density, current) bounds per solve tolerance, relative to the largest entry
BOUNDS = {1e-10: (5e-6, 5e-6, 5e-4), 1e-12: (5e-8, 5e-8, 5e-6)}


def _check_end_to_end(P, G, st, full_res, tol):
    bx, bd, bc = BOUNDS[tol]
    assert st["status"] == 0 and st["rel_residual"] < tol, st
    assert full_res < 10 * tol
    x, dens, cur = G.results()
    A = P.matrix(3)
    xr, _ = O.csr_solve(A, A.rhs, precond=1, tol=1e-13, maxit=20000)
    xf_r, dens_r, cur_r, res_r = P.finish(xr)
    assert np.max(np.abs(x - xf_r)) <= bx * np.max(np.abs(xf_r))
    # densities: relative to the largest (contact) density, and per cell 100x that (the
    # channel is ~1e3 below the contacts)
    assert np.max(np.abs(dens - dens_r)) < bd * np.max(np.abs(dens_r))
    assert np.max(np.abs(dens - dens_r) / np.abs(dens_r)) < 100 * bd
    if len(cur_r):
        # currents are the small anisotropic part of f; near equilibrium they are a cancellation
        # of one-way fluxes (cases.current_scale)
        assert np.max(np.abs(cur - cur_r[:len(cur)])) <= bc * cases.current_scale(dens_r, cur_r)


def test_config1_diode_matches_oracle(gpu_ctx):
    """The reference's own CPU-runnable case: the 1D n+/n/n+ diode 50/150/50 nm, 1e25/1e21/1e25
    m^-3, 250 boxes, L = 1, spacing hbar*omega_op/4, 1.5 eV kinetic range, 0.5 V, with the
    preconditioner the reference's serial solver really runs (natural-order ILU(0); the ILUT
    that the benchmark configuration names needs 5896 iterations here on the oracle, against
    19).  Assembled system bit-identical in pattern and to 1e-12 in values; terminal currents
    and densities within 1e-8 of the oracle's 1e-14 solve after a 1e-14 solve on the device."""
    dev, cfg = D.config1()
    cpl = O.golden_coupling(1)
    P = O.OracleProblem(dev, cfg, cpl)
    G = gpu.SheProblem(gpu_ctx, dev, cfg, coupling=cpl, precision="fp64", precond="ilu0", ordering="natural",
                       tol=1e-14, max_iters=4000)
    try:
        G.assemble(3)
        _assert_same(P.matrix(3), G.export("reduced"))
        st, full_res = G.run()
        assert st["status"] == 0 and st["rel_residual"] < 1e-14, st
        A = P.matrix(3)
        xr, sr = O.csr_solve(A, A.rhs, precond=1, tol=1e-14, maxit=20000)
        assert sr["rc"] == 0, sr
        _, dens_r, cur_r, _ = P.finish(xr)
        x, dens, cur = G.results()
        assert np.max(np.abs(cur - cur_r)) <= 1e-8 * np.max(np.abs(cur_r))
        assert np.max(np.abs(dens - dens_r) / dens_r) < 1e-8
    finally:
        G.free()

"""Device-side SHE assembly, odd elimination, normalisation and post-processing
(through the C ABI) against the CPU oracle, fed the reference's own coupling tables.

Bar: the sparsity patterns (row offsets and column indices) are bit-identical;
values and right-hand sides agree to 1e-12 relative per entry; terminal
currents to 1e-8 relative.
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
    _check_end_to_end(P, G, st, full_res)


def test_end_to_end_multicolour(gpu_ctx):
    """The node-coloured ILU(0) ordering (2D) reaches the same solution."""
    dev, cfg = cases.bar_small(L=3, nx=12, ny=5, n_energies=30)
    cpl = O.golden_coupling(3)
    P = O.OracleProblem(dev, cfg, cpl)
    G = gpu.SheProblem(gpu_ctx, dev, cfg, coupling=cpl, precision="mixed", precond="ilu0", ordering="multicolor")
    try:
        st, full_res = G.run()
        _check_end_to_end(P, G, st, full_res)
    finally:
        G.free()


def _check_end_to_end(P, G, st, full_res):
    assert st["status"] == 0 and st["rel_residual"] < 1e-10, st
    assert full_res < 1e-9
    x, dens, cur = G.results()
    A = P.matrix(3)
    xr, _ = O.csr_solve(A, A.rhs, precond=1, tol=1e-13, maxit=20000)
    xf_r, dens_r, cur_r, res_r = P.finish(xr)
    assert np.max(np.abs(x - xf_r)) <= 1e-7 * np.max(np.abs(xf_r))
    # densities: 1e-7 of the largest (contact) density; the channel is ~1e3 below it, so per
    # cell the bar at a 1e-10 residual is 1e-5
    assert np.max(np.abs(dens - dens_r)) < 1e-7 * np.max(np.abs(dens_r))
    assert np.max(np.abs(dens - dens_r) / np.abs(dens_r)) < 1e-5
    if len(cur_r):
        # currents are the small anisotropic part: 1e-5 at a 1e-10 solve (1e-8 at 1e-12, see
        # test_gpu_solver).  At equilibrium (the resistor) the net current is round-off of the
        # one-way fluxes; there the bar is an absolute 1e-9 A/m.
        assert np.max(np.abs(cur - cur_r[:len(cur)])) <= max(1e-5 * np.max(np.abs(cur_r)), 1e-9)

"""The outer loop's Gummel update of the potential on the device (vshe_poisson_*, through the C
ABI) against the oracle's restatement (oracle/poisson_oracle.cpp, viennashe/assemble.hpp:165-345,
viennashe/simulator.hpp:606-647), and a short Gummel loop of device SHE solves and device
Poisson updates on a 1D diode, step by step against the oracle's Poisson step."""
import dataclasses

import numpy as np
import pytest

from vshe import devices as D
from vshe import gpu
import oracle_api as O

pytestmark = pytest.mark.gpu

NI = 1.08e16  # physics/constants.hpp:78


def oxide_diode():
    dev = D.nin_diode_1d(boxes=40, bias=0.2)
    dev.cell_material[20:30] = 1  # SiO2
    return dev


CASES = {
    "bar": lambda: D.nin_bar_2d(nx=40, ny=10, bias=0.8),
    "diode": lambda: D.nin_diode_1d(boxes=120, bias=0.5),
    "oxide": oxide_diode,
    "mosfet": lambda: D.mosfet_2d(nx=30, ny=10),
}


def inputs(dev, seed):
    rng = np.random.default_rng(seed)
    psi = dev.potential + rng.normal(0.0, 0.005, dev.n_cells) * (dev.contact_id < 0)
    n = dev.doping_n * rng.uniform(0.2, 1.5, dev.n_cells)
    p = NI * NI / np.maximum(n, 1.0)
    return psi, n, p


@pytest.mark.parametrize("name", sorted(CASES))
def test_assembly_and_update_match_oracle(gpu_ctx, name):
    dev = CASES[name]()
    fc = D.facet_centres(dev)
    psi, n, p = inputs(dev, 5)
    G = gpu.PoissonProblem(gpu_ctx, dev, fc, precond="ilu0", tol=1e-13, max_iters=20000)
    try:
        out, st = G.update(psi, n, p, damping=0.6)
        rp, ci, v, b = G.export()
    finally:
        G.free()
    ref_out, dpsi, M = O.poisson_update(dev, fc, psi, n, p, damping=0.6, tol=1e-13)
    assert np.array_equal(rp, M.rp) and np.array_equal(ci, M.ci)
    assert np.max(np.abs(v - M.v)) <= 1e-13 * np.max(np.abs(M.v))
    assert np.max(np.abs(b - M.rhs)) <= 1e-12 * np.max(np.abs(M.rhs))
    assert st["status"] == 0 and st["rel_residual"] < 1e-13
    assert abs(st["rhs_norm"] - np.linalg.norm(M.rhs)) <= 1e-12 * np.linalg.norm(M.rhs)
    # two solves of one system to a 1e-13 residual differ by up to its condition number times
    # that (about 1e6 on the MOSFET, whose gate and body differ by 1 V over 1e23 m^-3 doping)
    assert abs(st["update_norm"] - np.linalg.norm(dpsi)) <= 1e-6 * np.linalg.norm(dpsi)
    contact = dev.contact_id >= 0
    assert np.array_equal(out[contact], psi[contact] * 0.4 + dev.potential[contact] * 0.6)
    assert np.max(np.abs(out - ref_out)) <= 1e-6 * np.max(np.abs(dpsi))


def test_errors(gpu_ctx):
    dev = D.nin_diode_1d(boxes=20)
    fc = D.facet_centres(dev)
    G = gpu.PoissonProblem(gpu_ctx, dev, fc)
    try:
        psi, n, p = inputs(dev, 1)
        n[3] = np.nan
        with pytest.raises(gpu.VsheError) as e:
            G.update(psi, n, p)
        assert e.value.code == -3  # VSHE_E_NAN
        with pytest.raises(gpu.VsheError):
            G.update(psi, inputs(dev, 1)[1], p, damping=0.0)
    finally:
        G.free()
    bad = D.nin_diode_1d(boxes=20)
    bad.cell_material[7] = D.METAL  # a metal cell that is not a contact has no permittivity
    with pytest.raises(gpu.VsheError):
        gpu.PoissonProblem(gpu_ctx, bad, D.facet_centres(bad))


def test_gummel_loop_on_device_follows_oracle_steps(gpu_ctx):
    """Three Gummel iterations: SHE on the device for the current potential (vshe_she_*),
    its densities into the device Poisson update (damping 0.5); every Poisson step equals the
    oracle's step from the same densities."""
    dev0 = D.nin_diode_1d(boxes=100, bias=0.3)
    cfg = D.SheConfig(max_expansion_order=1, energy_spacing=D.HBAR_OMEGA_OP / 4.0, min_kinetic_energy_range=1.0 * D.Q)
    fc = D.facet_centres(dev0)
    G = gpu.PoissonProblem(gpu_ctx, dev0, fc, precond="ilu0", tol=1e-13, max_iters=20000)
    psi = dev0.potential.copy()
    norms = []
    try:
        for it in range(3):
            dev = dataclasses.replace(dev0, potential=psi.copy())
            S = gpu.SheProblem(gpu_ctx, dev, cfg, precision="fp64", precond="ilu0", ordering="natural", tol=1e-12, max_iters=20000)
            try:
                st, _ = S.run()
                assert st["status"] == 0, st
                _, dens, _ = S.results()
            finally:
                S.free()
            n = np.where(dev0.contact_id < 0, dens, dev0.doping_n)
            p = NI * NI / np.maximum(n, 1.0)
            new, pst = G.update(psi, n, p, damping=0.5)
            ref, dpsi, _ = O.poisson_update(dev0, fc, psi, n, p, damping=0.5, tol=1e-13)
            assert np.max(np.abs(new - ref)) <= 1e-6 * max(np.max(np.abs(dpsi)), 1e-12)
            assert np.all(np.isfinite(new))
            norms.append(pst["rhs_norm"])
            psi = new
    finally:
        G.free()
    assert len(norms) == 3 and all(np.isfinite(norms))


def test_gummel_solve_matches_oracle_loop(gpu_ctx):
    """vshe_gummel_solve (device SHE + device Poisson, the reference's damping and stopping rules)
    against the oracle's restatement of the same loop: the same iteration at which the potential
    increment falls below tol, the same norms per iteration, the same final potential and
    density.  (Past about 1e-6 V the increments of this loop stop falling on both sides: the
    energy grid is rebuilt for every potential.)"""
    dev = D.nin_diode_1d(boxes=60, bias=0.3)
    cfg = D.SheConfig(max_expansion_order=1, energy_spacing=D.HBAR_OMEGA_OP / 4.0, min_kinetic_energy_range=1.0 * D.Q)
    n0 = dev.doping_n.copy()
    p0 = NI * NI / n0
    cpl = O.golden_coupling(1)
    psi, dens, cur, hist, st = gpu.gummel_solve(gpu_ctx, dev, cfg, n0, p0, coupling=cpl, tol=3e-2, damping=0.3,
                                                max_iters=100, precision="fp64", precond="ilu0", ordering="natural")
    r_psi, r_n, r_cur, r_hist = O.gummel_solve(dev, cfg, cpl, n0, p0, max_iters=100, tol=3e-2, damping=0.3)
    assert st["rc"] == 0 and st["status"] == 0, st
    assert st["iterations"] == len(r_hist) < 100
    assert np.allclose(hist[:, 0], r_hist[:, 0], rtol=1e-6, atol=0)
    assert np.allclose(hist[:, 1], r_hist[:, 1], rtol=1e-6, atol=0)
    assert hist[-2, 1] < 3e-2  # stopped one undamped update after the increment fell below tol
    assert np.max(np.abs(psi - r_psi)) <= 1e-7 * np.max(np.abs(r_psi))
    semi = dev.contact_id < 0
    assert np.max(np.abs(dens[semi] - r_n[semi]) / r_n[semi]) <= 1e-6
    assert np.max(np.abs(cur - r_cur)) <= 1e-5 * np.max(np.abs(r_cur))

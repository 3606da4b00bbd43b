"""The CPU oracle pinned against the reference's own known answers and invariants.

Reference tests restated here:
  * tests/src/spherical_harmonics_iter.cpp:62-117 -- harmonic index sequences for L = 3;
  * tests/src/spherical_harmonics.cpp:103-203 -- coupling selection rule |l - l'| = 1;
  * tests/src/equilibrium_resistor.cpp:121-198 -- zero bias gives a Maxwellian f_00 (1e-3)
    and vanishing first-order coefficients;
  * tests/src/ushape_2d.cpp:178-201 -- terminal currents conserve (|I_L + I_R| / max < 1e-5).
"""
import math

import numpy as np
import pytest

from vshe import devices as D
import oracle_api as O
import cases


def test_harmonics_iterator_kat():
    # spherical_harmonics_iter.cpp:62-117
    assert O.harmonics(3, "all") == list(range(16))
    assert O.harmonics(3, "even") == [0, 4, 5, 6, 7, 8]
    assert O.harmonics(3, "odd") == [1, 2, 3, 9, 10, 11, 12, 13, 14, 15]
    # counts per node: 1/3, 6/10, 15/21 (even/odd) for L = 1, 3, 5
    for L, e, o in ((1, 1, 3), (3, 6, 10), (5, 15, 21)):
        assert len(O.harmonics(L, "even")) == e and len(O.harmonics(L, "odd")) == o


@pytest.mark.parametrize("L", [1, 3, 5, 7])
def test_coupling_tables_selection_rule(L):
    cpl = O.golden_coupling(L)
    D2 = (L + 1) ** 2
    lm = [(l, m) for l in range(L + 1) for m in range(-l, l + 1)]
    for t in range(6):
        nz = np.argwhere(cpl.data[t] != 0)
        for i, j in nz:
            assert abs(lm[i][0] - lm[j][0]) == 1
    # a_{x,y,z} are symmetric; pattern(b) is inside pattern(a) (so a zero drift
    # coefficient never creates a new matrix entry)
    for t in range(3):
        assert np.array_equal(cpl.data[t], cpl.data[t].T)
        assert np.all((cpl.data[t + 3] != 0) <= (cpl.data[t] != 0))


def test_energy_grid_and_phonon_snap():
    dev, cfg = cases.diode_small()
    P = cases.oracle_problem(dev, cfg)
    H, sc, sf, w = P.energies()
    # she/setup_energies.hpp:108-120
    semi = dev.cell_material == 0
    dphi = dev.potential[semi].max() - dev.potential[semi].min()
    rng = D.Q * dphi + 2 * cfg.energy_spacing + cfg.min_kinetic_energy_range
    assert P.NH == int(rng / cfg.energy_spacing) + 1
    assert np.allclose(np.diff(H), cfg.energy_spacing, rtol=1e-9)
    # optical phonon energy snapped to the grid: 62 meV with spacing 15.5 meV -> 4 steps
    assert w == pytest.approx(4 * cfg.energy_spacing, rel=1e-12)
    # band edge shift on facets is the mean of its two cells
    fc = dev.facet_cells
    inner = fc[:, 1] >= 0
    assert np.allclose(sf[inner], 0.5 * (sc[fc[inner, 0]] + sc[fc[inner, 1]]))


@pytest.mark.parametrize("T", [300.0, 400.0])
def test_equilibrium_maxwellian(T):
    dev, cfg = cases.resistor_2d(T=T)
    P = cases.oracle_problem(dev, cfg)
    A = P.matrix(3)
    x = O.dense_solve(A, A.rhs) if A.n <= 1500 else O.csr_solve(A, A.rhs, tol=1e-14)[0]
    xf, dens, cur, res = P.finish(x)
    assert res < 1e-9
    ic, jf, oc, of, bc = P.mapping()
    H, sc, sf, w = P.energies()
    NH = P.NH
    kT = D.KB * T
    for c in range(dev.n_cells):
        base = ic[c * NH + 1]
        assert base >= 0
        for h in range(1, NH - 1):
            u = ic[c * NH + h]
            if u < 0:
                continue
            ek = H[h] - sc[c]
            ref = math.exp(-ek / kT) * xf[base]
            # equilibrium_resistor.cpp:135-147, relative tolerance 1e-3 (fuzzy_equal)
            assert abs(xf[u] - ref) <= 1e-3 * max(abs(xf[u]), abs(ref))
    # first-order (odd) coefficients vanish in equilibrium
    odd = xf[P.n_even:]
    assert np.max(np.abs(odd)) <= 1e-10 * np.max(np.abs(xf[:P.n_even]))


def test_terminal_current_conservation_1d():
    dev, cfg = D.config1()
    P = cases.oracle_problem(dev, cfg)
    A = P.matrix(3)
    x, st = O.csr_solve(A, A.rhs, precond=1, tol=1e-13, maxit=5000)
    assert st["rc"] == 0
    xf, dens, cur, res = P.finish(x)
    assert res < 1e-9
    # ushape_2d.cpp:196
    assert abs(cur[0] + cur[1]) / max(abs(cur[0]), abs(cur[1])) < 1e-5
    # density is positive and the contact density matches the doping order of magnitude
    assert np.all(dens > 0)
    assert 1e24 < dens[0] < 1e26


def test_reduced_system_solves_full_system():
    dev, cfg = cases.bar_small(L=3, nx=10, ny=4, n_energies=30)
    P = cases.oracle_problem(dev, cfg)
    A = P.matrix(3)
    x = O.dense_solve(A, A.rhs) if A.n <= 3000 else O.csr_solve(A, A.rhs, tol=1e-14, maxit=20000)[0]
    xf, dens, cur, res = P.finish(x)
    assert res < 1e-8
    # the unscaled, recovered solution satisfies the full (even + odd) system directly
    F = P.matrix(1)
    r = O.spmv(F, xf) - F.rhs
    assert np.linalg.norm(r) / np.linalg.norm(F.rhs) < 1e-8


def test_pattern_rules():
    dev, cfg = cases.bar_small(L=3, nx=8, ny=4, n_energies=30)
    P = cases.oracle_problem(dev, cfg)
    F = P.matrix(1)
    ne = P.n_even
    # she/eliminate.hpp:195-212: rows >= n_even - 1 carry no explicit zeros
    for i in range(ne - 1, F.n):
        assert np.all(F.v[F.rp[i]:F.rp[i + 1]] != 0.0)
    # S^oo is diagonal with a positive diagonal
    for i in range(ne, F.n):
        cols = F.ci[F.rp[i]:F.rp[i + 1]]
        vals = F.v[F.rp[i]:F.rp[i + 1]]
        odd = cols >= ne
        assert np.array_equal(cols[odd], [i]) and vals[odd][0] > 0
    # normalised reduced system: ascending columns, diagonal present, unit row 2-norms,
    # positive diagonal (linalg_util.hpp:202-282)
    A = P.matrix(3)
    for i in range(A.n):
        cols = A.ci[A.rp[i]:A.rp[i + 1]]
        vals = A.v[A.rp[i]:A.rp[i + 1]]
        assert np.all(np.diff(cols) > 0)
        assert i in cols
        assert abs(np.linalg.norm(vals) - 1.0) < 1e-12
        assert vals[list(cols).index(i)] > 0


def test_ilu0_block_variants_solve():
    dev, cfg = cases.bar_small(L=3, nx=10, ny=4, n_energies=30)
    P = cases.oracle_problem(dev, cfg)
    A = P.matrix(3)
    xd = O.dense_solve(A, A.rhs)
    for pc, bl in ((1, None), (3, P.blocks())):
        x, st = O.csr_solve(A, A.rhs, precond=pc, blocks=bl, tol=1e-12, maxit=5000)
        assert st["rc"] == 0
        assert np.linalg.norm(x - xd) / np.linalg.norm(xd) < 1e-8
    x, st = O.csr_solve(A, A.rhs, precond=2, ilut_p=20, ilut_tau=1e-4, tol=1e-12, maxit=5000)
    assert st["rc"] == 0 and np.linalg.norm(x - xd) / np.linalg.norm(xd) < 1e-8


@pytest.mark.parametrize("L", [1, 3, 5, 7])
def test_library_coupling_quadrature_matches_reference_tables(L):
    """The library's own quadrature of the coupling integrals (harmonics_coupling.hpp:39-278)
    against the reference's tabulated literals (harmonics_coupling.hpp:282-1048): same
    pattern, values within the literals' precision (they carry ~12 digits)."""
    from vshe import gpu
    c = gpu.coupling_tables(L)
    g = O.golden_coupling(L)
    assert np.array_equal(c.data != 0, g.data != 0)
    assert np.max(np.abs(c.data - g.data)) < 1e-7

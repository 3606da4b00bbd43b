"""The oracle's restatement of the outer loop's Poisson system (oracle/poisson_oracle.cpp:
viennashe/assemble.hpp:165-345) against known answers and against a second, vectorised numpy
restatement written here from the same reference lines; and the damped update
(viennashe/simulator.hpp:606-647).  CPU only."""
import math

import numpy as np
import pytest

from vshe import devices as D
import oracle_api as O

Q, KB = 1.602176565e-19, 1.3806488e-23
EPS0 = 1.0e7 / (4.0 * 3.1415926535897932384626433832795 * 299792458.0 * 299792458.0)
EPS = {0: 11.9 * EPS0, 1: 3.9 * EPS0, 2: 25.0 * EPS0, 3: 10.0 * EPS0, 4: 1.0 * EPS0}


def numpy_poisson(dev, fcen, psi, n, p):
    """assemble.hpp:165-300 in numpy, dense: rows and columns are the non-contact cells."""
    unk = np.full(dev.n_cells, -1)
    ids = np.where(dev.contact_id < 0)[0]
    unk[ids] = np.arange(len(ids))
    A = np.zeros((len(ids), len(ids)))
    b = np.zeros(len(ids))
    cen = dev.cell_centroid.reshape(dev.n_cells, dev.dim)
    nrm = dev.facet_normal.reshape(dev.n_facets, dev.dim)
    vt = KB * dev.temperature / Q
    for c in ids:
        r = unk[c]
        for k in range(dev.cell_facet_ptr[c], dev.cell_facet_ptr[c + 1]):
            f = dev.cell_facet_idx[k]
            c1, c2 = dev.facet_cells[f]
            o = c2 if c1 == c else c1
            if o < 0:
                continue
            conn = cen[o] - cen[c]
            ln = np.linalg.norm(conn)
            w = dev.facet_volume[f] * float(np.dot((1.0 if c1 == c else -1.0) * nrm[f], conn / ln))
            if unk[o] >= 0:
                dc, do = np.linalg.norm(fcen[f] - cen[c]), np.linalg.norm(fcen[f] - cen[o])
                em = (dc + do) / (dc / EPS[int(dev.cell_material[c])] + do / EPS[int(dev.cell_material[o])])
                A[r, unk[o]] = em * w / ln
                A[r, r] -= em * w / ln
                b[r] -= em * w * (psi[o] - psi[c]) / ln
            else:
                A[r, r] -= EPS[int(dev.cell_material[c])] * w / ln
                b[r] -= EPS[int(dev.cell_material[c])] * w / ln * (dev.potential[o] - psi[c])
        if dev.cell_material[c] == D.SI:
            A[r, r] -= dev.cell_volume[c] * Q * (n[c] + p[c]) / vt
            b[r] += dev.cell_volume[c] * Q * (n[c] - dev.doping_n[c] - p[c] + dev.doping_p[c])
    return A, b


def dense(M):
    A = np.zeros((M.n, M.n))
    for i in range(M.n):
        A[i, M.ci[M.rp[i]:M.rp[i + 1]]] = M.v[M.rp[i]:M.rp[i + 1]]
    return A


def small_bar():
    return D.nin_bar_2d(nx=12, ny=5, name="poisson_bar")


def test_neutral_constant_potential_has_zero_rhs():
    # uniform doping, n = N_D, p = 0, the same potential everywhere (contacts included): the
    # Laplacian of a constant and the charge both vanish
    dev = D.nin_diode_1d(dopings=(1e23, 1e23, 1e23), boxes=40, bias=0.0)
    dev.potential[:] = 0.3
    fc = D.facet_centres(dev)
    M = O.poisson_assemble(dev, fc, dev.potential, dev.doping_n.copy(), np.zeros(dev.n_cells))
    assert M.n == int(np.sum(dev.contact_id < 0))
    assert np.all(M.rhs == 0.0)


def test_1d_row_is_the_finite_volume_stencil():
    dev = D.nin_diode_1d(boxes=30, bias=0.2)
    fc = D.facet_centres(dev)
    rng = np.random.default_rng(3)
    n = dev.doping_n * rng.uniform(0.5, 1.5, dev.n_cells)
    p = rng.uniform(0.0, 1e10, dev.n_cells)
    M = O.poisson_assemble(dev, fc, dev.potential, n, p)
    A = dense(M)
    h = float(dev.cell_volume[5])
    vt = KB * dev.temperature / Q
    c = 5 + 1  # unknown row 5 is cell 6 (cell 0 is the left contact)
    r = 5
    assert math.isclose(A[r, r - 1], EPS[0] / h, rel_tol=1e-14)
    assert math.isclose(A[r, r + 1], EPS[0] / h, rel_tol=1e-14)
    assert math.isclose(A[r, r], -2 * EPS[0] / h - h * Q * (n[c] + p[c]) / vt, rel_tol=1e-13)
    lap = EPS[0] * (dev.potential[c + 1] - 2 * dev.potential[c] + dev.potential[c - 1]) / h
    assert math.isclose(M.rhs[r], -lap + h * Q * (n[c] - dev.doping_n[c] - p[c] + dev.doping_p[c]),
                        rel_tol=1e-9, abs_tol=1e-9 * abs(lap))


def test_harmonic_mean_permittivity_at_an_interface():
    dev = D.nin_diode_1d(boxes=20, bias=0.0)
    dev.cell_material[10:] = 1  # SiO2 from cell 10 on
    fc = D.facet_centres(dev)
    M = O.poisson_assemble(dev, fc, dev.potential, dev.doping_n, np.zeros(dev.n_cells))
    A = dense(M)
    h = float(dev.cell_volume[9])
    em = 2.0 / (1.0 / EPS[0] + 1.0 / EPS[1])
    assert math.isclose(A[8, 9], em / h, rel_tol=1e-13)  # unknown rows 8, 9 = cells 9, 10
    # oxide cells carry no charge and no Gummel term
    M2 = O.poisson_assemble(dev, fc, dev.potential, dev.doping_n * 2, np.zeros(dev.n_cells))
    assert np.array_equal(M.rhs[10:], M2.rhs[10:])


@pytest.mark.parametrize("make", [small_bar, lambda: D.nin_diode_1d(boxes=60, bias=0.4),
                                  lambda: D.mosfet_2d(nx=12, ny=6)])
def test_oracle_matches_numpy_restatement(make):
    dev = make()
    fc = D.facet_centres(dev)
    rng = np.random.default_rng(11)
    psi = dev.potential + rng.normal(0, 0.01, dev.n_cells)
    n = dev.doping_n * rng.uniform(0.1, 2.0, dev.n_cells)
    p = rng.uniform(0.0, 1e12, dev.n_cells)
    M = O.poisson_assemble(dev, fc, psi, n, p)
    A, b = numpy_poisson(dev, fc, psi, n, p)
    Ad = dense(M)
    assert np.array_equal(Ad != 0.0, A != 0.0)
    assert np.max(np.abs(Ad - A)) <= 1e-13 * np.max(np.abs(A))
    assert np.max(np.abs(M.rhs - b)) <= 1e-12 * np.max(np.abs(b))


def test_damped_update_keeps_contacts_and_solves_the_step():
    dev = small_bar()
    fc = D.facet_centres(dev)
    n = dev.doping_n * 0.9
    p = np.zeros(dev.n_cells)
    psi_out, dpsi, M = O.poisson_update(dev, fc, dev.potential, n, p, damping=0.4)
    contact = dev.contact_id >= 0
    assert np.array_equal(psi_out[contact], dev.potential[contact])
    assert np.allclose(psi_out[~contact], dev.potential[~contact] + 0.4 * dpsi, rtol=0, atol=1e-15)
    A = dense(M)
    assert np.linalg.norm(A @ dpsi - M.rhs) <= 1e-10 * np.linalg.norm(M.rhs)

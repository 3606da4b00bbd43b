"""Small seeded SHE problems shared by the tests (sizes the CPU oracle builds in well under a second)."""
import numpy as np

from vshe import devices as D
import oracle_api as O


def resistor_2d(T=300.0, nx=9, ny=1):
    """The reference's equilibrium resistor (tests/src/equilibrium_resistor.cpp:176-190): 600 x 600 nm,
    doping n = p = 1e16 m^-3, zero bias, contact potential on cells with x < 0.1 L and x > 0.9 L."""
    lx = ly = 6.0e-7
    vol, cen, fc, fvol, fn, cfp, cfi = D._mesh_2d(nx, ny, lx / nx, ly / ny)
    n = nx * ny
    mat = np.zeros(n, np.int32)
    nd = np.full(n, 1e16)
    na = np.full(n, 1e16)
    contact = np.full(n, -1, np.int32)
    contact[cen[:, 0] < 0.1 * lx] = 0
    contact[cen[:, 0] > 0.9 * lx] = 1
    phi = D._built_in_potential(T, nd, na)
    dev = D.Device(2, mat, vol, cen, nd, na, phi, contact, fc, fvol, fn, cfp, cfi, T, np.zeros(2), "resistor")
    cfg = D.SheConfig(max_expansion_order=1, energy_spacing=6.2 * D.Q / 1000.0)
    return dev, cfg


def diode_small(L=1, boxes=40, bias=0.3, n_energy_range=0.5):
    dev = D.nin_diode_1d(lengths=(10e-9, 30e-9, 10e-9), dopings=(1e25, 1e22, 1e25), boxes=boxes, bias=bias, name="diode_small")
    cfg = D.SheConfig(max_expansion_order=L, energy_spacing=D.HBAR_OMEGA_OP / 4.0, min_kinetic_energy_range=n_energy_range * D.Q)
    return dev, cfg


def bar_small(L=3, nx=16, ny=6, n_energies=40, bias=0.1):
    """The 2D bar at a coarse mesh.  A few tens of energies cover the 0.8 V drop of the full
    workload only barely (negative kinetic range, no current), so the small cases use 0.1 V."""
    dev, cfg = D.config2(nx=nx, ny=ny, n_energies=n_energies, L=L, bias=bias)
    return dev, cfg


def oracle_problem(dev, cfg):
    return O.OracleProblem(dev, cfg, O.golden_coupling(cfg.max_expansion_order))


def current_scale(dens_ref, cur_ref):
    """Scale for comparing terminal currents: the larger of the largest current and the
    one-way thermal flux q * n_max * 1e5 m/s of the densest cell.  Near equilibrium the net
    current is a cancellation of one-way fluxes, so its error scales with the flux, not with
    the (vanishing) net current."""
    return max(float(np.max(np.abs(cur_ref))) if len(cur_ref) else 0.0, 1.602176634e-19 * float(np.max(dens_ref)) * 1e5)


def arrow_csr(n=1500, seed=5):
    """Seeded n x n 'arrow' system with one dense first row and one dense last row, diagonally
    dominant: the first row's U part and the last row's L part hold about n entries each, longer
    than any SHE row, which is what ILUT's p-largest selection has to handle at any length."""
    rng = np.random.default_rng(seed)
    rows = []
    for i in range(n):
        cols = {i: 4.0}
        if i > 0:
            cols[i - 1] = -1.0
        if i + 1 < n:
            cols[i + 1] = -1.0
        if i == 0 or i == n - 1:
            others = np.arange(2, n) if i == 0 else np.arange(0, n - 2)
            vals = rng.uniform(0.1, 1.0, len(others)) * rng.choice([-1.0, 1.0], len(others))
            cols.update({int(j): float(v) for j, v in zip(others, vals)})
            cols[i] = 1.1 * float(np.sum(np.abs(vals))) + 2.0
        rows.append(sorted(cols.items()))
    rp = np.zeros(n + 1, np.int64)
    rp[1:] = np.cumsum([len(r) for r in rows])
    ci = np.array([j for r in rows for j, _ in r], np.int32)
    v = np.array([x for r in rows for _, x in r], np.float64)
    rhs = rng.uniform(-1.0, 1.0, n)
    return O.CSR(rp, ci, v, rhs)

"""The row-length bounds behind the HBM admission estimate (SheProblem::estimate_bytes, reported by
vshe_she_plan as bytes_estimate), checked on the oracle's systems on the CPU.  The server admits
a request by that estimate before anything is allocated, so the bounds must hold for every
request:
* a full-system even row holds at most 3 + f o(L) entries (the diagonal, two optical
  in-scattering entries, o(L) odd couplings per facet of its cell, f = the mesh's largest facet
  count per cell), an odd row at most 1 + 2 e(L);
* a reduced row at most 3 + (1 + f) e(L) (its cell and every neighbour);
* the ILU(k) factor at most (1 + k) times the reduced pattern, for the orders the library uses.
The GPU tests check the estimate against the device allocation itself."""
import numpy as np
import pytest

from vshe import devices as D
from vshe import gpu
import oracle_api as O


def _oxide_diode():
    dev, cfg = D.config1()
    dev.cell_material[dev.n_cells // 2:] = 1
    return dev, cfg


CASES = {
    "diode": D.config1,
    "bar_L3": lambda: D.config2(nx=16, ny=5, n_energies=40, L=3),
    "bar_L5": lambda: D.config2(nx=10, ny=4, n_energies=30, L=5),
    "mosfet_L5": lambda: D.config5(nx=16, ny=8, n_energies=40, L=5),
    "oxide_diode": _oxide_diode,
}


def _e_o(L):
    e = sum(2 * l + 1 for l in range(0, L + 1, 2))
    return e, (L + 1) ** 2 - e


@pytest.mark.parametrize("name", sorted(CASES))
def test_row_length_bounds(name):
    dev, cfg = CASES[name]()
    cpl = O.golden_coupling(cfg.max_expansion_order)
    P = O.OracleProblem(dev, cfg, cpl)
    e, o = _e_o(cfg.max_expansion_order)
    f = int(np.max(np.diff(dev.cell_facet_ptr)))
    assert f <= 2 * dev.dim
    full = P.matrix(0)
    lens = np.diff(full.rp)
    assert lens[:P.n_even].max() <= 3 + f * o
    assert lens[P.n_even:].max(initial=0) <= 1 + 2 * e
    red = P.matrix(3)
    assert np.diff(red.rp).max() <= 3 + (1 + f) * e
    info = gpu.she_plan(dev, cfg, coupling=cpl)
    assert info["n_even"] == P.n_even and info["n_odd"] == P.n_odd
    # the footprint bound covers at least the reduced system's and the full system's CSR bytes
    assert info["bytes_estimate"] >= 12 * (full.nnz + red.nnz) + 8 * (full.n + red.n)


@pytest.mark.parametrize("name", ["bar_L3", "bar_L5", "mosfet_L5"])
@pytest.mark.parametrize("fill", [0, 1])
def test_factor_bound(name, fill):
    dev, cfg = CASES[name]()
    cpl = O.golden_coupling(cfg.max_expansion_order)
    P = O.OracleProblem(dev, cfg, cpl)
    red = P.matrix(3)
    perm, _ = gpu.she_node_order(dev, cfg, coupling=cpl, fill_level=fill)
    for kw in (dict(perm=perm), dict(ordering="multicolor")):
        lay = gpu.layout(red.rp, red.ci, None, precond="block_ilu0", fill_level=fill, blocks=P.blocks(), **kw)
        assert lay["nnzL"] + lay["nnzU"] + red.n <= (1 + fill) * red.nnz

"""The host layout (solver order, ILU(k) pattern, levels, SELL tables) built on several host
threads equals the one built on one thread, array for array (vshe_set_host_threads).  CPU only:
the layout needs no device."""
import numpy as np
import pytest

from vshe import devices as D
from vshe import gpu
import oracle_api as O


CASES = {
    "bar_block_ilu1": (lambda: D.config2(nx=40, ny=10, n_energies=40, L=3),
                       dict(precond="block_ilu0", ordering="multicolor", fill_level=1), True),
    "bar_block_ilu2": (lambda: D.config2(nx=24, ny=6, n_energies=24, L=3),
                       dict(precond="block_ilu0", ordering="multicolor", fill_level=2), True),
    "bar_multicolour_ilu1": (lambda: D.config2(nx=24, ny=6, n_energies=24, L=3),
                             dict(precond="ilu0", ordering="multicolor", fill_level=1), False),
    "diode_natural": (lambda: D.config1(), dict(precond="ilu0", ordering="natural"), False),
    "bar_ilut": (lambda: D.config2(nx=24, ny=6, n_energies=24, L=3),
                 dict(precond="ilut", ordering="natural", ilut_entries=20, ilut_drop=1e-3), False),
    "bar_slab_ilut": (lambda: D.config2(nx=24, ny=6, n_energies=24, L=3),
                      dict(precond="ilut", ordering="natural", ilut_entries=20, ilut_drop=1e-3), True),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_layout_does_not_depend_on_host_threads(name):
    make, kw, blocks = CASES[name]
    dev, cfg = make()
    P = O.OracleProblem(dev, cfg, O.golden_coupling(cfg.max_expansion_order))
    A = P.matrix(3)
    if blocks:
        kw = dict(kw, blocks=P.blocks())
    try:
        vals = A.v if kw["precond"] == "ilut" else None  # the ILUT pattern comes from the values
        gpu.set_host_threads(1)
        one = gpu.layout(A.rp, A.ci, vals, **kw)
        gpu.set_host_threads(8)
        many = gpu.layout(A.rp, A.ci, vals, **kw)
    finally:
        gpu.set_host_threads(0)
    assert one.keys() == many.keys()
    for k in one:
        a, b = one[k], many[k]
        if isinstance(a, np.ndarray):
            assert a.dtype == b.dtype and np.array_equal(a, b), k
        else:
            assert a == b, k

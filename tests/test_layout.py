"""Host logic of the solver layout (no GPU): the level-sorted solver order and the SELL-32
tables of A, L and U that the CUDA kernels read (vshe_layout_export).

The kernels' arithmetic is replayed here in numpy exactly as the device runs it: the SELL-32
SpMV, and the forward / backward sweeps level by level, where every row not yet computed holds
NaN, so a row scheduled before one it depends on shows up as NaN.  The results must match the
oracle's CSR SpMV and ILU(0) apply (1e-13 relative, summation order differs).
"""
import numpy as np
import pytest

from vshe import devices as D
from vshe import gpu
import oracle_api as O
import cases


def _problems():
    return [("diode_L1", *cases.diode_small(L=1, boxes=40)),
            ("diode_L3", *cases.diode_small(L=3, boxes=30)),
            ("bar_L3", *cases.bar_small(L=3, nx=12, ny=5, n_energies=30))]


PROBLEMS = _problems()


@pytest.fixture(scope="module", params=PROBLEMS, ids=[p[0] for p in PROBLEMS])
def prob(request):
    name, dev, cfg = request.param
    P = cases.oracle_problem(dev, cfg)
    return name, P, P.matrix(3)


def sell_spmv(Lt, aval, x_p):
    """y = A x over the SELL-32 slices (x_p in solver order, with the zero entry n)."""
    n = Lt["n"]
    xz = np.append(x_p, 0.0)
    y = np.zeros(n)
    aoff = Lt["aoff"]
    for j in range(len(aoff) - 1):
        w = (aoff[j + 1] - aoff[j]) // 32
        slots = aoff[j] + 32 * np.arange(w)[:, None] + np.arange(32)[None, :]
        part = (aval[slots] * xz[Lt["acol"][slots]]).sum(axis=0)
        rows = 32 * j + np.arange(32)
        m = rows < n
        y[rows[m]] = part[m]
    return y


def sell_ilu_apply(Lt, lval, uval, udinv, b_p):
    """U^{-1} L^{-1} b over the SELL-32 factor slices, forward then backward levels; rows
    not computed yet hold NaN."""
    n = Lt["n"]
    y = np.full(n + 1, np.nan)
    y[n] = 0.0
    lrow0, loff = Lt["lrow0"], Lt["loff"]
    for j in range(len(loff) - 1):  # slices are stored level by level
        w = (loff[j + 1] - loff[j]) // 32
        slots = loff[j] + 32 * np.arange(w)[:, None] + np.arange(32)[None, :]
        cols = Lt["lcol"][slots]
        nr = lrow0[j + 1] - lrow0[j]
        v = lval[slots][:, :nr]
        c = cols[:, :nr]
        s = (v * np.where(v != 0.0, y[c], 0.0)).sum(axis=0) if w else np.zeros(nr)
        # padded slots carry value 0 and point at the zero entry n
        assert np.all(c[v == 0.0] == n) or np.all(v[c == n] == 0.0)
        y[lrow0[j]:lrow0[j] + nr] = b_p[lrow0[j]:lrow0[j] + nr] - s
    out = np.full(n + 1, np.nan)
    out[n] = 0.0
    us, uoff, urow = Lt["uslot0"], Lt["uoff"], Lt["urow"]
    for j in range(len(uoff) - 1):
        w = (uoff[j + 1] - uoff[j]) // 32
        slots = uoff[j] + 32 * np.arange(w)[:, None] + np.arange(32)[None, :]
        nr = us[j + 1] - us[j]
        v = uval[slots][:, :nr]
        c = Lt["ucol"][slots][:, :nr]
        s = (v * np.where(v != 0.0, out[c], 0.0)).sum(axis=0) if w else np.zeros(nr)
        t = np.arange(us[j], us[j] + nr)
        rows = urow[t]
        out[rows] = (y[rows] - s) * udinv[t]
    return out[:n]


def _diag_entries(A):
    d = np.zeros(A.n, np.int64)
    for i in range(A.n):
        k = np.searchsorted(A.ci[A.rp[i]:A.rp[i + 1]], i)
        d[i] = A.rp[i] + k
    return d


def _factor_slots(Lt, lu, A):
    lval = np.where(Lt["lmap"] >= 0, lu[np.maximum(Lt["lmap"], 0)], 0.0)
    uval = np.where(Lt["umap"] >= 0, lu[np.maximum(Lt["umap"], 0)], 0.0)
    diag = _diag_entries(A)
    udinv = 1.0 / lu[diag[Lt["perm"][Lt["urow"]]]]
    return lval, uval, udinv


def test_solver_order_is_a_level_sorted_permutation(prob):
    name, P, A = prob
    Lt = gpu.layout(A.rp, A.ci, precond="ilu0")
    perm = Lt["perm"]
    assert np.array_equal(np.sort(perm), np.arange(A.n))
    assert Lt["lvr"][0] == 0 and Lt["lvr"][-1] == A.n and np.all(np.diff(Lt["lvr"]) > 0)
    # every stored slot maps to a distinct entry of A; together they cover A exactly once
    amap = Lt["amap"][Lt["amap"] >= 0]
    assert np.array_equal(np.sort(amap), np.arange(A.nnz))
    # widths: SELL slices hold whole 32-lane columns
    assert np.all(np.diff(Lt["aoff"]) % 32 == 0)


@pytest.mark.parametrize("ordering", ["natural", "multicolor"])
def test_sell_spmv_matches_csr(prob, ordering):
    name, P, A = prob
    Lt = gpu.layout(A.rp, A.ci, precond="ilu0", ordering=ordering)
    perm = Lt["perm"]
    aval = np.where(Lt["amap"] >= 0, A.v[np.maximum(Lt["amap"], 0)], 0.0)
    x = np.random.default_rng(3).standard_normal(A.n)
    y_p = sell_spmv(Lt, aval, x[perm])
    y = np.empty(A.n)
    y[perm] = y_p
    y_ref = O.spmv(A, x)
    assert np.max(np.abs(y - y_ref)) <= 1e-13 * np.max(np.abs(y_ref))


@pytest.mark.parametrize("block", [False, True])
def test_sell_ilu0_apply_matches_oracle(prob, block):
    """Natural base order: the level-sorted factors are the reference order's ILU(0), relabelled."""
    name, P, A = prob
    bl = P.blocks() if block else None
    Lt = gpu.layout(A.rp, A.ci, precond="block_ilu0" if block else "ilu0", blocks=bl)
    lu = O.ilu0_values(A, blocks=bl)
    lval, uval, udinv = _factor_slots(Lt, lu, A)
    b = np.random.default_rng(5).standard_normal(A.n)
    perm = Lt["perm"]
    z_p = sell_ilu_apply(Lt, lval, uval, udinv, b[perm])
    assert np.all(np.isfinite(z_p)), "a row was scheduled before a row it depends on"
    z = np.empty(A.n)
    z[perm] = z_p
    z_ref = O.ilu0_apply(A, lu, b, blocks=bl)
    assert np.max(np.abs(z - z_ref)) <= 1e-11 * np.max(np.abs(z_ref))


def test_sell_ilu0_apply_multicolour(prob):
    """Multicolour base order: the sweeps over the SELL tables reproduce the oracle's ILU(0) of
    the solver-order matrix."""
    name, P, A = prob
    Lt = gpu.layout(A.rp, A.ci, precond="ilu0", ordering="multicolor")
    perm = Lt["perm"]
    inv = np.empty(A.n, np.int64)
    inv[perm] = np.arange(A.n)
    # solver-order CSR and the map of its entries back to A's
    rows, cols, src = [], [], []
    for q in range(A.n):
        o = perm[q]
        ks = np.arange(A.rp[o], A.rp[o + 1])
        c = inv[A.ci[ks]]
        order = np.argsort(c)
        rows.append(np.full(len(ks), q)); cols.append(c[order]); src.append(ks[order])
    cols = np.concatenate(cols); src = np.concatenate(src)
    rp = np.zeros(A.n + 1, np.int64)
    rp[1:] = np.cumsum([len(r) for r in rows])
    Ap = O.CSR(rp, cols.astype(np.int32), A.v[src])
    lup = O.ilu0_values(Ap)
    lu = np.empty(A.nnz)
    lu[src] = lup
    lval, uval, udinv = _factor_slots(Lt, lu, A)
    b = np.random.default_rng(7).standard_normal(A.n)
    z_p = sell_ilu_apply(Lt, lval, uval, udinv, b[perm])
    assert np.all(np.isfinite(z_p)), "a row was scheduled before a row it depends on"
    z_ref = O.ilu0_apply(Ap, lup, b[perm])
    assert np.max(np.abs(z_p - z_ref)) <= 1e-11 * np.max(np.abs(z_ref))


def _csr_lookup(rp, ci, vals):
    """(row, col) -> value of a CSR, as a dict (small cases only)."""
    d = {}
    for i in range(len(rp) - 1):
        for k in range(rp[i], rp[i + 1]):
            d[(i, int(ci[k]))] = vals[k]
    return d


@pytest.mark.parametrize("ordering", ["natural", "multicolor"])
def test_sell_iluk_apply_matches_oracle(prob, ordering):
    """ILU(1): the symbolic fill, the levels over the filled pattern and the SELL factor tables
    reproduce the oracle's ILU(1) (Saad Alg. 10.5) apply of the solver-order matrix."""
    name, P, A = prob
    Lt = gpu.layout(A.rp, A.ci, precond="ilu0", ordering=ordering, fill_level=1)
    perm = Lt["perm"]
    n = A.n
    inv = np.empty(n, np.int64)
    inv[perm] = np.arange(n)
    # solver-order matrix (the relabelling is exact for ILU(k): no coupled pair changes order)
    rows, cols, src = [], [], []
    for q in range(n):
        o = perm[q]
        ks = np.arange(A.rp[o], A.rp[o + 1])
        c = inv[A.ci[ks]]
        od = np.argsort(c)
        cols.append(c[od]); src.append(ks[od]); rows.append(len(ks))
    rpp = np.zeros(n + 1, np.int64)
    rpp[1:] = np.cumsum(rows)
    Ap = O.CSR(rpp, np.concatenate(cols).astype(np.int32), A.v[np.concatenate(src)])
    frp, fci, flu = O.iluk_csr(Ap, 1)
    assert frp[-1] == Lt["nnzL"] + Lt["nnzU"] + n, "fill pattern differs from the oracle's"
    look = _csr_lookup(frp, fci, flu)
    # factor slot values from (row, column) of every slot
    lval = np.zeros(len(Lt["lcol"]))
    for j in range(len(Lt["loff"]) - 1):
        w = (Lt["loff"][j + 1] - Lt["loff"][j]) // 32
        for lane in range(Lt["lrow0"][j + 1] - Lt["lrow0"][j]):
            row = Lt["lrow0"][j] + lane
            for k in range(w):
                slot = Lt["loff"][j] + 32 * k + lane
                c = Lt["lcol"][slot]
                if c < n:
                    lval[slot] = look[(row, int(c))]
    uval = np.zeros(len(Lt["ucol"]))
    udinv = np.zeros(n)
    for j in range(len(Lt["uoff"]) - 1):
        w = (Lt["uoff"][j + 1] - Lt["uoff"][j]) // 32
        for lane in range(Lt["uslot0"][j + 1] - Lt["uslot0"][j]):
            t = Lt["uslot0"][j] + lane
            row = Lt["urow"][t]
            udinv[t] = 1.0 / look[(row, row)]
            for k in range(w):
                slot = Lt["uoff"][j] + 32 * k + lane
                c = Lt["ucol"][slot]
                if c < n:
                    uval[slot] = look[(row, int(c))]
    b = np.random.default_rng(9).standard_normal(n)
    z_p = sell_ilu_apply(Lt, lval, uval, udinv, b[perm])
    assert np.all(np.isfinite(z_p)), "a row was scheduled before a row it depends on"
    z_ref = O.ilu0_apply(O.CSR(frp, fci, flu), flu, b[perm])
    assert np.max(np.abs(z_p - z_ref)) <= 1e-11 * np.max(np.abs(z_ref))


def _slot_pattern(Lt):
    """(solver row, solver column) of every non-padding L and U slot, and the diagonal."""
    n = Lt["n"]
    pat = set((i, i) for i in range(n))
    for off, first, colk, rowof in (("loff", "lrow0", "lcol", None), ("uoff", "uslot0", "ucol", "urow")):
        o, f, c = Lt[off], Lt[first], Lt[colk]
        for j in range(len(o) - 1):
            w = (o[j + 1] - o[j]) // 32
            for lane in range(f[j + 1] - f[j]):
                t = f[j] + lane
                row = Lt[rowof][t] if rowof else t
                for k in range(w):
                    col = c[o[j] + 32 * k + lane]
                    if col < n:
                        pat.add((int(row), int(col)))
    return pat


@pytest.mark.parametrize("p,tau", [(20, 1e-3), (5, 1e-2)])
def test_ilut_pattern_matches_oracle(prob, p, tau):
    """VSHE_PRECOND_ILUT: the host analysis keeps, per row, every position whose entry passes
    ILUT(p, tau)'s tau test (Saad Alg. 10.6, before its p-largest rule), the diagonal and A's
    entries; natural order, so solver rows map to the caller's through perm.  The final ILUT
    pattern lies inside it."""
    name, P, A = prob
    Lt = gpu.layout(A.rp, A.ci, values=A.v, precond="ilut", ilut_entries=p, ilut_drop=tau)
    perm = Lt["perm"]
    got = set((int(perm[i]), int(perm[j])) for i, j in _slot_pattern(Lt))
    rp, ci = O.ilut_passed(A, p, tau)
    want = set()
    for i in range(A.n):
        want.update((i, int(j)) for j in ci[rp[i]:rp[i + 1]])
        want.update((i, int(j)) for j in A.ci[A.rp[i]:A.rp[i + 1]])
        want.add((i, i))
    assert got == want
    frp, fci, _ = O.ilut_csr(A, p, tau)
    final = set((i, int(j)) for i in range(A.n) for j in fci[frp[i]:frp[i + 1]])
    assert final <= got


def test_ilut_pattern_long_rows():
    """Rows whose ILUT parts hold about 1500 entries: the host analysis takes them and its pass
    sets still match the oracle's ILUT(20, 1e-6) entry for entry."""
    A = cases.arrow_csr()
    p, tau = 20, 1e-6
    Lt = gpu.layout(A.rp, A.ci, values=A.v, precond="ilut", ilut_entries=p, ilut_drop=tau)
    perm = Lt["perm"]
    got = set((int(perm[i]), int(perm[j])) for i, j in _slot_pattern(Lt))
    rp, ci = O.ilut_passed(A, p, tau)
    assert np.diff(rp)[0] > 1024 and np.diff(rp)[-1] > 1024
    want = set()
    for i in range(A.n):
        want.update((i, int(j)) for j in ci[rp[i]:rp[i + 1]])
        want.update((i, int(j)) for j in A.ci[A.rp[i]:A.rp[i + 1]])
        want.add((i, i))
    assert got == want


@pytest.mark.parametrize("p,tau", [(20, 1e-3), (60, 1e-4)])
def test_slab_ilut_pattern_matches_oracle(p, tau):
    """VSHE_PRECOND_ILUT with energy-slab blocks: the elimination stays inside each slab (no
    elimination with, and no fill from, rows of other slabs; tau ||a_i|| over the whole row).  The
    host analysis keeps, inside the slabs, exactly the positions that pass the oracle's
    slab-restricted ILUT tau test, the diagonal and A's entries; the oracle's final factor lies
    inside them; and the sweeps run one task per slab group."""
    dev, cfg = D.config2(nx=16, ny=5, n_energies=40, L=5)
    P = O.OracleProblem(dev, cfg, O.golden_coupling(5))
    A = P.matrix(3)
    bl = P.blocks()
    blk = np.searchsorted(bl, np.arange(A.n), side="right") - 1
    Lt = gpu.layout(A.rp, A.ci, values=A.v, precond="ilut", ilut_entries=p, ilut_drop=tau, blocks=bl)
    perm = Lt["perm"]
    got = set((int(perm[i]), int(perm[j])) for i, j in _slot_pattern(Lt))
    rp, ci = O.ilut_passed(A, p, tau, blocks=bl)
    want = set()
    for i in range(A.n):
        want.update((i, int(j)) for j in ci[rp[i]:rp[i + 1]] if blk[j] == blk[i])
        want.update((i, int(j)) for j in A.ci[A.rp[i]:A.rp[i + 1]] if blk[j] == blk[i])
        want.add((i, i))
    assert got == want
    frp, fci, _ = O.ilut_csr(A, p, tau, blocks=bl)
    final = set((i, int(j)) for i in range(A.n) for j in fci[frp[i]:frp[i + 1]])
    assert all(blk[j] == blk[i] for i, j in final) and final <= got
    # without blocks the same options give the whole-matrix ILUT, which reaches across slabs
    whole = O.ilut_passed(A, p, tau)
    assert any(blk[int(j)] != blk[i] for i in range(A.n) for j in whole[1][whole[0][i]:whole[0][i + 1]] if j > i)
    assert gpu.sweep_plan(A.rp, A.ci, A.v, precond="ilut", ilut_entries=p, ilut_drop=tau, blocks=bl)["kind"] == 2

"""Request files and result writers (vshe/io.py), CPU only: a request survives the round trip
bit for bit (and the oracle builds the same system from it), the gnuplot file has the
reference writer's layout (viennashe/io/gnuplot_writer.hpp:71-86), the VTK point cloud reads
back."""
import numpy as np
import pytest

from vshe import devices as D
from vshe import io as vio
import oracle_api as O


def test_request_round_trip(tmp_path):
    dev, cfg = D.config4(6, rate=200.0)[3][1:]
    path = tmp_path / "req.npz"
    vio.save_request(path, dev, cfg)
    dev2, cfg2 = vio.load_request(path)
    for k in vio._DEVICE_ARRAYS:
        a, b = np.asarray(getattr(dev, k)), np.asarray(getattr(dev2, k))
        assert a.dtype == b.dtype and np.array_equal(a, b), k
    assert dev2.dim == dev.dim and dev2.temperature == dev.temperature and dev2.name == dev.name
    assert cfg2 == cfg


def test_request_replays_to_the_same_system(tmp_path):
    dev, cfg = D.config1()
    path = tmp_path / "c1.npz"
    vio.save_request(path, dev, cfg)
    dev2, cfg2 = vio.load_request(path)
    cpl = O.golden_coupling(cfg.max_expansion_order)
    A = O.OracleProblem(dev, cfg, cpl).matrix(3)
    B = O.OracleProblem(dev2, cfg2, cpl).matrix(3)
    assert np.array_equal(A.rp, B.rp) and np.array_equal(A.ci, B.ci)
    assert np.array_equal(A.v, B.v) and np.array_equal(A.rhs, B.rhs)


def test_gnuplot_layout(tmp_path):
    dev = D.nin_bar_2d(nx=4, ny=2, name="tiny")
    vals = np.linspace(1e21, 2e21, dev.n_cells)
    path = tmp_path / "n.dat"
    vio.write_gnuplot(path, dev, vals)
    lines = open(path).read().split("\n")
    assert lines[0] == "## ViennaSHE - gnuplot output "
    cen = dev.cell_centroid.reshape(dev.n_cells, 2)
    for c in range(dev.n_cells):
        assert lines[1 + c] == "%g %g %g " % (cen[c, 0], cen[c, 1], vals[c])
    assert lines[1 + dev.n_cells] == ""


def test_vtk_point_cloud_reads_back(tmp_path):
    dev = D.nin_diode_1d(boxes=12)
    path = tmp_path / "r.vtk"
    vio.write_vtk(path, dev, {"potential": dev.potential, "electron density": dev.doping_n})
    pts, fields = vio.read_vtk_fields(path)
    assert np.array_equal(pts[:, 0], dev.cell_centroid.reshape(-1)) and np.all(pts[:, 1:] == 0)
    assert np.array_equal(fields["potential"], dev.potential)
    assert np.array_equal(fields["electron_density"], dev.doping_n)


def test_she_plan_sizes_match_oracle():
    """vshe_she_plan (the host set-up alone, no GPU): the sizes the oracle's set-up gives."""
    from vshe import gpu
    for dev, cfg in (D.config1(), D.config2(nx=20, ny=5, n_energies=30, L=3)):
        info = gpu.she_plan(dev, cfg, coupling=O.golden_coupling(cfg.max_expansion_order))
        P = O.OracleProblem(dev, cfg, O.golden_coupling(cfg.max_expansion_order))
        assert info["n_even"] == P.n_even and info["n_odd"] == P.n_odd and info["n_energies"] == P.NH
        assert info["bytes_estimate"] > 0


def _space_case():
    return D.config2(nx=12, ny=4, n_energies=20, L=3)


def test_she_space_matches_oracle_mapping():
    """vshe_she_space (host set-up, no GPU): the oracle's energies and (x, H) mapping, entry for
    entry, and the density of states of the oracle's restatement of the Modena dispersion."""
    import ctypes as C
    from vshe import gpu
    oxide = D.config1()
    oxide[0].cell_material[oxide[0].n_cells // 2:] = 1  # SiO2 from the middle on: nodes without unknowns
    for dev, cfg in (D.config1(), _space_case(), D.config5(nx=16, ny=8, n_energies=40, L=5), oxide):
        cpl = O.golden_coupling(cfg.max_expansion_order)
        sp = gpu.she_space(dev, cfg, coupling=cpl)
        P = O.OracleProblem(dev, cfg, cpl)
        H, sc, sf, _ = P.energies()
        ic, jf, oc, of, _ = P.mapping()
        nc, nf, nh = dev.n_cells, dev.n_facets, P.NH
        assert np.array_equal(sp["energies"], H)
        assert np.array_equal(sp["even_index"], ic.reshape(nc, nh))
        assert np.array_equal(sp["odd_index"], jf.reshape(nf, nh))
        assert np.array_equal(sp["even_order"], oc.reshape(nc, nh))
        assert np.array_equal(sp["odd_order"], of.reshape(nf, nh))
        assert np.array_equal(sp["kinetic_energy"], H[None, :] - sc[:, None])
        probe = O.lib().vsheo_physics_probe
        probe.argtypes = [C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_double)]
        eps = sp["kinetic_energy"].reshape(-1)
        ref = np.zeros_like(eps)
        out = np.zeros(8)
        for k in range(0, eps.size, max(1, eps.size // 200)):
            a = np.array([eps[k]])
            probe(0, a.ctypes.data_as(C.POINTER(C.c_double)), out.ctypes.data_as(C.POINTER(C.c_double)))
            ref[k] = out[0]
            assert sp["density_of_states"].reshape(-1)[k] == ref[k]
        # every even unknown belongs to exactly one node
        used = sp["even_index"][sp["even_index"] >= 0]
        assert np.unique(used).size == used.size and used.max() < P.n_even


def test_gnuplot_edf_layouts(tmp_path):
    """The two layouts of the reference's EDF writer (gnuplot_writer_edf.hpp:54-110, 117-175) from
    a full solution of the oracle (the tiny bar's reduced system solved on the CPU)."""
    from vshe import gpu
    dev, cfg = _space_case()
    cpl = O.golden_coupling(cfg.max_expansion_order)
    sp = gpu.she_space(dev, cfg, coupling=cpl)
    P = O.OracleProblem(dev, cfg, cpl)
    A = P.matrix(3)
    x_red, st = O.csr_solve(A, A.rhs, tol=1e-12)
    assert st["rc"] == 0 and st["relres"] <= 1e-12
    xf = P.finish(x_red)[0]
    y00 = 1.0 / np.sqrt(4.0 * np.pi)
    edf = vio.edf_values(sp, xf)
    m = sp["even_index"] >= 0
    assert np.allclose(edf[m], xf[sp["even_index"][m]] * y00, rtol=1e-15, atol=0)
    cen = dev.cell_centroid.reshape(dev.n_cells, 2)
    # filtered writer: the cells of the bottom row
    cells = [c for c in range(dev.n_cells) if cen[c, 1] == cen[0, 1]]
    path = tmp_path / "edf.dat"
    vio.write_gnuplot_edf(path, dev, sp, xf, cells=lambda c: cen[c, 1] == cen[0, 1])
    want = []
    for c in cells:
        for h in range(1, P.NH - 1):
            if sp["even_index"][c, h] > -1 and sp["kinetic_energy"][c, h] > 0:
                want.append("%g %g %g %g %g" % (cen[c, 0], cen[c, 1], sp["kinetic_energy"][c, h] / 1.602176565e-19,
                                                edf[c, h], sp["density_of_states"][c, h]))
        want += ["", ""]
    got = open(path).read().split("\n")
    k = 0
    for w in want:
        if w:
            assert got[k] == w, (k, got[k], w)
        else:
            assert got[k] == ""
        k += 1
    # line writer at the first column's x: sorted by (y, kinetic energy), a blank line per y
    path2 = tmp_path / "edf_line.dat"
    x0 = cen[int(np.argmax((sp["even_index"] >= 0).sum(axis=1))), 0]
    vio.write_gnuplot_edf_line(path2, dev, sp, xf, x0)
    lines = open(path2).read().split("\n")[:-1]
    col = [c for c in range(dev.n_cells) if cen[c, 0] == x0]
    expect = []
    for c in sorted(col, key=lambda c: cen[c, 1]):
        rows = sorted((sp["kinetic_energy"][c, h], edf[c, h]) for h in range(1, P.NH - 1) if sp["even_index"][c, h] > -1)
        expect += [""] * bool(rows) + ["%g %g %g" % (cen[c, 1], e, v) for e, v in rows]
    assert len(expect) > 4 * len(col) and lines == expect
    # the EDF is positive where the carrier population lives (well above the band edge)
    assert np.all(edf[m & (sp["kinetic_energy"] > 0)] > 0)


def _node_of_rows(sp, n_even):
    """Node id (cell * N_H + H) of every reduced row, from the (x, H) space."""
    idx, order = sp["even_index"].reshape(-1), sp["even_order"].reshape(-1)
    node = np.full(n_even, -1, np.int64)
    for a in np.nonzero(idx >= 0)[0]:
        ne = sum(2 * l + 1 for l in range(0, int(order[a]) + 1, 2))
        node[idx[a]:idx[a] + ne] = a
    assert np.all(node >= 0)
    return node


def test_she_node_order_colours_against_the_oracle_pattern():
    """vshe_she_node_order (host only): the SHE pipeline's multicolour order is a stable sort of
    the rows by colour, and rows of different (cell, H) nodes that the oracle's reduced system
    couples have different colours -- directly for ILU(0), at distance two (the pattern of A^2)
    for ILU(k > 0)."""
    import scipy.sparse as sps
    from vshe import gpu
    for dev, cfg in (D.config2(nx=16, ny=5, n_energies=40, L=3), D.config1()):
        cpl = O.golden_coupling(cfg.max_expansion_order)
        P = O.OracleProblem(dev, cfg, cpl)
        A = P.matrix(3)
        node = _node_of_rows(gpu.she_space(dev, cfg, coupling=cpl), P.n_even)
        M = sps.csr_matrix((np.ones(A.nnz), A.ci, A.rp), shape=(A.n, A.n))
        for fill, pat in ((0, M), (1, M @ M)):
            perm, colour = gpu.she_node_order(dev, cfg, coupling=cpl, fill_level=fill)
            assert np.array_equal(np.sort(perm), np.arange(P.n_even))
            assert np.array_equal(perm, np.argsort(colour, kind="stable"))
            coo = pat.tocoo()
            other = node[coo.row] != node[coo.col]
            assert np.all(colour[coo.row[other]] != colour[coo.col[other]]), (dev.name, fill)
            assert colour.max() + 1 <= (64 * (3 if fill else 2))


def test_system_file_round_trip(tmp_path):
    """A drop-in request (CSR system, slab bounds, options) survives the file bit for bit, and the
    oracle solves the loaded system to the same x."""
    from vshe import gpu
    dev, cfg = D.config2(nx=12, ny=4, n_energies=24, L=3)
    P = O.OracleProblem(dev, cfg, O.golden_coupling(3))
    A = P.matrix(3)
    path = tmp_path / "sys.npz"
    vio.save_system(path, A.rp, A.ci, A.v, A.rhs, blocks=P.blocks(), precond="block_ilu0", fill_level=1,
                    precision="mixed", tol=1e-10)
    r = vio.load_system(path)
    for a, b in ((r["rp"], A.rp), (r["ci"], A.ci), (r["values"], A.v), (r["rhs"], A.rhs), (r["blocks"], P.blocks())):
        assert a.dtype == np.asarray(b).dtype or a.dtype.kind == np.asarray(b).dtype.kind
        assert np.array_equal(a, b)
    assert r["opts"] == dict(precond="block_ilu0", fill_level=1, precision="mixed", tol=1e-10)
    o, _ = gpu.make_opts(blocks=r["blocks"], **r["opts"])  # the stored keywords are make_opts keywords
    assert o.fill_level == 1 and o.precond == gpu.PRECOND["block_ilu0"] and o.n_blocks == len(P.blocks()) - 1
    x1, s1 = O.csr_solve(A, A.rhs, tol=1e-12)
    B = O.CSR(r["rp"], r["ci"], r["values"], r["rhs"])
    x2, s2 = O.csr_solve(B, r["rhs"], tol=1e-12)
    assert s1["iters"] == s2["iters"] and np.array_equal(x1, x2)
    with pytest.raises(ValueError):
        vio.save_system(tmp_path / "bad.npz", A.rp, A.ci, A.v, A.rhs[:-1])

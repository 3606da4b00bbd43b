"""Request files and result writers (vshe/io.py), CPU only: a request survives the round trip
bit for bit (and the oracle builds the same system from it), the gnuplot file has the
reference writer's layout (viennashe/io/gnuplot_writer.hpp:71-86), the VTK point cloud reads
back."""
import numpy as np

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

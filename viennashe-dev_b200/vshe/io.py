"""Files of the SHE path: requests on disk and results for plotting.

* ``save_request`` / ``load_request``: a served request (the device description of
  ``vshe_device_desc`` and the SHE configuration of ``vshe_she_config``) as one ``.npz`` file:
  flat arrays under the C field names, so a request can be replayed or exchanged without the
  generator that made it.
* ``save_system`` / ``load_system``: a drop-in request -- the linear system the reference hands
  to its solver slot (CSR row offsets, columns, values, rhs), the energy-slab bounds that
  ``she::solve`` puts into the solver configuration, and the solver options as keyword
  arguments of ``vshe.gpu.make_opts`` -- as one ``.npz`` file.
* ``write_gnuplot``: a per-cell quantity in the layout of the reference's gnuplot writer
  (viennashe/io/gnuplot_writer.hpp:47-118): a ``## ViennaSHE - gnuplot output`` line, then one
  line per cell with the centroid coordinates and the value, each followed by a space, numbers
  as C++ streams print doubles by default (``%g``).
* ``write_gnuplot_edf`` / ``write_gnuplot_edf_line``: the energy distribution function of a
  solved problem, in the layouts of the reference's EDF writer
  (viennashe/io/gnuplot_writer_edf.hpp:54-110 and :117-175), from ``x_full`` and the (x, H)
  space of ``vshe.gpu.she_space``.
* ``write_vtk``: per-cell quantities as a legacy-format VTK point cloud at the cell centroids.
  The reference's VTK writers (viennashe/io/she_vtk_writer.hpp) write the mesh cells; a
  ``vshe_device_desc`` carries no vertices, so the cells are written as points.
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

from .devices import Device, SheConfig

_DEVICE_ARRAYS = ("cell_material", "cell_volume", "cell_centroid", "doping_n", "doping_p", "potential", "contact_id",
                  "facet_cells", "facet_volume", "facet_normal", "cell_facet_ptr", "cell_facet_idx")


def save_request(path, dev: Device, cfg: SheConfig):
    arrays = {"device." + k: np.asarray(getattr(dev, k)) for k in _DEVICE_ARRAYS}
    arrays["device.dim"] = np.int32(dev.dim)
    arrays["device.temperature"] = np.float64(dev.temperature)
    if dev.contact_potential is not None:
        arrays["device.contact_potential"] = np.asarray(dev.contact_potential, np.float64)
    arrays["device.name"] = np.array(dev.name)
    for f in dataclasses.fields(cfg):
        arrays["config." + f.name] = np.asarray(getattr(cfg, f.name))
    np.savez(path, **arrays)


def load_request(path):
    """-> (Device, SheConfig)."""
    z = np.load(path, allow_pickle=False)
    kw = {k: z["device." + k] for k in _DEVICE_ARRAYS}
    dev = Device(dim=int(z["device.dim"]), temperature=float(z["device.temperature"]),
                 contact_potential=z["device.contact_potential"] if "device.contact_potential" in z else None,
                 name=str(z["device.name"]), **kw)
    ck = {}
    for f in dataclasses.fields(SheConfig):
        key = "config." + f.name
        if key in z:
            v = z[key]
            ck[f.name] = v.item() if v.ndim == 0 else v
    return dev, SheConfig(**ck)


_OPT_KEYS = ("precision", "precond", "ordering", "tol", "max_iters", "trsv", "check_every", "shadow",
             "fill_level", "ilut_entries", "ilut_drop")


def save_system(path, rp, ci, values, rhs, blocks=None, **opts):
    """A CSR system with its slab bounds and solver options (make_opts keywords)."""
    unknown = set(opts) - set(_OPT_KEYS)
    if unknown:
        raise ValueError("options not stored in a system file: %s" % sorted(unknown))
    arrays = {"system.row_ptr": np.ascontiguousarray(rp, np.int64), "system.col": np.ascontiguousarray(ci, np.int32),
              "system.val": np.ascontiguousarray(values, np.float64), "system.rhs": np.ascontiguousarray(rhs, np.float64)}
    n = len(arrays["system.row_ptr"]) - 1
    if arrays["system.row_ptr"][-1] != len(arrays["system.col"]) or len(arrays["system.col"]) != len(arrays["system.val"]):
        raise ValueError("row_ptr, col and val do not describe one CSR matrix")
    if len(arrays["system.rhs"]) != n:
        raise ValueError("rhs has %d entries for %d rows" % (len(arrays["system.rhs"]), n))
    if blocks is not None:
        arrays["system.blocks"] = np.ascontiguousarray(blocks, np.int64)
    for k, v in opts.items():
        arrays["opts." + k] = np.asarray(v)
    np.savez(path, **arrays)


def load_system(path):
    """-> dict(rp, ci, values, rhs, blocks (or None), opts: the make_opts keywords stored)."""
    z = np.load(path, allow_pickle=False)
    opts = {}
    for k in _OPT_KEYS:
        if "opts." + k in z:
            v = z["opts." + k]
            opts[k] = v.item() if v.ndim == 0 else v
    return {"rp": z["system.row_ptr"], "ci": z["system.col"], "values": z["system.val"], "rhs": z["system.rhs"],
            "blocks": z["system.blocks"] if "system.blocks" in z else None, "opts": opts}


def write_gnuplot(path, dev: Device, values, cells=None):
    """values: one number (or a vector of numbers) per cell; cells: the cells to write (all by
    default), in cell order."""
    cen = np.asarray(dev.cell_centroid, np.float64).reshape(dev.n_cells, dev.dim)
    vals = np.asarray(values, np.float64)
    idx = range(dev.n_cells) if cells is None else cells
    with open(path, "w") as f:
        f.write("## ViennaSHE - gnuplot output \n")
        for c in idx:
            line = "".join("%g " % x for x in cen[c])
            v = vals[c]
            line += "".join("%g " % x for x in np.atleast_1d(v))
            f.write(line + "\n")


_Q = 1.602176565e-19   # viennashe/physics/constants.hpp
# Y_0^0 as the reference evaluates it (viennashe/math/spherical_harmonics.hpp:100-115): the
# normalisation sqrt((2l+1) (l-m)! / (2 pi (l+m)!)) times P_0^0 = 1, over sqrt(2) for m = 0
_Y00 = math.sqrt((2.0 * 0 + 1.0) * 1.0 / (2.0 * math.pi * 1.0)) * 1.0 / math.sqrt(2.0)


def edf_values(space, x_full):
    """The energy distribution function f_00 Y_00 per cell and energy (shape (n_cells, N_H)) from a
    full solution, as the reference's edf_wrapper returns it at a node's own kinetic energy
    (viennashe/she/df_wrappers.hpp:517-562, even-odd DF discretisation): the node's first even
    unknown times Y_0^0; 0 where the node has no unknown."""
    idx = space["even_index"]
    x = np.asarray(x_full, np.float64)
    out = np.zeros(idx.shape)
    m = idx >= 0
    out[m] = x[idx[m]] * _Y00
    return out


def _cell_list(dev, cells):
    if cells is None:
        return range(dev.n_cells)
    if callable(cells):
        return [c for c in range(dev.n_cells) if cells(c)]
    return cells


def write_gnuplot_edf(path, dev: Device, space, x_full, cells=None):
    """The reference's EDF writer with a cell filter (gnuplot_writer_edf.hpp:117-175): for every
    cell that passes (cells: None = all, a callable on the cell index, or a list of cells), one
    line per interior energy with an unknown and a positive kinetic energy -- the centroid
    coordinates, the kinetic energy in eV, the EDF and the density of states -- then two empty
    lines (a gnuplot block).  Numbers as C++ streams print doubles by default (%g)."""
    cen = np.asarray(dev.cell_centroid, np.float64).reshape(dev.n_cells, dev.dim)
    idx, eps, dos = space["even_index"], space["kinetic_energy"], space["density_of_states"]
    f_edf = edf_values(space, x_full)
    nh = idx.shape[1]
    with open(path, "w") as f:
        for c in _cell_list(dev, cells):
            pre = "".join("%g " % v for v in cen[c])
            for h in range(1, nh - 1):
                if idx[c, h] > -1 and eps[c, h] > 0:
                    f.write(pre + "%g %g %g\n" % (eps[c, h] / _Q, f_edf[c, h], dos[c, h]))
            f.write("\n\n")


def write_gnuplot_edf_line(path, dev: Device, space, x_full, coordinate_x):
    """The reference's EDF writer along a vertical line of a 2D device (gnuplot_writer_edf.hpp:
    54-110): the cells whose centroid has x == coordinate_x, every interior energy with an unknown,
    as lines "y kinetic_energy(J) EDF" sorted by (y, kinetic energy), with an empty line before
    each new y (and before the first, as the reference starts from y = -1)."""
    if dev.dim < 2:
        raise ValueError("write_gnuplot_edf_line needs a 2D device (it sorts by the centroid's y)")
    cen = np.asarray(dev.cell_centroid, np.float64).reshape(dev.n_cells, dev.dim)
    idx, eps = space["even_index"], space["kinetic_energy"]
    f_edf = edf_values(space, x_full)
    nh = idx.shape[1]
    values = {}
    for c in range(dev.n_cells):
        if cen[c, 0] != coordinate_x:
            continue
        for h in range(1, nh - 1):
            if idx[c, h] > -1:
                values[(float(cen[c, 1]), float(eps[c, h]))] = f_edf[c, h]
    last_y = -1.0
    with open(path, "w") as f:
        for (y, e) in sorted(values):
            if y != last_y:
                f.write("\n")
                last_y = y
            f.write("%g %g %g\n" % (y, e, values[(y, e)]))


def write_vtk(path, dev: Device, fields: dict, title="ViennaSHE B200 results"):
    """fields: name -> one value per cell.  Legacy VTK POLYDATA, ASCII."""
    cen = np.asarray(dev.cell_centroid, np.float64).reshape(dev.n_cells, dev.dim)
    pts = np.zeros((dev.n_cells, 3))
    pts[:, :dev.dim] = cen
    with open(path, "w") as f:
        f.write("# vtk DataFile Version 3.0\n%s\nASCII\nDATASET POLYDATA\n" % title)
        f.write("POINTS %d double\n" % dev.n_cells)
        for p in pts:
            f.write("%.17g %.17g %.17g\n" % tuple(p))
        f.write("VERTICES %d %d\n" % (dev.n_cells, 2 * dev.n_cells))
        for c in range(dev.n_cells):
            f.write("1 %d\n" % c)
        f.write("POINT_DATA %d\n" % dev.n_cells)
        for name, v in fields.items():
            v = np.asarray(v, np.float64)
            f.write("SCALARS %s double 1\nLOOKUP_TABLE default\n" % name.replace(" ", "_"))
            for x in v:
                f.write("%.17g\n" % x)


def read_vtk_fields(path):
    """Reads back what write_vtk wrote -> (points (n, 3), {name: values})."""
    with open(path) as f:
        tok = f.read().split("\n")
    i = 0
    pts, fields = None, {}
    while i < len(tok):
        line = tok[i].strip()
        if line.startswith("POINTS"):
            n = int(line.split()[1])
            pts = np.array([[float(x) for x in tok[i + 1 + k].split()] for k in range(n)])
            i += n + 1
            continue
        if line.startswith("SCALARS"):
            name = line.split()[1]
            vals = np.array([float(tok[i + 2 + k]) for k in range(len(pts))])
            fields[name] = vals
            i += 2 + len(pts)
            continue
        i += 1
    return pts, fields

"""Files of the SHE path: requests on disk and results for plotting.

* ``save_request`` / ``load_request``: a served request (the device description of
  ``vshe_device_desc`` and the SHE configuration of ``vshe_she_config``) as one ``.npz`` file:
  flat arrays under the C field names, so a request can be replayed or exchanged without the
  generator that made it.
* ``write_gnuplot``: a per-cell quantity in the layout of the reference's gnuplot writer
  (viennashe/io/gnuplot_writer.hpp:47-118): a ``## ViennaSHE - gnuplot output`` line, then one
  line per cell with the centroid coordinates and the value, each followed by a space, numbers
  as C++ streams print doubles by default (``%g``).
* ``write_vtk``: per-cell quantities as a legacy-format VTK point cloud at the cell centroids.
  The reference's VTK writers (viennashe/io/she_vtk_writer.hpp) write the mesh cells; a
  ``vshe_device_desc`` carries no vertices, so the cells are written as points.
"""
from __future__ import annotations

import dataclasses

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

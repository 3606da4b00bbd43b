"""ctypes mirror of include/vshe_types.h and include/vshe_gpu.h.

The library (libvshe_b200.so) is C++/CUDA behind a C ABI; this module only
marshals numpy arrays into the plain structs and pointers the ABI takes.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(os.path.dirname(_HERE), "lib", "libvshe_b200.so")

i32p = C.POINTER(C.c_int32)
i64p = C.POINTER(C.c_int64)
f64p = C.POINTER(C.c_double)
f32p = C.POINTER(C.c_float)


class DeviceDescC(C.Structure):
    _fields_ = [
        ("dim", C.c_int32), ("n_cells", C.c_int32), ("n_facets", C.c_int32),
        ("cell_material", i32p), ("cell_volume", f64p), ("cell_centroid", f64p),
        ("doping_n", f64p), ("doping_p", f64p), ("potential", f64p), ("contact_id", i32p),
        ("facet_cells", i32p), ("facet_volume", f64p), ("facet_normal", f64p),
        ("cell_facet_ptr", i32p), ("cell_facet_idx", i32p), ("temperature", C.c_double),
    ]


class SheConfigC(C.Structure):
    _fields_ = [
        ("max_expansion_order", C.c_int32), ("energy_spacing", C.c_double),
        ("min_kinetic_energy_range", C.c_double), ("max_kinetic_energy_range", C.c_double),
        ("acoustic_phonon", C.c_int32), ("optical_phonon", C.c_int32),
        ("acoustic_fit_factor", C.c_double), ("optical_fit_factor", C.c_double),
        ("boundary_type", C.c_int32), ("gr_tau", C.c_double), ("scaling_type", C.c_int32),
        ("scale", C.c_int32),
    ]


class CouplingC(C.Structure):
    _fields_ = [("L", C.c_int32), ("data", f64p)]


class SolveOptsC(C.Structure):
    _fields_ = [
        ("precision", C.c_int32), ("precond", C.c_int32), ("ordering", C.c_int32),
        ("tol", C.c_double), ("max_iters", C.c_int32), ("inner_tol", C.c_double),
        ("max_refinements", C.c_int32), ("n_blocks", C.c_int64), ("block_ptr", i64p),
        ("trsv_mode", C.c_int32), ("check_every", C.c_int32), ("perm", C.POINTER(C.c_int32)),
        ("shadow", C.c_int32), ("fill_level", C.c_int32), ("ilut_entries", C.c_int32), ("ilut_drop", C.c_double),
    ]


class SolveStatsC(C.Structure):
    _fields_ = [
        ("status", C.c_int32), ("iterations", C.c_int32), ("refinements", C.c_int32),
        ("rel_residual", C.c_double), ("setup_ms", C.c_double), ("solve_ms", C.c_double),
        ("levels_L", C.c_int32), ("levels_U", C.c_int32), ("bytes_device", C.c_int64),
        ("sweep_ctas", C.c_int32), ("tile_rows", C.c_int32), ("sweep_mode", C.c_int32),
    ]


def ptr(a, ctype):
    return a.ctypes.data_as(C.POINTER(ctype))


class DeviceDesc:
    """Keeps the numpy arrays alive while the C struct points into them."""

    def __init__(self, dev):
        self._keep = []

        def arr(x, dt):
            a = np.ascontiguousarray(x, dtype=dt)
            self._keep.append(a)
            return a
        s = DeviceDescC()
        s.dim = dev.dim
        s.n_cells = dev.n_cells
        s.n_facets = dev.n_facets
        s.cell_material = ptr(arr(dev.cell_material, np.int32), C.c_int32)
        s.cell_volume = ptr(arr(dev.cell_volume, np.float64), C.c_double)
        s.cell_centroid = ptr(arr(dev.cell_centroid, np.float64), C.c_double)
        s.doping_n = ptr(arr(dev.doping_n, np.float64), C.c_double)
        s.doping_p = ptr(arr(dev.doping_p, np.float64), C.c_double)
        s.potential = ptr(arr(dev.potential, np.float64), C.c_double)
        s.contact_id = ptr(arr(dev.contact_id, np.int32), C.c_int32)
        s.facet_cells = ptr(arr(dev.facet_cells, np.int32), C.c_int32)
        s.facet_volume = ptr(arr(dev.facet_volume, np.float64), C.c_double)
        s.facet_normal = ptr(arr(dev.facet_normal, np.float64), C.c_double)
        s.cell_facet_ptr = ptr(arr(dev.cell_facet_ptr, np.int32), C.c_int32)
        s.cell_facet_idx = ptr(arr(dev.cell_facet_idx, np.int32), C.c_int32)
        s.temperature = float(dev.temperature)
        self.c = s


def she_config_c(cfg):
    s = SheConfigC()
    s.max_expansion_order = int(cfg.max_expansion_order)
    s.energy_spacing = float(cfg.energy_spacing)
    s.min_kinetic_energy_range = float(cfg.min_kinetic_energy_range)
    s.max_kinetic_energy_range = float(cfg.max_kinetic_energy_range)
    s.acoustic_phonon = int(bool(cfg.acoustic_phonon))
    s.optical_phonon = int(bool(cfg.optical_phonon))
    s.acoustic_fit_factor = float(cfg.acoustic_fit_factor)
    s.optical_fit_factor = float(cfg.optical_fit_factor)
    s.boundary_type = int(cfg.boundary_type)
    s.gr_tau = float(cfg.gr_tau)
    s.scaling_type = int(cfg.scaling_type)
    s.scale = int(bool(cfg.scale))
    return s


class Coupling:
    def __init__(self, L, data):
        self.data = np.ascontiguousarray(data, dtype=np.float64)
        D = (L + 1) ** 2
        assert self.data.shape == (6, D, D)
        self.c = CouplingC(int(L), ptr(self.data, C.c_double))

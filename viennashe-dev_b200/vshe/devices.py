"""Seeded synthetic devices on structured 1D/2D meshes (flat vshe_device_desc arrays).

The reference builds its devices with ViennaGrid (viennashe/util/generate_device.hpp)
and takes the potential from its Poisson/drift-diffusion solve.  This module is
the stand-in used to feed the SHE linear-solve path: it generates the mesh,
doping and a frozen potential profile, deterministically from a seed.

Mesh convention (it fixes the odd unknown numbering, i.e. the S^oo block):
  * cells: segment by segment; in 2D row-major with x fastest (y-outer,
    x-inner), as generate_device.hpp:435-448 orders them;
  * 1D facets are the mesh vertices left to right; facet k lies between
    cells k-1 and k; the cells on a facet are listed (left, right);
  * 2D facets are created cell by cell in the order bottom, left, right, top
    (a quadrilateral's edges [0,1], [0,2], [1,3], [2,3]), skipping edges that
    already exist; the cells on a facet are listed in creation order, so c1
    is the lower-numbered cell;
  * the facets of a cell are listed in its local order: (left, right) in 1D,
    (bottom, left, right, top) in 2D.

Potential: the built-in potential of the (smoothed) doping plus a linear ramp
of the applied bias between the contacts, then smoothed with a Gaussian
(sigma = 5 nm).  Contact (metal) cells carry their Dirichlet value, contact
potential + built-in potential of the neighbouring semiconductor doping
(viennashe/accessors.hpp:205-227).  This is a frozen analytic profile, not a
self-consistent Poisson solution.
"""
from __future__ import annotations

import dataclasses
import math
from typing import List, Optional

import numpy as np

Q = 1.602176565e-19
KB = 1.3806488e-23
SI, METAL = 0, 100
HBAR_OMEGA_OP = 1.24 * (Q / 20.0)   # 62 meV optical phonon energy


def _built_in_potential(T, nd, na):
    """viennashe/physics/physics.hpp:125-148 (vectorised)."""
    eg = 1.11 * Q
    ncv0 = 2.50933670314359713002e19 * 100 * 100 * 100
    nc = ncv0 * (0.33 * (T / 300.0)) ** 1.5 * 6.0
    nv = ncv0 * (0.6 * (T / 300.0)) ** 1.5 * 6.0
    naux = nc * math.exp(-eg * 0.5 / (KB * T))
    paux = nv * math.exp(-eg * 0.5 / (KB * T))
    net = np.asarray(nd, float) - np.asarray(na, float)
    x = np.sqrt(net * net + 4.0 * naux * paux)
    pos = net >= 0
    out = np.empty_like(net)
    out[pos] = T * np.log((x[pos] + net[pos]) * 0.5 / naux) * KB / Q
    out[~pos] = -T * np.log((x[~pos] - net[~pos]) * 0.5 / paux) * KB / Q
    return out


def _gauss_smooth_1d(v, h, sigma):
    if sigma <= 0:
        return v
    r = int(math.ceil(3 * sigma / h))
    k = np.exp(-0.5 * (np.arange(-r, r + 1) * h / sigma) ** 2)
    k /= k.sum()
    pad = np.pad(v, r, mode="edge")
    return np.convolve(pad, k, mode="valid")


@dataclasses.dataclass
class Device:
    """Flat arrays matching vshe_device_desc (include/vshe_types.h)."""
    dim: int
    cell_material: np.ndarray      # int32
    cell_volume: np.ndarray        # float64
    cell_centroid: np.ndarray      # float64 (n_cells, dim)
    doping_n: np.ndarray
    doping_p: np.ndarray
    potential: np.ndarray
    contact_id: np.ndarray         # int32, -1 for non-contact cells
    facet_cells: np.ndarray        # int32 (n_facets, 2)
    facet_volume: np.ndarray
    facet_normal: np.ndarray       # (n_facets, dim)
    cell_facet_ptr: np.ndarray     # int32
    cell_facet_idx: np.ndarray     # int32
    temperature: float = 300.0
    contact_potential: Optional[np.ndarray] = None  # per contact, V
    name: str = ""

    @property
    def n_cells(self):
        return int(self.cell_material.shape[0])

    @property
    def n_facets(self):
        return int(self.facet_cells.shape[0])

    @property
    def n_contacts(self):
        return int(self.contact_id.max()) + 1 if (self.contact_id >= 0).any() else 0


def facet_centres(dev: Device) -> np.ndarray:
    """Facet centres (n_facets, dim) for the outer loop's Poisson system: the midpoint of the two
    cell centroids of an interior facet (exact on the uniform tensor meshes built here), the
    cell centroid on a boundary facet (which the Poisson system does not use)."""
    fc = dev.facet_cells
    cen = dev.cell_centroid.reshape(dev.n_cells, dev.dim)
    c1 = cen[fc[:, 0]]
    c2 = np.where((fc[:, 1] >= 0)[:, None], cen[np.maximum(fc[:, 1], 0)], c1)
    return np.ascontiguousarray(0.5 * (c1 + c2))


@dataclasses.dataclass
class SheConfig:
    """Mirror of vshe_she_config; defaults follow viennashe/config.hpp:131-159."""
    max_expansion_order: int = 1
    energy_spacing: float = 31.0 * Q / 1000.0
    min_kinetic_energy_range: float = Q
    max_kinetic_energy_range: float = 5.0 * Q
    acoustic_phonon: bool = True
    optical_phonon: bool = True
    acoustic_fit_factor: float = 1.05
    optical_fit_factor: float = 0.7
    boundary_type: int = 0          # generation/recombination
    gr_tau: float = 1e-16
    scaling_type: int = 0           # kinetic energy
    scale: bool = True


def _mesh_1d(xs_nodes):
    n = len(xs_nodes) - 1
    h = np.diff(xs_nodes)
    cen = (0.5 * (xs_nodes[:-1] + xs_nodes[1:])).reshape(-1, 1)
    fc = np.full((n + 1, 2), -1, np.int32)
    fc[0, 0] = 0
    for k in range(1, n):
        fc[k] = (k - 1, k)
    fc[n, 0] = n - 1
    cfp = np.arange(0, 2 * n + 1, 2, dtype=np.int32)
    cfi = np.empty(2 * n, np.int32)
    cfi[0::2] = np.arange(n)
    cfi[1::2] = np.arange(1, n + 1)
    return h, cen, fc, np.ones(n + 1), np.ones((n + 1, 1)), cfp, cfi


def _mesh_2d(nx, ny, hx, hy):
    """Quad mesh, cells row-major (x fastest); facets created per cell in the order
    bottom, left, right, top, skipping existing ones."""
    ncell = nx * ny
    cen = np.empty((ncell, 2))
    jj, ii = np.meshgrid(np.arange(ny), np.arange(nx), indexing="ij")
    cen[:, 0] = ((ii + 0.5) * hx).ravel()
    cen[:, 1] = ((jj + 0.5) * hy).ravel()
    hedge = -np.ones((ny + 1, nx), np.int64)   # horizontal edge (j, i): bottom of cell (i, j)
    vedge = -np.ones((ny, nx + 1), np.int64)   # vertical edge (j, i): left of cell (i, j)
    fcells: List[List[int]] = []
    fvol: List[float] = []
    fnorm: List[List[float]] = []
    cfi = np.empty(4 * ncell, np.int32)
    for j in range(ny):
        for i in range(nx):
            c = j * nx + i
            loc = []
            for kind, (a, b) in (("h", (j, i)), ("v", (j, i)), ("v", (j, i + 1)), ("h", (j + 1, i))):
                tab = hedge if kind == "h" else vedge
                if tab[a, b] < 0:
                    tab[a, b] = len(fcells)
                    fcells.append([c, -1])
                    fvol.append(hx if kind == "h" else hy)
                    fnorm.append([0.0, 1.0] if kind == "h" else [1.0, 0.0])
                else:
                    fcells[tab[a, b]][1] = c
                loc.append(tab[a, b])
            cfi[4 * c:4 * c + 4] = loc
    fc = np.asarray(fcells, np.int32)
    fn = np.asarray(fnorm)
    # orient the normal from c1 to c2 (cells are created in increasing x/y, so c2 is
    # to the right/top of c1 and the +x/+y normal is already c1 -> c2)
    return (np.full(ncell, hx * hy), cen, fc, np.asarray(fvol), fn,
            np.arange(0, 4 * ncell + 1, 4, dtype=np.int32), cfi)


def nin_diode_1d(lengths=(50e-9, 150e-9, 50e-9), dopings=(1e25, 1e21, 1e25), boxes=250, bias=0.5,
                 contact_boxes=1, T=300.0, smooth=5e-9, name="nin1d"):
    """1D n+/n/n+ diode with one metal contact box on each side (uniform boxes)."""
    total = sum(lengths)
    h = total / boxes
    n = boxes + 2 * contact_boxes
    xs = np.arange(n + 1) * h - contact_boxes * h
    vol, cen, fc, fvol, fn, cfp, cfi = _mesh_1d(xs)
    x = cen[:, 0]
    mat = np.full(n, SI, np.int32)
    contact = np.full(n, -1, np.int32)
    mat[:contact_boxes] = METAL
    mat[-contact_boxes:] = METAL
    contact[:contact_boxes] = 0
    contact[-contact_boxes:] = 1
    nd = np.zeros(n)
    edges = np.cumsum((0.0,) + tuple(lengths))
    for k in range(3):
        sel = (x >= edges[k]) & (x < edges[k + 1])
        nd[sel] = dopings[k]
    nd[:contact_boxes] = dopings[0]
    nd[-contact_boxes:] = dopings[2]
    na = np.zeros(n)
    semi = mat == SI
    phi_bi = _built_in_potential(T, nd, na)
    ramp = np.clip((x - 0.0) / total, 0.0, 1.0) * bias
    phi = _gauss_smooth_1d(phi_bi + ramp, h, smooth)
    cpot = np.array([0.0, bias])
    # contact cells: contact potential + built-in potential of the neighbouring doping
    phi[:contact_boxes] = cpot[0] + _built_in_potential(T, [dopings[0]], [0.0])[0]
    phi[-contact_boxes:] = cpot[1] + _built_in_potential(T, [dopings[2]], [0.0])[0]
    return Device(1, mat, vol, cen, nd, na, phi, contact, fc, fvol, fn, cfp, cfi, T, cpot, name)


def nin_bar_2d(nx=200, ny=50, lx=400e-9, ly=100e-9, n_contact=1e25, n_channel=1e22, bias=0.8,
               contact_frac=0.25, sigma=5e-9, seed=7, T=300.0, name="nin2d"):
    """2D n+/n/n+ bar with metal contact columns at x = 0 and x = lx.  The n+/n edges
    have Gaussian (sigma) profiles whose positions are jittered per row from `seed`."""
    rng = np.random.default_rng(seed)
    hx, hy = lx / nx, ly / ny
    NX = nx + 2
    vol, cen, fc, fvol, fn, cfp, cfi = _mesh_2d(NX, ny, hx, hy)
    cen[:, 0] -= hx
    x, y = cen[:, 0], cen[:, 1]
    ii = np.tile(np.arange(NX), ny)
    mat = np.where((ii == 0) | (ii == NX - 1), METAL, SI).astype(np.int32)
    contact = np.full(NX * ny, -1, np.int32)
    contact[ii == 0] = 0
    contact[ii == NX - 1] = 1
    # jittered edge positions: a smooth random perturbation along y (amplitude ~ sigma)
    modes = rng.uniform(-1, 1, size=(2, 3)) * sigma
    phases = rng.uniform(0, 2 * np.pi, size=(2, 3))
    def edge(k, yy):
        return sum(modes[k, m] * np.sin((m + 1) * np.pi * yy / ly + phases[k, m]) for m in range(3))
    xl = contact_frac * lx + edge(0, y)
    xr = (1 - contact_frac) * lx + edge(1, y)
    from math import erf
    verf = np.vectorize(erf)
    s = sigma * math.sqrt(2.0)
    frac = 0.5 * (1 + verf((xl - x) / s)) + 0.5 * (1 + verf((x - xr) / s))
    frac = np.clip(frac, 0.0, 1.0)
    logn = np.log(n_channel) + frac * (np.log(n_contact) - np.log(n_channel))
    nd = np.exp(logn)
    na = np.zeros_like(nd)
    phi_bi = _built_in_potential(T, nd, na)
    ramp = np.clip(x / lx, 0.0, 1.0) * bias
    phi = (phi_bi + ramp).reshape(ny, NX)
    # separable Gaussian smoothing (sigma = 5 nm) of the semiconductor potential
    for axis, hh in ((1, hx), (0, hy)):
        phi = np.apply_along_axis(lambda v: _gauss_smooth_1d(v, hh, 5e-9), axis, phi)
    phi = phi.ravel()
    cpot = np.array([0.0, bias])
    left, right = ii == 0, ii == NX - 1
    phi[left] = cpot[0] + _built_in_potential(T, nd[left], na[left])
    phi[right] = cpot[1] + _built_in_potential(T, nd[right], na[right])
    return Device(2, mat, vol, cen, nd, na, phi, contact, fc, fvol, fn, cfp, cfi, T, cpot, name)


def energy_range_for(dev: Device, spacing: float, n_energies: int) -> float:
    """min_kinetic_energy_range that makes setup_energies (she/setup_energies.hpp:108-120)
    produce exactly n_energies energy points for this device's potential."""
    semi = dev.cell_material == SI
    dphi = float(dev.potential[semi].max() - dev.potential[semi].min())
    return (n_energies - 1 + 0.5) * spacing - Q * dphi - 2.0 * spacing


# ------------------------------------------------------------------ workloads
def config1():
    """1D silicon n+/n/n+ diode 50/150/50 nm, 1e25/1e21/1e25 m^-3, 250 boxes, L = 1,
    spacing hbar*omega_op/4, 1.5 eV kinetic range, 0.5 V."""
    dev = nin_diode_1d(bias=0.5, name="config1_nin1d_250")
    cfg = SheConfig(max_expansion_order=1, energy_spacing=HBAR_OMEGA_OP / 4.0, min_kinetic_energy_range=1.5 * Q)
    return dev, cfg


def config2(nx=200, ny=50, n_energies=160, L=3, bias=0.8):
    """2D n+/n/n+ bar 400 x 100 nm on a 200 x 50 quad mesh, contacts 1e25, channel 1e22,
    Gaussian lateral edges (sigma 5 nm, seed 7), L = 3, 160 energies, 0.8 V."""
    dev = nin_bar_2d(nx=nx, ny=ny, bias=bias, seed=7, name="config2_nin2d_%dx%d" % (nx, ny))
    sp = HBAR_OMEGA_OP / 4.0
    cfg = SheConfig(max_expansion_order=L, energy_spacing=sp, min_kinetic_energy_range=energy_range_for(dev, sp, n_energies))
    return dev, cfg


def config3(count=64, seed=11):
    """Batched bias sweep: `count` 1D n+/n/n+ diodes from `seed` (length U[100, 500] nm,
    50-400 boxes, channel log-U[1e21, 1e23], contacts 1e25, L in {1, 3}, bias U[0, 1] V)."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(count):
        length = rng.uniform(100e-9, 500e-9)
        boxes = int(rng.integers(50, 401))
        nch = float(np.exp(rng.uniform(np.log(1e21), np.log(1e23))))
        L = int(rng.choice([1, 3]))
        bias = float(rng.uniform(0.0, 1.0))
        lens = (0.2 * length, 0.6 * length, 0.2 * length)
        dev = nin_diode_1d(lengths=lens, dopings=(1e25, nch, 1e25), boxes=boxes, bias=bias, name="config3_%02d" % k)
        cfg = SheConfig(max_expansion_order=L, energy_spacing=HBAR_OMEGA_OP / 4.0, min_kinetic_energy_range=1.0 * Q)
        out.append((dev, cfg))
    return out


def config4(count=40, seed=23, rate=200.0):
    """Served stream: `count` requests arriving as a Poisson process at `rate` req/s (seed 23).
    70 % are 1D n+/n/n+ diodes drawn as in config3; 30 % are 2D bars as in config2 with a mesh of
    50-200 x 20-50 cells, L in {1, 3, 5}, 60-160 energies and the bar's 0.8 V bias (lateral
    edge jitter from the stream's generator).  Returns [(arrival_s, dev, cfg)]."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for k in range(count):
        t += float(rng.exponential(1.0 / rate))
        if rng.random() < 0.7:
            length = rng.uniform(100e-9, 500e-9)
            boxes = int(rng.integers(50, 401))
            nch = float(np.exp(rng.uniform(np.log(1e21), np.log(1e23))))
            L = int(rng.choice([1, 3]))
            bias = float(rng.uniform(0.0, 1.0))
            lens = (0.2 * length, 0.6 * length, 0.2 * length)
            dev = nin_diode_1d(lengths=lens, dopings=(1e25, nch, 1e25), boxes=boxes, bias=bias, name="config4_%03d_1d" % k)
            cfg = SheConfig(max_expansion_order=L, energy_spacing=HBAR_OMEGA_OP / 4.0, min_kinetic_energy_range=1.0 * Q)
        else:
            nx = int(rng.integers(50, 201))
            ny = int(rng.integers(20, 51))
            L = int(rng.choice([1, 3, 5]))
            ne = int(rng.integers(60, 161))
            dev = nin_bar_2d(nx=nx, ny=ny, bias=0.8, seed=int(rng.integers(0, 2 ** 31)), name="config4_%03d_2d" % k)
            sp = HBAR_OMEGA_OP / 4.0
            cfg = SheConfig(max_expansion_order=L, energy_spacing=sp, min_kinetic_energy_range=energy_range_for(dev, sp, ne))
        out.append((t, dev, cfg))
    return out


def mosfet_2d(nx=240, ny=80, lx=300e-9, ly=150e-9, n_sd=1e26, n_body=1e23, v_drain=1.0, v_gate=1.0,
              well_len=75e-9, well_depth=40e-9, sigma=5e-9, gate_decay=20e-9, T=300.0, name="mosfet2d"):
    """Three-terminal MOSFET-like structure: a p-type body (acceptors n_body) with n+ source and
    drain wells (donors n_sd, Gaussian edges of width sigma) under the top surface at both ends,
    metal source / drain contact cells beside the wells (contacts 0 and 1), and a gate modelled
    as a fixed-potential top boundary at v_gate: it enters only through the frozen potential,
    which adds to the built-in potential the drain bias across the channel and the gate bias
    decaying from the top surface (gate_decay), smoothed with a 5 nm Gaussian.  The gate carries
    no SHE current (it is insulated), so the SHE sees two contacts."""
    hx, hy = lx / nx, ly / ny
    NX = nx + 2
    vol, cen, fc, fvol, fn, cfp, cfi = _mesh_2d(NX, ny, hx, hy)
    cen[:, 0] -= hx
    x, y = cen[:, 0], cen[:, 1]
    ii = np.tile(np.arange(NX), ny)
    top = y > ly - well_depth
    mat = np.full(NX * ny, SI, np.int32)
    contact = np.full(NX * ny, -1, np.int32)
    src = (ii == 0) & top
    drn = (ii == NX - 1) & top
    mat[src | drn] = METAL
    contact[src] = 0
    contact[drn] = 1
    from math import erf
    verf = np.vectorize(erf)
    s = sigma * math.sqrt(2.0)
    depth = 0.5 * (1 + verf((y - (ly - well_depth)) / s))
    wl = 0.5 * (1 + verf((well_len - x) / s))
    wr = 0.5 * (1 + verf((x - (lx - well_len)) / s))
    frac = np.clip((wl + wr) * depth, 0.0, 1.0)
    nd = np.maximum(np.exp(np.log(1.0) + frac * np.log(n_sd)) - 1.0, 0.0)
    na = np.full(NX * ny, n_body)
    phi_bi = _built_in_potential(T, nd, na)
    ramp = np.clip((x - well_len) / (lx - 2 * well_len), 0.0, 1.0) * v_drain
    channel = np.clip(1.0 - wl - wr, 0.0, 1.0)
    gate = v_gate * channel * np.exp(-(ly - y) / gate_decay)
    phi = (phi_bi + ramp + gate).reshape(ny, NX)
    for axis, hh in ((1, hx), (0, hy)):
        phi = np.apply_along_axis(lambda v: _gauss_smooth_1d(v, hh, 5e-9), axis, phi)
    phi = phi.ravel()
    cpot = np.array([0.0, v_drain])
    phi[src] = cpot[0] + _built_in_potential(T, nd[src], na[src] * 0.0)
    phi[drn] = cpot[1] + _built_in_potential(T, nd[drn], na[drn] * 0.0)
    return Device(2, mat, vol, cen, nd, na, phi, contact, fc, fvol, fn, cfp, cfi, T, cpot, name)


def config5(nx=240, ny=80, n_energies=140, L=5):
    """MOSFET-like structure of 300 x 150 nm on a 240 x 80 mesh, source / drain wells 1e26 m^-3,
    body 1e23 m^-3, gate (top boundary) and drain at 1.0 V, SHE order L = 5, 140 energies."""
    dev = mosfet_2d(nx=nx, ny=ny, name="config5_mosfet_%dx%d" % (nx, ny))
    sp = HBAR_OMEGA_OP / 4.0
    cfg = SheConfig(max_expansion_order=L, energy_spacing=sp, min_kinetic_energy_range=energy_range_for(dev, sp, n_energies))
    return dev, cfg

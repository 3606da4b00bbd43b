// she_host.cpp -- host setup of the SHE (x, H) space (product code).
//
// Restates, on flat arrays, what ViennaSHE computes on the host before
// assembly:
//   * energies and band-edge shifts   viennashe/she/setup_energies.hpp:61-153
//   * expansion orders                viennashe/she/expansion_order.hpp:60-129, 140-199, 262-364
//   * SHE unknown mask                viennashe/simulator.hpp:94-120
//   * boundary values                 viennashe/she/boundary_conditions.hpp:57-134,
//                                     viennashe/accessors.hpp:51-81, 316-367
//   * unknown numbering (H-major)     viennashe/mapping.hpp:97-323
//   * energy-slab blocks              viennashe/she/linear_solver.hpp:44-83
//   * coupling matrices per direction viennashe/she/assemble_common.hpp:177-290 with the
//     reference matrix type's scalar product (viennashe/math/linalg_util.hpp:151-161,
//     which scales the transposed position) and sum (:163-172).
// The device kernels (she_kernels.cu) assemble, eliminate and normalise from these tables.

#include "she_host.h"

#include <algorithm>
#include <cmath>
#include <limits>
#include <map>
#include <stdexcept>
#include <utility>

namespace vshe {

namespace {
const double PI = SheConst::PI, Q = SheConst::Q, KB = SheConst::KB, M0 = SheConst::M0;
double m_dos() { return 0.32 * M0; }
double m_trans() { return 0.19 * M0; }
double band_gap() { return 1.11 * Q; }
const double HBAR = 6.62606896e-34 / (2.0 * 3.1415926535897932384626433832795);
const double ALPHA = 0.5 / Q;

// Modena dispersion (viennashe/physics/dispersion.hpp:207-286), electrons
double dos(double eps) {
  if (eps > 0.0) {
    const double mstar = m_dos();
    const double prefactor = mstar * std::sqrt(2.0 * mstar) / (8.0 * PI * PI * PI * HBAR * HBAR * HBAR);
    return prefactor * 4.0 * PI * (1.0 + 2.0 * ALPHA * eps) * std::sqrt(eps * (1.0 + ALPHA * eps));
  }
  return 0.0;
}

long even_on_node(long L) { long n = 0; for (long l = 0; l <= L; l += 2) n += 2 * l + 1; return n; }
long odd_on_node(long L) { long n = 0; for (long l = 1; l <= L; l += 2) n += 2 * l + 1; return n; }

// physics.hpp:84-90, 105-148, 158-170
double band_weight(double T, double me) {
  const double Ncv0 = 2.50933670314359713002e19 * 100 * 100 * 100;
  return Ncv0 * std::pow(me * (T / 300.0), 1.5) * 6.0;
}
double built_in_potential(double T, double nd, double na) {
  if (nd <= 0 && na <= 0) return 0;
  const double net = nd - na;
  const double naux = band_weight(T, 0.33) * std::exp(-1.0 * (band_gap() * 0.5) / (KB * T));
  const double paux = band_weight(T, 0.6) * std::exp(1.0 * (-band_gap() * 0.5) / (KB * T));
  double x = std::sqrt(net * net + 4.0 * naux * paux);
  if (net >= 0.0) { x = (x + net) * 0.5 / naux; return T * std::log(x) * KB / Q; }
  x = (x - net) * 0.5 / paux;
  return -T * std::log(x) * KB / Q;
}
double contact_carrier_ohm_n(double T, double nd, double na) {
  const double phiB = built_in_potential(T, nd, na);
  return band_weight(T, 0.33) * std::exp(-1.0 * (band_gap() * 0.5 - Q * phiB) / (KB * T));
}
}  // namespace

double density_of_states(double eps) { return dos(eps); }

// ------------------------------------------------------------------ build
std::string SheSetup::build(const vshe_device_desc &d, const vshe_she_config &c, const vshe_coupling_tables &ct) {
  if (d.dim < 1 || d.dim > 2) return "dim must be 1 or 2";
  if (d.n_cells <= 0 || d.n_facets <= 0) return "empty mesh";
  if (c.max_expansion_order < 1 || c.max_expansion_order % 2 == 0 || c.max_expansion_order > 7) return "max_expansion_order must be 1, 3, 5 or 7";
  if (ct.L != c.max_expansion_order || !ct.data) return "coupling tables must have order max_expansion_order";
  if (!(c.energy_spacing > 0)) return "energy_spacing must be positive";
  dim = d.dim; nc = d.n_cells; nf = d.n_facets; T = d.temperature; cfg = c; L = c.max_expansion_order;
  mat.assign(d.cell_material, d.cell_material + nc);
  vol.assign(d.cell_volume, d.cell_volume + nc);
  cen.assign(d.cell_centroid, d.cell_centroid + size_t(nc) * dim);
  nd.assign(d.doping_n, d.doping_n + nc);
  na.assign(d.doping_p, d.doping_p + nc);
  phi.assign(d.potential, d.potential + nc);
  contact.assign(d.contact_id, d.contact_id + nc);
  fcell.assign(d.facet_cells, d.facet_cells + 2 * size_t(nf));
  fvol.assign(d.facet_volume, d.facet_volume + nf);
  fnorm.assign(d.facet_normal, d.facet_normal + size_t(nf) * dim);
  cf_ptr.assign(d.cell_facet_ptr, d.cell_facet_ptr + nc + 1);
  cf_idx.assign(d.cell_facet_idx, d.cell_facet_idx + cf_ptr[nc]);
  for (int f = 0; f < nf; ++f) {
    if (fcell[2 * f] < 0 || fcell[2 * f] >= nc || fcell[2 * f + 1] >= nc) return "facet_cells out of range";
  }
  for (int k = 0; k < cf_ptr[nc]; ++k)
    if (cf_idx[k] < 0 || cf_idx[k] >= nf) return "cell_facet_idx out of range";

  // optical phonon energy snapped to the grid: optical_phonon_scattering.hpp:66-81
  {
    double w = 1.24 * (Q / 20.0), sp = cfg.energy_spacing;
    size_t steps = size_t(w / sp);
    double e0 = w - steps * sp, e1 = (steps + 1.0) * sp - w;
    if (e1 < e0) ++steps;
    hbar_omega = steps * sp;
  }
  // energies: setup_energies.hpp:61-153
  double maxp = -1.0 * std::numeric_limits<double>::max(), minp = std::numeric_limits<double>::max();
  for (int i = 0; i < nc; ++i) {
    if (!is_semi(i)) continue;
    double v = phi[i] + 0.0;
    minp = std::min(minp, v);
    maxp = std::max(maxp, v);
  }
  if (maxp < minp) return "no semiconductor cells";
  const double dE = cfg.energy_spacing;
  const double range = Q * (maxp - minp) + 2.0 * dE + cfg.min_kinetic_energy_range;
  const double bandedge = -Q * maxp - dE + band_gap() / 2.0;
  const size_t nh = size_t(range / dE) + 1;
  if (nh < 3 || nh > 100000) return "energy range gives fewer than 3 or too many energies";
  NH = int32_t(nh);
  Hval.resize(nh);
  for (size_t h = 0; h < nh; ++h) Hval[h] = bandedge + h * (1.0 * dE);
  shift_c.resize(nc); shift_f.resize(nf);
  for (int i = 0; i < nc; ++i) shift_c[i] = -Q * phi[i] + band_gap() / 2.0;
  for (int f = 0; f < nf; ++f) {
    int c1 = fcell[2 * f], c2 = fcell[2 * f + 1];
    shift_f[f] = c2 >= 0 ? (shift_c[c1] + shift_c[c2]) / 2.0 : shift_c[c1];
  }
  auto box_height = [&](bool facet, int e, int H) {
    auto EK = [&](int h) { return facet ? ekin_f(e, h) : ekin_c(e, h); };
    double hh = 0;
    if (H > 0) hh = std::fabs(EK(H) - EK(H - 1));
    if (H < NH - 1) hh += std::fabs(EK(H + 1) - EK(H));
    return hh / 2.0;
  };
  auto avg_dos = [&](bool facet, int e, int H) {
    auto EK = [&](int h) { return facet ? ekin_f(e, h) : ekin_c(e, h); };
    double Z = dos(EK(H)), n = 1;
    if (H < NH - 1) { Z += dos((EK(H) + EK(H + 1)) / 2.0); ++n; }
    if (H > 0) { Z += dos((EK(H) + EK(H - 1)) / 2.0); ++n; }
    return Z / n;
  };
  // expansion orders: uniform L, lowered to 1 near the band edge, smoothed
  ord_c.assign(size_t(nc) * NH, L);
  ord_f.assign(size_t(nf) * NH, L);
  for (int i = 0; i < nc; ++i) {
    for (int H = 1; H < NH - 1; ++H) {
      if (ekin_c(i, H) <= 0) { ord_c[size_t(i) * NH + H] = 1; continue; }
      bool all_pos = true;
      for (int k = cf_ptr[i]; k < cf_ptr[i + 1]; ++k) {
        int o = other_cell(cf_idx[k], i);
        if (o >= 0 && ekin_c(o, H - 1) <= 0) all_pos = false;
      }
      if (all_pos) break;
      ord_c[size_t(i) * NH + H] = 1;
      for (int k = cf_ptr[i]; k < cf_ptr[i + 1]; ++k) {
        int o = other_cell(cf_idx[k], i);
        if (o >= 0) ord_c[size_t(o) * NH + H] = 1;
      }
    }
  }
  for (int it = 0; it < 10; ++it) {  // expansion_order.hpp:158-196 (second test compares c2 with itself)
    bool changed = false;
    for (int f = 0; f < nf; ++f) {
      int c1 = fcell[2 * f], c2 = fcell[2 * f + 1];
      if (c2 < 0) continue;
      for (int H = 0; H < NH; ++H) {
        int32_t &o1 = ord_c[size_t(c1) * NH + H];
        int32_t o2 = ord_c[size_t(c2) * NH + H];
        if (o1 > o2 + 2) { o1 = o2 + 2; changed = true; }
      }
    }
    if (!changed) break;
  }
  // boundary values
  bnd_c.assign(size_t(nc) * NH, 0.0);
  for (int i = 0; i < nc; ++i) {
    double nd_i = nd[i], na_i = na[i];
    if (is_metal(i)) {
      double dn = 1, dp = 1; long N = 0;
      for (int k = cf_ptr[i]; k < cf_ptr[i + 1]; ++k) {
        int o = other_cell(cf_idx[k], i);
        if (o >= 0 && is_semi(o)) { dn *= nd[o]; dp *= na[o]; ++N; }
      }
      if (N > 1) { dn = std::pow(dn, 1.0 / N); dp = std::pow(dp, 1.0 / N); }
      nd_i = dn; na_i = dp;
    }
    const double dens = contact_carrier_ohm_n(T, nd_i, na_i);
    double corr = 0;
    for (int H = 1; H < NH - 1; ++H) {
      double em = ekin_c(i, H);
      double lo = std::max<double>((ekin_c(i, H - 1) + em) / 2.0, 0.0), up = (ekin_c(i, H + 1) + em) / 2.0;
      if (lo < up && up >= 0) corr += std::exp(-em / (KB * T)) * avg_dos(false, i, H) * box_height(false, i, H);
    }
    corr *= 6.0;
    for (int H = 1; H < NH - 1; ++H) {
      double en = ekin_c(i, H);
      double lo = std::max<double>((ekin_c(i, H - 1) + en) / 2.0, 0.0), up = (ekin_c(i, H + 1) + en) / 2.0;
      double v = 0.0;
      if (lo < up && up >= 0) v = dens * std::exp(-en / (KB * T)) / corr;
      bnd_c[size_t(i) * NH + H] = v;
    }
  }
  // SHE unknown mask and mapping
  mask_c.assign(nc, 0);
  for (int i = 0; i < nc; ++i) {
    if (is_semi(i)) mask_c[i] = 1;
    else if (is_metal(i))
      for (int k = cf_ptr[i]; k < cf_ptr[i + 1]; ++k) {
        int o = other_cell(cf_idx[k], i);
        if (o >= 0 && is_semi(o)) { mask_c[i] = 1; break; }
      }
  }
  idx_c.assign(size_t(nc) * NH, -1);
  idx_f.assign(size_t(nf) * NH, -1);
  even_nodes.clear(); odd_nodes.clear();
  slab_ptr.assign(size_t(NH) + 1, 0);
  int64_t idx = 0;
  for (int H = 0; H < NH; ++H) {
    slab_ptr[H] = idx;
    for (int i = 0; i < nc; ++i) {
      const size_t a = size_t(i) * NH + H;
      if (!mask_c[i] || H == 0 || H == NH - 1) continue;
      if (avg_dos(false, i, H) > 0 && ekin_c(i, H) < cfg.max_kinetic_energy_range) {
        idx_c[a] = idx;
        idx += even_on_node(ord_c[a]);
        even_nodes.push_back(i); even_nodes.push_back(H);
      } else {
        ord_c[a] = 0;
      }
    }
  }
  slab_ptr[NH] = idx;
  n_even = idx;
  // the slab bounds as fill_block_indices (viennashe/she/linear_solver.hpp:44-83) writes them:
  // block H starts at the first unknown of the most recent slab <= H that has unknowns, so the
  // rows of a slab followed by an empty one carry the empty one's index (the row partition is
  // the same)
  {
    int64_t last_found = 0;
    std::vector<int64_t> first(size_t(NH) + 1, 0);
    for (int H = 0; H < NH; ++H) {
      if (slab_ptr[size_t(H) + 1] > slab_ptr[size_t(H)]) last_found = slab_ptr[size_t(H)];
      first[size_t(H)] = last_found;
    }
    first[size_t(NH)] = n_even;
    slab_ptr.swap(first);
  }
  for (int H = 0; H < NH; ++H) {
    for (int f = 0; f < nf; ++f) {
      const size_t a = size_t(f) * NH + H;
      int c1 = fcell[2 * f], c2 = fcell[2 * f + 1];
      if (c2 < 0) { ord_f[a] = 0; continue; }
      int64_t d1 = idx_c[size_t(c1) * NH + H], d2 = idx_c[size_t(c2) * NH + H];
      if (d1 > -1 && d2 > -1 && avg_dos(true, f, H) > 0 && (is_semi(c1) || is_semi(c2))) {
        idx_f[a] = idx;
        idx += odd_on_node(ord_f[a]);
        odd_nodes.push_back(f); odd_nodes.push_back(H);
      } else {
        ord_f[a] = 0;
      }
    }
  }
  n_odd = idx - n_even;
  if (n_even == 0) return "no SHE unknowns";
  if (idx >= (int64_t(1) << 31)) return "more than 2^31 unknowns";

  // harmonic index sequences (spherical_harmonics.hpp:213-252) of order L
  even_harm.clear(); odd_harm.clear();
  for (int l = 0; l <= L; ++l)
    for (int m = -l; m <= l; ++m) (l % 2 == 0 ? even_harm : odd_harm).push_back(l * l + l + m);
  D = (L + 1) * (L + 1);

  // coupling blocks per direction
  const double *tab = ct.data;
  auto A = [&](int t, int i, int j) { return tab[size_t(t) * D * D + size_t(i) * D + j]; };
  const double s = std::sqrt(m_dos() / m_trans());
  // reference scalar product: result(j,i) *= f for every stored (i,j), i.e. an entry is
  // scaled iff its transposed position is stored
  auto Tscaled = [&](int t, bool transpose, double f, int i, int j) {
    double mij = transpose ? A(t, j, i) : A(t, i, j);
    double mji = transpose ? A(t, i, j) : A(t, j, i);
    if (mij == 0.0) return 0.0;
    return mji != 0.0 ? mij * f : mij;
  };
  std::map<std::pair<double, double>, int> dir_id;
  auto get_dir = [&](double u0, double u1) {
    auto key = std::make_pair(u0, u1);
    auto it = dir_id.find(key);
    if (it != dir_id.end()) return it->second;
    int k = int(dir_id.size());
    dir_id[key] = k;
    dirs.push_back(u0); dirs.push_back(u1);
    const size_t base = cblocks.size();
    cblocks.resize(base + 4 * size_t(D) * D, 0.0);
    for (int b = 0; b < 4; ++b) {
      // even rows: diffusion uses p = u, drift p = -u; odd rows (transposed tables) use p = -u
      const double sg = (b == 0) ? 1.0 : -1.0;
      const bool tr = b >= 2;
      const int tx = (b == 0 || b == 2) ? 0 : 3;  // a_x or b_x
      const double f0 = (sg * u0) * s, f1 = (sg * u1) * s;
      for (int i = 0; i < D; ++i)
        for (int j = 0; j < D; ++j) {
          double v = Tscaled(tx, tr, f0, i, j);
          if (dim == 2) {
            const bool has2 = (tr ? A(tx + 1, j, i) : A(tx + 1, i, j)) != 0.0 || (tr ? A(tx + 1, i, j) : A(tx + 1, j, i)) != 0.0;
            if (has2) v = v + Tscaled(tx + 1, tr, f1, i, j);
          }
          cblocks[base + size_t(b) * D * D + size_t(i) * D + j] = v;
        }
    }
    return k;
  };
  auto unit = [&](int from, int to, double &u0, double &u1) {
    double p[2] = {0, 0}, nrm = 0;
    for (int k = 0; k < dim; ++k) { p[k] = cen[size_t(to) * dim + k] - cen[size_t(from) * dim + k]; nrm += p[k] * p[k]; }
    nrm = std::sqrt(nrm);
    u0 = p[0] / nrm; u1 = dim > 1 ? p[1] / nrm : 0.0;
    return nrm > 0;
  };
  inc_dir_even.assign(cf_idx.size(), -1);
  for (int i = 0; i < nc; ++i)
    for (int k = cf_ptr[i]; k < cf_ptr[i + 1]; ++k) {
      int o = other_cell(cf_idx[k], i);
      if (o < 0) continue;
      double u0, u1;
      if (!unit(i, o, u0, u1)) return "two cells share a centroid";
      inc_dir_even[k] = get_dir(u0, u1);
    }
  inc_dir_odd.assign(size_t(nf) * 2, -1);
  for (int f = 0; f < nf; ++f) {
    for (int side = 0; side < 2; ++side) {
      int cc = fcell[2 * f + side];
      if (cc < 0) continue;
      int o = other_cell(f, cc);
      if (o < 0) continue;
      double u0, u1;
      if (!unit(cc, o, u0, u1)) return "two cells share a centroid";
      inc_dir_odd[size_t(f) * 2 + side] = get_dir(u0, u1);
    }
  }
  // L = 1 entries for the current density (current_density.hpp:58-61, 102-112)
  for (int j = 0; j < 3; ++j) { a_x01[j] = A(0, 0, j + 1); a_y01[j] = A(1, 0, j + 1); }
  return "";
}

// ------------------------------------------------------------ multicolour order of the reduced rows
void node_colour_order(const SheSetup &H, int fill_level, std::vector<int32_t> &perm, std::vector<int32_t> *colour) {
  // Colour the (cell, H) nodes so that no two coupled nodes share a colour: cells by a
  // greedy colouring of the mesh graph, energies by the parity of H / n_op (in-scattering
  // couples H and H +- n_op).  All harmonics of a node share its colour; rows are ordered
  // by colour, then by their original position.
  // ILU(k > 0) colours at distance 2 (cells with a common neighbour differ, and energies in
  // three classes of H / n_op), so that the fill does not chain nodes of one colour.
  const bool d2 = fill_level > 0;
  std::vector<int32_t> ccol((size_t)H.nc, -1);
  for (int c = 0; c < H.nc; ++c) {
    uint64_t used = 0;
    for (int k = H.cf_ptr[c]; k < H.cf_ptr[c + 1]; ++k) {
      const int o = H.other_cell(H.cf_idx[k], c);
      if (o < 0) continue;
      if (ccol[(size_t)o] >= 0 && ccol[(size_t)o] < 64) used |= (uint64_t(1) << ccol[(size_t)o]);
      if (!d2) continue;
      for (int k2 = H.cf_ptr[o]; k2 < H.cf_ptr[o + 1]; ++k2) {
        const int o2 = H.other_cell(H.cf_idx[k2], o);
        if (o2 >= 0 && o2 != c && ccol[(size_t)o2] >= 0 && ccol[(size_t)o2] < 64) used |= (uint64_t(1) << ccol[(size_t)o2]);
      }
    }
    int col = 0;
    while (col < 63 && (used >> col) & 1) ++col;
    ccol[(size_t)c] = col;
  }
  const int nop = std::max(1, int(std::lround(H.hbar_omega / H.cfg.energy_spacing)));
  const int nh_classes = d2 ? 3 : 2;
  std::vector<int32_t> rowcol((size_t)H.n_even);
  for (size_t k = 0; k + 1 < H.even_nodes.size(); k += 2) {
    const int c = H.even_nodes[k], h = H.even_nodes[k + 1];
    const int64_t base = H.idx_c[(size_t)c * H.NH + h];
    int ne = 0;
    for (int l = 0; l <= H.ord_c[(size_t)c * H.NH + h]; l += 2) ne += 2 * l + 1;
    const int32_t col = ccol[(size_t)c] * nh_classes + ((h / nop) % nh_classes);
    for (int q = 0; q < ne; ++q) rowcol[(size_t)(base + q)] = col;
  }
  // rows by colour, then position: a stable counting sort over the few colours
  const int32_t ncol = rowcol.empty() ? 1 : *std::max_element(rowcol.begin(), rowcol.end()) + 1;
  std::vector<int64_t> cpos((size_t)ncol + 1, 0);
  for (int32_t c : rowcol) cpos[(size_t)c + 1]++;
  for (int32_t c = 0; c < ncol; ++c) cpos[(size_t)c + 1] += cpos[(size_t)c];
  perm.resize((size_t)H.n_even);
  for (int64_t i = 0; i < H.n_even; ++i) perm[(size_t)cpos[(size_t)rowcol[(size_t)i]]++] = int32_t(i);
  if (colour) colour->swap(rowcol);
}

// ---------------------------------------------------------------- quadrature
namespace {
// associated Legendre P_n^m(x), m >= 0, with the (-1)^n factor on P_n^n
// (viennashe/math/spherical_harmonics.hpp:66-91), by upward recurrence in n.
double assoc_legendre(int n, int m, double x) {
  double pmm = 1.0;
  const double sx = std::sqrt(std::max(0.0, 1.0 - x * x));
  double df = 1.0;
  for (int i = 1; i <= m; ++i) { pmm *= -df * sx; df += 2.0; }
  if (n == m) return pmm;
  double pm1 = x * (2.0 * m + 1.0) * pmm;
  if (n == m + 1) return pm1;
  double pn = 0;
  for (int k = m + 2; k <= n; ++k) {
    pn = ((2.0 * k - 1.0) * x * pm1 - (k + m - 1.0) * pmm) / (k - m);
    pmm = pm1; pm1 = pn;
  }
  return pn;
}
double factorial(int n) { double r = 1; for (int i = 2; i <= n; ++i) r *= i; return r; }
// real spherical harmonic (spherical_harmonics.hpp:96-125)
double Y(int n, int m, double th, double ph) {
  const double norm = std::sqrt((2.0 * n + 1.0) * factorial(n - std::abs(m)) / (2.0 * PI * factorial(n + std::abs(m))));
  if (m > 0) return norm * assoc_legendre(n, m, std::cos(th)) * std::cos(m * ph);
  if (m == 0) return norm * assoc_legendre(n, 0, std::cos(th)) / std::sqrt(2.0);
  return norm * assoc_legendre(n, -m, std::cos(th)) * std::sin(m * ph);
}
double dY_dtheta(int n, int m, double th, double ph) {
  if (n == 0) return 0.0;
  if (std::abs(m) < n) {
    double s1 = n * std::cos(th) * Y(n, m, th, ph);
    double s2 = std::sqrt(double(n * n - m * m) * (2.0 * n + 1.0) / (2.0 * n - 1.0)) * Y(n - 1, m, th, ph);
    return (s1 - s2) / std::sin(th);
  }
  return n * std::cos(th) * Y(n, m, th, ph) / std::sin(th);
}
double dY_dphi(int n, int m, double th, double ph) { return m == 0 ? 0.0 : m * Y(n, -m, th, ph); }

// Gauss-Legendre nodes/weights on [-1, 1] (Newton on P_N)
void gauss_legendre(int N, std::vector<double> &x, std::vector<double> &w) {
  x.resize(N); w.resize(N);
  for (int i = 0; i < N; ++i) {
    double z = std::cos(PI * (i + 0.75) / (N + 0.5)), pp = 0;
    for (int it = 0; it < 100; ++it) {
      double p1 = 1.0, p2 = 0.0;
      for (int j = 1; j <= N; ++j) { double p3 = p2; p2 = p1; p1 = ((2.0 * j - 1.0) * z * p2 - (j - 1.0) * p3) / j; }
      pp = N * (z * p1 - p2) / (z * z - 1.0);
      double z1 = z;
      z = z1 - p1 / pp;
      if (std::fabs(z - z1) < 1e-16) break;
    }
    x[i] = z;
    w[i] = 2.0 / ((1.0 - z * z) * pp * pp);
  }
}
}  // namespace

void coupling_quadrature(int L, double *out) {
  const int D = (L + 1) * (L + 1);
  std::fill(out, out + 6 * size_t(D) * D, 0.0);
  const int NT = 2 * L + 24, NP = 4 * L + 24;
  std::vector<double> gx, gw;
  gauss_legendre(NT, gx, gw);
  std::vector<double> th(NT), wt(NT);
  for (int i = 0; i < NT; ++i) { th[i] = PI * 0.5 * (gx[i] + 1.0); wt[i] = PI * 0.5 * gw[i]; }
  for (int l = 0; l <= L; ++l)
    for (int m = -l; m <= l; ++m) {
      const int row = l * l + l + m;
      for (int lp = 0; lp <= L; ++lp) {
        if (std::abs(l - lp) != 1) continue;
        for (int mp = -lp; mp <= lp; ++mp) {
          if (std::abs(std::abs(m) - std::abs(mp)) > 1) continue;
          const int col = lp * lp + lp + mp;
          double r[6] = {0, 0, 0, 0, 0, 0};
          for (int i = 0; i < NT; ++i) {
            const double t = th[i], st = std::sin(t), ctt = std::cos(t);
            double acc[6] = {0, 0, 0, 0, 0, 0};
            for (int j = 0; j < NP; ++j) {
              const double p = 2.0 * PI * j / NP, sp = std::sin(p), cp = std::cos(p);
              const double y = Y(l, m, t, p), y1 = Y(lp, mp, t, p);
              const double dt = dY_dtheta(l, m, t, p), dp = dY_dphi(l, m, t, p);
              acc[0] += y * st * cp * y1 * st;                 // vIntegrand_x
              acc[1] += y * st * sp * y1 * st;                 // vIntegrand_y
              acc[2] += y * ctt * y1 * st;                     // vIntegrand_z
              acc[3] += (dt * ctt * cp * st - dp * sp) * y1;   // GammaIntegrand_x
              acc[4] += (dt * ctt * sp * st + dp * cp) * y1;   // GammaIntegrand_y
              acc[5] += (dt * (-1.0) * st) * y1 * st;          // GammaIntegrand_z
            }
            for (int k = 0; k < 6; ++k) r[k] += wt[i] * acc[k] * (2.0 * PI / NP);
          }
          for (int k = 0; k < 6; ++k)
            if (std::fabs(r[k]) > 1e-8) out[size_t(k) * D * D + size_t(row) * D + col] += r[k];
        }
      }
    }
}

}  // namespace vshe

// she_oracle.cpp -- TEST INFRASTRUCTURE, not product code.
//
// A CPU restatement (FP64, single-threaded) of ViennaSHE's SHE linear-solve
// path, used only by tests/, __graft_entry__.smoke() and bench.py's CPU
// baseline as the checker.  Nothing in the product links, loads or calls it.
//
// Every function cites the reference file:line it restates (paths relative to
// the viennashe-dev project root).  The reference's matrix container
// (viennashe/math/linalg_util.hpp:68-196, a vector of std::map rows whose
// non-const operator() inserts on access) is kept as-is, because the sparsity
// pattern of the assembled, eliminated and normalised systems depends on it.
//
// The mesh (ViennaGrid) is replaced by the flat vshe_device_desc; the facet
// order and the (c1, c2) order of the cells on a facet are therefore whatever
// the description says (the generator documents its convention).
//
// ILU0, ILUT and BiCGStab are written from the published algorithms (Saad,
// "Iterative Methods for Sparse Linear Systems", 2nd ed., Alg. 10.4 and 10.6;
// van der Vorst 1992), because the reference takes them from ViennaCL, which
// is not part of the reference tree.
//
// Build: oracle/build.sh (g++ -O2 -ffp-contract=off, no FMA contraction, the
// arithmetic the reference gets from a default x86-64 build).

#include "../include/vshe_types.h"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <map>
#include <set>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

namespace vsheo {

// ---------------------------------------------------------------------------
// constants: viennashe/physics/constants.hpp:59-76, viennashe/math/constants.hpp:43
// ---------------------------------------------------------------------------
static const double PI = 3.1415926535897932384626433832795;
static const double Q = 1.602176565e-19;
static const double KB = 1.3806488e-23;
static const double HBAR = 6.62606896e-34 / (2.0 * 3.1415926535897932384626433832795);
static const double M0 = 9.10938291e-31;

// silicon, electrons: viennashe/materials/all.hpp:58-99
static double m_dos() { return 0.32 * M0; }
static double m_long() { return 0.98 * M0; }
static double m_trans() { return 0.19 * M0; }
static double m_cond() { return 3.0 / (1.0 / m_long() + 1.0 / m_trans() + 1.0 / m_trans()); }
static double band_gap() { return 1.11 * Q; }

// Modena dispersion, electrons: viennashe/physics/dispersion.hpp:207-286
static const double ALPHA = 0.5 / Q;
static double dos(double eps) {
  if (eps > 0.0) {
    const double mstar = m_dos();
    const double prefactor = mstar * std::sqrt(2.0 * mstar) / (8.0 * PI * PI * PI * HBAR * HBAR * HBAR);
    return prefactor * 4.0 * PI * (1.0 + 2.0 * ALPHA * eps) * std::sqrt(eps * (1.0 + ALPHA * eps));
  }
  return 0.0;
}
static double velocity(double eps) {
  if (eps < 0) return 0;
  double gamma = eps * (1.0 + ALPHA * eps);
  double dgam = 1.0 + 2.0 * ALPHA * eps;
  double mc = m_cond(), md = m_dos();
  return std::sqrt(mc / md) * std::sqrt(2.0 * gamma / m_dos()) / dgam;
}
static const double SYMMETRY = 6.0;

// viennashe/physics/physics.hpp:71-75
static double optical_phonon_number(double eps, double T) { return 1.0 / (std::exp(eps / (KB * T)) - 1.0); }
// viennashe/physics/physics.hpp:84-90, 105-116, 125-148, 158-170
static double band_weight(double T) {
  const double Ncv0 = 2.50933670314359713002e19 * 100 * 100 * 100;
  return Ncv0 * std::pow(0.33 * (T / 300.0), 1.5) * 6.0;
}
static double band_weight_h(double T) {
  const double Ncv0 = 2.50933670314359713002e19 * 100 * 100 * 100;
  return Ncv0 * std::pow(0.6 * (T / 300.0), 1.5) * 6.0;
}
static double built_in_potential(double T, double nd, double na) {
  if (nd <= 0 && na <= 0) return 0;
  const double net = nd - na;
  const double naux = band_weight(T) * std::exp(-1.0 * (band_gap() * 0.5) / (KB * T));
  const double paux = band_weight_h(T) * std::exp(1.0 * (-band_gap() * 0.5) / (KB * T));
  double x = std::sqrt(net * net + 4.0 * naux * paux);
  if (net >= 0.0) {
    x = (x + net) * 0.5 / naux;
    return T * std::log(x) * KB / Q;
  }
  x = (x - net) * 0.5 / paux;
  return -T * std::log(x) * KB / Q;
}
static double contact_carrier_ohm_n(double T, double nd, double na) {
  const double phiB = built_in_potential(T, nd, na);
  return band_weight(T) * std::exp(-1.0 * (band_gap() * 0.5 - Q * phiB) / (KB * T));
}

// ---------------------------------------------------------------------------
// matrix container: viennashe/math/linalg_util.hpp:68-196
// ---------------------------------------------------------------------------
typedef std::map<size_t, double> Row;
struct Mat {
  std::vector<Row> r;
  Mat() {}
  explicit Mat(size_t n) : r(n) {}
  size_t size() const { return r.size(); }
  double &at(size_t i, size_t j) { return r[i][j]; }  // non-const operator(): inserts
  double get(size_t i, size_t j) const {              // const operator(): no insert
    auto it = r[i].find(j);
    return it == r[i].end() ? 0.0 : it->second;
  }
  size_t nnz() const { size_t s = 0; for (auto &x : r) s += x.size(); return s; }
  Mat trans() const {  // linalg_util.hpp:139-149
    Mat t(r.size());
    for (size_t i = 0; i < r.size(); ++i)
      for (auto &e : r[i]) t.r[e.first][i] = e.second;
    return t;
  }
  // operator*(factor): linalg_util.hpp:151-161.  Note result(col, row) *= factor.
  Mat scaled_as_reference(double f) const {
    Mat res = *this;
    for (size_t i = 0; i < r.size(); ++i)
      for (auto &e : r[i]) res.r[e.first][i] *= f;
    return res;
  }
  // operator+=: linalg_util.hpp:163-172
  void add(const Mat &B) {
    for (size_t i = 0; i < B.size(); ++i)
      for (auto &e : B.r[i]) r[i][e.first] += e.second;
  }
};

// viennashe/math/spherical_harmonics.hpp:213-252
struct HarmIter {
  long L, l, m; bool odd; bool all;
  HarmIter(long Lmax, int type /*0 all, 1 even, 2 odd*/) : L(Lmax), l(type == 2 ? 1 : 0), m(type == 2 ? -1 : 0), odd(type == 2), all(type == 0) {}
  void next() {
    if (m < l) ++m;
    else { l += all ? 1 : 2; m = -l; }
  }
  bool valid() const { return l <= L; }
  long operator*() const { return l * l + m + l; }
};
enum { ITER_ALL = 0, ITER_EVEN = 1, ITER_ODD = 2 };

// viennashe/she/she_quantity.hpp:35-52
static long even_unknowns_on_node(long L) { long n = 0; for (long l = 0; l <= L; l += 2) n += 2 * l + 1; return n; }
static long odd_unknowns_on_node(long L) { long n = 0; for (long l = 1; l <= L; l += 2) n += 2 * l + 1; return n; }

// viennashe/util/block_matrix_writer.hpp:48-81
static void add_block_matrix(Mat &A, size_t row_index, size_t col_index, double prefactor, const Mat &C,
                             HarmIter row_iter, const HarmIter &col_iter_init, bool elastic_prev = false) {
  size_t row = row_index;
  for (; row_iter.valid(); row_iter.next(), ++row) {
    size_t col = col_index;
    for (HarmIter col_iter(col_iter_init); col_iter.valid(); col_iter.next(), ++col) {
      double entry = C.get(size_t(*row_iter), size_t(*col_iter));
      if (entry) {
        if (elastic_prev && row == row_index && col == col_index) continue;
        A.at(row, col) += prefactor * entry;
      }
    }
  }
}

// viennashe/she/assemble_common.hpp:302-319
static void write_boundary(std::vector<double> &rhs, size_t row_start, double prefactor, const Mat &C, HarmIter row_iter) {
  size_t row = row_start;
  for (; row_iter.valid(); row_iter.next()) {
    rhs[row] -= prefactor * C.get(size_t(*row_iter), 0);
    ++row;
  }
}

// ---------------------------------------------------------------------------
// problem state
// ---------------------------------------------------------------------------
struct Problem {
  // device
  int dim = 1, nc = 0, nf = 0;
  std::vector<int> mat, contact, fcell, cf_ptr, cf_idx;
  std::vector<double> vol, cen, nd, na, phi, fvol, fnorm;
  double T = 300.0;
  // config
  vshe_she_config cfg;
  int L = 1;
  Mat ax, ay, az, bx, by, bz;
  // SHE quantity (viennashe/she/she_quantity.hpp:58-266), array index = id * NH + H
  size_t NH = 0;
  std::vector<double> Hval, shift_c, shift_f, bnd_c;
  std::vector<long> idx_c, idx_f;
  std::vector<size_t> ord_c, ord_f;
  std::vector<char> mask_c;
  long n_even = 0, n_odd = 0;
  double hbar_omega = 0.0;
  // systems
  Mat A_full;                   // as assembled
  std::vector<double> b_full;
  Mat A_diag;                   // after diagonalise_odd2odd_coupling_matrix
  std::vector<double> b_diag;
  Mat A_red0; std::vector<double> b_red0;   // after elimination
  Mat A_red;  std::vector<double> b_red;    // after scaling + normalisation
  std::vector<double> scaling, scale_factors;
  std::vector<std::pair<size_t, size_t>> blocks;  // fill_block_indices
  std::string err;

  bool is_semi(int c) const { return mat[c] == VSHE_MATERIAL_SI; }
  bool is_metal(int c) const { return mat[c] == VSHE_MATERIAL_METAL; }
  int other_cell(int f, int c) const {  // viennashe/util/misc.hpp get_other_cell_of_facet
    int c1 = fcell[2 * f], c2 = fcell[2 * f + 1];
    if (c2 < 0) return -1;
    return c1 == c ? c2 : c1;
  }
  double ekin_c(size_t c, size_t H) const { return Hval[H] - shift_c[c]; }  // she_quantity.hpp:207-216 (electrons)
  double ekin_f(size_t f, size_t H) const { return Hval[H] - shift_f[f]; }
  double dist(int c1, int c2) const {
    double s = 0; for (int d = 0; d < dim; ++d) { double t = cen[c1 * dim + d] - cen[c2 * dim + d]; s += t * t; }
    return std::sqrt(s);
  }
};

// Element accessor abstraction (cell or facet) for the per-element helpers.
struct Elem { const Problem *p; bool facet; int id; };
static double EK(const Elem &e, size_t H) { return e.facet ? e.p->ekin_f(e.id, H) : e.p->ekin_c(e.id, H); }

// viennashe/she/assemble_common.hpp:412-427
static double box_height(const Elem &e, size_t H) {
  double h = 0;
  if (H > 0) h = std::fabs(EK(e, H) - EK(e, H - 1));
  if (H < e.p->NH - 1) h += std::fabs(EK(e, H + 1) - EK(e, H));
  return h / 2.0;
}
// viennashe/she/assemble_common.hpp:433-462
static double averaged_dos(const Elem &e, size_t H) {
  double Z = dos(EK(e, H)); double n = 1;
  if (H < e.p->NH - 1) { Z += dos((EK(e, H) + EK(e, H + 1)) / 2.0); ++n; }
  if (H > 0) { Z += dos((EK(e, H) + EK(e, H - 1)) / 2.0); ++n; }
  return Z / n;
}
// viennashe/she/assemble_common.hpp:521-551
static double integral_vZ(const Elem &e, size_t H) {
  double kc = EK(e, H);
  double vZ = velocity(kc) * dos(kc); double n = 1;
  if (H < e.p->NH - 1) { double k = (EK(e, H) + EK(e, H + 1)) / 2.0; vZ += velocity(k) * dos(k); ++n; }
  if (H > 0) { double k = (EK(e, H) + EK(e, H - 1)) / 2.0; vZ += velocity(k) * dos(k); ++n; }
  vZ /= n;
  return vZ * box_height(e, H);
}
// viennashe/she/assemble_common.hpp:153-164
static double integral_Z_over_hk(double em, double ep) {
  if (ep < em) throw std::runtime_error("negative integration interval in integral_Z_over_hk");
  return 0.5 * (dos(ep) * velocity(ep) - dos(em) * velocity(em));
}
// viennashe/she/assemble_common.hpp:325-355 (including the "c1 + c2 / 2.0" precedence at H == 0)
static double lower_kinetic_energy_at_facet(const Problem &p, int f, size_t H) {
  int c1 = p.fcell[2 * f], c2 = p.fcell[2 * f + 1];
  if (c2 < 0) return p.ekin_c(c1, H);
  if (H == 0) return p.ekin_c(c1, H) + p.ekin_c(c2, H) / 2.0;
  return (p.ekin_c(c1, H - 1) + p.ekin_c(c2, H - 1) + p.ekin_c(c1, H) + p.ekin_c(c2, H)) / 4.0;
}
// viennashe/she/assemble_common.hpp:358-388
static double upper_kinetic_energy_at_facet(const Problem &p, int f, size_t H) {
  int c1 = p.fcell[2 * f], c2 = p.fcell[2 * f + 1];
  if (c2 < 0) return p.ekin_c(c1, H);
  if (H == p.NH - 1) return p.ekin_c(c1, H) + p.ekin_c(c2, H) / 2.0;
  return (p.ekin_c(c1, H + 1) + p.ekin_c(c2, H + 1) + p.ekin_c(c1, H) + p.ekin_c(c2, H)) / 4.0;
}

// viennashe/she/assemble_common.hpp:177-290 (1D, 2D) with the reference's operator* (Mat::scaled_as_reference)
static Mat coupling_matrix_in_direction(const Problem &p, const Mat &m1, const Mat &m2, int c1, int c2) {
  double pt[2] = {0, 0};
  for (int d = 0; d < p.dim; ++d) pt[d] = p.cen[c2 * p.dim + d] - p.cen[c1 * p.dim + d];
  double nrm = 0; for (int d = 0; d < p.dim; ++d) nrm += pt[d] * pt[d];
  nrm = std::sqrt(nrm);
  for (int d = 0; d < p.dim; ++d) pt[d] /= nrm;
  if (p.dim == 1 && !pt[0]) throw std::runtime_error("Equal vertices encountered!");
  if (p.dim == 2 && !pt[0] && !pt[1]) throw std::runtime_error("Equal vertices encountered!");
  double mt = m_trans(), md = m_dos();
  Mat res = m1.scaled_as_reference(pt[0] * std::sqrt(md / mt));
  if (p.dim == 2) res.add(m2.scaled_as_reference(pt[1] * std::sqrt(md / mt)));
  return res;
}

// ---------------------------------------------------------------------------
// a1: viennashe/she/setup_energies.hpp:61-153 (electrons, H-transformation on)
// ---------------------------------------------------------------------------
static void setup_energies(Problem &p) {
  double maxp = -1.0 * std::numeric_limits<double>::max();
  double minp = std::numeric_limits<double>::max();
  for (int c = 0; c < p.nc; ++c) {
    if (!p.is_semi(c)) continue;
    double v = p.phi[c] + 0.0;  // quantum correction is zero
    if (v < minp) minp = v;
    if (v > maxp) maxp = v;
  }
  double dE = p.cfg.energy_spacing;
  double range = Q * (maxp - minp) + 2.0 * dE + p.cfg.min_kinetic_energy_range;
  double bandedge = -Q * maxp - dE + band_gap() / 2.0;
  double incr = 1.0 * dE;
  p.NH = size_t(range / dE) + 1;
  p.Hval.resize(p.NH);
  for (size_t h = 0; h < p.NH; ++h) p.Hval[h] = bandedge + h * incr;
  p.shift_c.resize(p.nc); p.shift_f.resize(p.nf);
  for (int c = 0; c < p.nc; ++c) p.shift_c[c] = -Q * p.phi[c] + band_gap() / 2.0;
  for (int f = 0; f < p.nf; ++f) {
    int c1 = p.fcell[2 * f], c2 = p.fcell[2 * f + 1];
    if (c2 >= 0) p.shift_f[f] = (p.shift_c[c1] + p.shift_c[c2]) / 2.0;
    else p.shift_f[f] = p.shift_c[c1];
  }
}

// ---------------------------------------------------------------------------
// a2: viennashe/she/expansion_order.hpp:60-129 (lowering), 140-199 (smoothing),
//     262-333 (uniform orders, non-adaptive), 349-364 (driver)
// ---------------------------------------------------------------------------
static void distribute_expansion_orders(Problem &p) {
  size_t NH = p.NH;
  p.ord_c.assign(size_t(p.nc) * NH, size_t(p.L));
  p.ord_f.assign(size_t(p.nf) * NH, size_t(p.L));
  // lower_expansion_order_near_bandedge
  for (int c = 0; c < p.nc; ++c) {
    for (size_t H = 1; H < NH - 1; ++H) {
      if (p.ekin_c(c, H) <= 0) { p.ord_c[c * NH + H] = 1; continue; }
      bool all_pos = true;
      for (int k = p.cf_ptr[c]; k < p.cf_ptr[c + 1]; ++k) {
        int o = p.other_cell(p.cf_idx[k], c);
        if (o < 0) continue;
        if (p.ekin_c(o, H - 1) <= 0) all_pos = false;
      }
      if (all_pos) break;
      p.ord_c[c * NH + H] = 1;
      for (int k = p.cf_ptr[c]; k < p.cf_ptr[c + 1]; ++k) {
        int o = p.other_cell(p.cf_idx[k], c);
        if (o < 0) continue;
        p.ord_c[o * NH + H] = 1;
      }
    }
  }
  // smooth_expansion_order (the second test compares c2 with itself, as in the reference)
  for (long i = 0; i < 10; ++i) {
    bool changed = false;
    for (int f = 0; f < p.nf; ++f) {
      int c1 = p.fcell[2 * f], c2 = p.fcell[2 * f + 1];
      if (c2 < 0) continue;
      for (size_t H = 0; H < NH; ++H) {
        if (p.ord_c[c1 * NH + H] > p.ord_c[c2 * NH + H] + 2) { changed = true; p.ord_c[c1 * NH + H] = p.ord_c[c2 * NH + H] + 2; }
        if (p.ord_c[c2 * NH + H] > p.ord_c[c2 * NH + H] + 2) { changed = true; p.ord_c[c2 * NH + H] = p.ord_c[c2 * NH + H] + 2; }
      }
    }
    if (!changed) break;
  }
}

// ---------------------------------------------------------------------------
// a4: viennashe/she/boundary_conditions.hpp:57-134 with
//     viennashe/accessors.hpp:316-367 (contact density) and :51-81 (neighbour dopings)
// ---------------------------------------------------------------------------
static double contact_density(const Problem &p, int c) {
  double nd = p.nd[c], na = p.na[c];
  if (p.is_metal(c)) {
    double dn = 1, dp = 1; long N = 0;
    for (int k = p.cf_ptr[c]; k < p.cf_ptr[c + 1]; ++k) {
      int o = p.other_cell(p.cf_idx[k], c);
      if (o < 0) continue;
      if (p.is_semi(o)) { dn *= p.nd[o]; dp *= p.na[o]; N += 1; }
    }
    if (N > 1) dn = std::pow(dn, 1.0 / N);
    if (N > 1) dp = std::pow(dp, 1.0 / N);
    nd = dn; na = dp;
  }
  return contact_carrier_ohm_n(p.T, nd, na);
}
static void write_boundary_conditions(Problem &p) {
  size_t NH = p.NH;
  p.bnd_c.assign(size_t(p.nc) * NH, 0.0);
  for (int c = 0; c < p.nc; ++c) {
    Elem e{&p, false, c};
    double T = p.T;
    double corr = 0;
    for (size_t H = 1; H < NH - 1; ++H) {
      double em = p.ekin_c(c, H);
      double lo = std::max<double>((p.ekin_c(c, H - 1) + em) / 2.0, 0.0);
      double up = (p.ekin_c(c, H + 1) + em) / 2.0;
      if (lo < up && up >= 0) corr += std::exp(-em / (KB * T)) * averaged_dos(e, H) * box_height(e, H);
    }
    corr *= SYMMETRY;
    for (size_t H = 1; H < NH - 1; ++H) {
      double en = p.ekin_c(c, H);
      double lo = std::max<double>((p.ekin_c(c, H - 1) + en) / 2.0, 0.0);
      double up = (p.ekin_c(c, H + 1) + en) / 2.0;
      double v = 0.0;
      if (lo < up && up >= 0) v = contact_density(p, c) * std::exp(-en / (KB * T)) / corr;
      p.bnd_c[c * NH + H] = v;
    }
  }
}

// ---------------------------------------------------------------------------
// a3: viennashe/simulator.hpp:94-120 (SHE mask), viennashe/mapping.hpp:97-189, 204-323
// ---------------------------------------------------------------------------
static void create_mapping(Problem &p) {
  size_t NH = p.NH;
  p.mask_c.assign(p.nc, 0);
  for (int c = 0; c < p.nc; ++c) {
    if (p.is_semi(c)) p.mask_c[c] = 1;
    else if (p.is_metal(c)) {
      for (int k = p.cf_ptr[c]; k < p.cf_ptr[c + 1]; ++k) {
        int o = p.other_cell(p.cf_idx[k], c);
        if (o >= 0 && p.is_semi(o)) { p.mask_c[c] = 1; break; }
      }
    }
  }
  const double kmax = p.cfg.max_kinetic_energy_range;
  p.idx_c.assign(size_t(p.nc) * NH, -1);
  p.idx_f.assign(size_t(p.nf) * NH, -1);
  long idx = 0;
  for (size_t H = 0; H < NH; ++H) {
    for (int c = 0; c < p.nc; ++c) {
      if (!p.mask_c[c]) { p.idx_c[c * NH + H] = -1; continue; }
      if (H == 0 || H == NH - 1) { p.idx_c[c * NH + H] = -1; continue; }
      Elem e{&p, false, c};
      if (averaged_dos(e, H) > 0 && p.ekin_c(c, H) < kmax) {
        p.idx_c[c * NH + H] = idx;
        idx += even_unknowns_on_node(long(p.ord_c[c * NH + H]));
      } else {
        p.idx_c[c * NH + H] = -1;
        p.ord_c[c * NH + H] = 0;
      }
    }
  }
  p.n_even = idx;
  for (size_t H = 0; H < NH; ++H) {
    for (int f = 0; f < p.nf; ++f) {
      int c1 = p.fcell[2 * f], c2 = p.fcell[2 * f + 1];
      if (c2 < 0) { p.idx_f[f * NH + H] = -1; p.ord_f[f * NH + H] = 0; continue; }
      long d1 = p.idx_c[c1 * NH + H], d2 = p.idx_c[c2 * NH + H];
      Elem e{&p, true, f};
      if (d1 > -1 && d2 > -1 && averaged_dos(e, H) > 0 && (p.is_semi(c1) || p.is_semi(c2))) {
        p.idx_f[f * NH + H] = idx;
        idx += odd_unknowns_on_node(long(p.ord_f[f * NH + H]));
      } else {
        p.idx_f[f * NH + H] = -1;
        p.ord_f[f * NH + H] = 0;
      }
    }
  }
  p.n_odd = idx - p.n_even;
}

// ---------------------------------------------------------------------------
// scattering: viennashe/she/scattering/acoustic_phonon_scattering.hpp:83-114,
// optical_phonon_scattering.hpp:66-81 (snap), 122-179; config.hpp:50-112
// ---------------------------------------------------------------------------
struct Event { double ei, ef, rate, gen; };
static double acoustic_rate(const Problem &p) {
  const double ul = 9040.0, rho = 2330.0, E1 = 8.9 * Q;
  const double r = 2.0 * PI * KB * p.T * E1 * E1 / (HBAR * ul * ul * rho);
  return p.cfg.acoustic_fit_factor * r;
}
static double optical_rate(const Problem &p) {
  const double rho = 2330.0, DtK = 5e10 * Q;
  const double r = PI * DtK * DtK * HBAR / (2.0 * rho * p.hbar_omega);
  return p.cfg.optical_fit_factor * r;
}
static void snap_phonon_energy(Problem &p) {
  double w = 1.24 * (Q / 20.0);
  double sp = p.cfg.energy_spacing;
  if (sp > 0) {
    size_t steps = size_t(w / sp);
    double e0 = w - steps * sp;
    double e1 = (steps + 1.0) * sp - w;
    if (e1 < e0) ++steps;
    w = steps * sp;
  }
  p.hbar_omega = w;
}

// viennashe/she/assemble_scattering.hpp:65-105
static long energy_index_H(const Elem &e, long hint, double kin) {
  long res = hint;
  if (kin < EK(e, size_t(res)) || kin > EK(e, size_t(res))) {
    long inc = 1;
    double diff = kin - EK(e, size_t(res));
    double diff0 = diff;
    if (diff < 0) inc = -1;
    while (res < long(e.p->NH - 1) && res > 0 && diff * diff0 > 0) {
      res += inc;
      diff = kin - EK(e, size_t(res));
    }
    if (diff * diff0 > 0) return -1;
    double e1 = std::abs(diff), e2 = e1;
    if (res - inc >= 0 && res - inc < long(e.p->NH)) e2 = std::abs(kin - EK(e, size_t(res - inc)));
    if (e2 < e1) return res - inc;
  }
  return res;
}

// viennashe/she/assemble_scattering.hpp:116-335 (DF discretisation)
static void assemble_scattering(Problem &p, const Elem &e, size_t H, const Mat &sin, const Mat &sout) {
  const long row = e.facet ? p.idx_f[e.id * p.NH + H] : p.idx_c[e.id * p.NH + H];
  if (row < 0) return;
  double kin = EK(e, H);
  const long ord = long(e.facet ? p.ord_f[e.id * p.NH + H] : p.ord_c[e.id * p.NH + H]);
  bool odd = e.facet;
  double V = e.facet ? p.fvol[e.id] : p.vol[e.id];
  if (odd) {
    int c1 = p.fcell[2 * e.id], c2 = p.fcell[2 * e.id + 1];
    V *= p.dist(c1, c2) / double(p.dim);
  }
  std::vector<std::vector<Event>> procs;
  if (p.cfg.acoustic_phonon) procs.push_back({Event{kin, kin, acoustic_rate(p), 0}});
  if (p.cfg.optical_phonon) {
    double N = optical_phonon_number(p.hbar_omega, p.T);
    double r = optical_rate(p);
    double w = p.hbar_omega;
    procs.push_back({Event{kin, kin - w, r * (N + 1.0), 0}, Event{kin + w, kin, r * (N + 1.0), 0},
                     Event{kin, kin + w, r * N, 0}, Event{kin - w, kin, r * N, 0}});
  }
  const int it = odd ? ITER_ODD : ITER_EVEN;
  for (auto &ev : procs) {
    for (auto &s : ev) {
      if (s.rate <= 0 && s.gen <= 0) continue;
      long iHi = energy_index_H(e, long(H), s.ei);
      long iHf = energy_index_H(e, long(H), s.ef);
      if (iHi == -1 || iHf == -1) continue;
      const double Zi = averaged_dos(e, size_t(iHi));
      const double Zf = averaged_dos(e, size_t(iHf));
      const double h = std::min(box_height(e, size_t(iHi)), box_height(e, size_t(iHf)));
      const bool elastic = (iHi == iHf) && !odd;
      if (s.ei <= kin && s.ei >= kin) {
        long col = e.facet ? p.idx_f[e.id * p.NH + iHf] : p.idx_c[e.id * p.NH + iHf];
        if (col >= 0) {
          double coef = 2.0 * PI * s.rate * Zi * Zf * V * h;
          add_block_matrix(p.A_full, size_t(row), size_t(row), coef, sout, HarmIter(ord, it), HarmIter(ord, it), elastic);
        }
      }
      if (s.ef <= kin && s.ef >= kin) {
        long col = e.facet ? p.idx_f[e.id * p.NH + iHi] : p.idx_c[e.id * p.NH + iHi];
        if (col >= 0) {
          double coef = -2.0 * PI * s.rate * Zi * Zf * V * h - s.gen * Zi * V * h;
          add_block_matrix(p.A_full, size_t(row), size_t(col), coef, sin, HarmIter(ord, it), HarmIter(ord, it), elastic);
        }
      }
    }
  }
}

// viennashe/she/assemble_boundary.hpp:69-183 (DF discretisation)
static void assemble_boundary(Problem &p, int c, size_t H, const Mat &ident) {
  long row = p.idx_c[c * p.NH + H];
  if (row < 0) return;
  long ord = long(p.ord_c[c * p.NH + H]);
  if (p.contact[c] < 0) return;  // device.has_contact_potential(cell)
  Elem e{&p, false, c};
  if (p.cfg.boundary_type == VSHE_BOUNDARY_DIRICHLET) {
    double bnd = p.bnd_c[c * p.NH + H];
    double height = box_height(e, H);
    double coef = height * averaged_dos(e, H);
    add_block_matrix(p.A_full, size_t(row), size_t(row), coef, ident, HarmIter(ord, ITER_EVEN), HarmIter(ord, ITER_EVEN));
    write_boundary(p.b_full, size_t(row), -bnd * coef, ident, HarmIter(1, ITER_EVEN));
    return;
  }
  double tau = p.cfg.gr_tau;
  double height = box_height(e, H);
  double bnd = p.bnd_c[c * p.NH + H];
  double V = p.vol[c];
  double coef = V * height / tau * averaged_dos(e, H);
  add_block_matrix(p.A_full, size_t(row), size_t(row), coef, ident, HarmIter(ord, ITER_EVEN), HarmIter(ord, ITER_EVEN));
  write_boundary(p.b_full, size_t(row), -bnd * coef, ident, HarmIter(1, ITER_EVEN));
}

// viennashe/she/assemble_streaming.hpp:73-365 (DF discretisation)
static void assemble_streaming(Problem &p, int cell, int facet, size_t H, const Mat &Cd, const Mat &Cb, bool odd) {
  int other = p.other_cell(facet, cell);
  if (other < 0) return;
  long row = odd ? p.idx_f[facet * p.NH + H] : p.idx_c[cell * p.NH + H];
  if (row < 0) return;
  long col = odd ? p.idx_c[cell * p.NH + H] : p.idx_f[facet * p.NH + H];
  if (col < 0) return;
  double conn[2] = {0, 0};
  for (int d = 0; d < p.dim; ++d) conn[d] = p.cen[cell * p.dim + d] - p.cen[other * p.dim + d];
  double len = 0; for (int d = 0; d < p.dim; ++d) len += conn[d] * conn[d];
  len = std::sqrt(len);
  double dot = 0;
  // outer unit normal of `cell` at `facet`: the stored normal points c1 -> c2
  double sgn = (p.fcell[2 * facet] == cell) ? 1.0 : -1.0;
  for (int d = 0; d < p.dim; ++d) dot += sgn * p.fnorm[facet * p.dim + d] * (conn[d] / len);
  const double warea = p.fvol[facet] * std::fabs(dot);
  long ord_row = long(odd ? p.ord_f[facet * p.NH + H] : p.ord_c[cell * p.NH + H]);
  long ord_col = long(odd ? p.ord_c[cell * p.NH + H] : p.ord_f[facet * p.NH + H]);
  double lo = lower_kinetic_energy_at_facet(p, facet, H);
  double up = upper_kinetic_energy_at_facet(p, facet, H);
  int itr = odd ? ITER_ODD : ITER_EVEN, itc = odd ? ITER_EVEN : ITER_ODD;
  Elem fe{&p, true, facet};
  double cd = integral_vZ(fe, H) * warea;
  add_block_matrix(p.A_full, size_t(row), size_t(col), cd, Cd, HarmIter(ord_row, itr), HarmIter(ord_col, itc));
  double izhk = integral_Z_over_hk(lo, up);
  double force = (p.ekin_c(cell, H) - p.ekin_c(other, H)) / p.dist(other, cell);  // force_on_facet_accessor(other, cell)
  double cdr = izhk * force * warea * len / 2.0;
  add_block_matrix(p.A_full, size_t(row), size_t(col), cdr, Cb, HarmIter(ord_row, itr), HarmIter(ord_col, itc));
}

// viennashe/she/assemble_all.hpp:46-424 (steady state, phonon scattering only)
static void assemble(Problem &p) {
  size_t N = size_t(p.n_even + p.n_odd);
  p.A_full = Mat(N);
  p.b_full.assign(N, 0.0);
  size_t D = size_t((p.L + 1) * (p.L + 1));
  Mat sin(D), sout(D), ident(D);
  for (size_t i = 0; i < D; ++i) sout.at(i, i) += 1.0;
  sin.at(0, 0) += 1.0;
  for (size_t i = 0; i < D; ++i)
    for (size_t j = 0; j < D; ++j) ident.at(i, j) = (i == j) ? 1.0 : 0.0;
  Mat axT = p.ax.trans(), ayT = p.ay.trans(), bxT = p.bx.trans(), byT = p.by.trans();
  for (int c = 0; c < p.nc; ++c) {
    for (size_t H = 0; H < p.NH; ++H) {
      assemble_boundary(p, c, H, ident);
      if (p.is_metal(c)) continue;
      assemble_scattering(p, Elem{&p, false, c}, H, sin, sout);
    }
    for (int k = p.cf_ptr[c]; k < p.cf_ptr[c + 1]; ++k) {
      int f = p.cf_idx[k];
      int o = p.other_cell(f, c);
      if (o < 0) continue;
      Mat Cd = coupling_matrix_in_direction(p, p.ax, p.ay, c, o);
      Mat Cb = coupling_matrix_in_direction(p, p.bx, p.by, o, c);
      for (size_t H = 0; H < p.NH; ++H) assemble_streaming(p, c, f, H, Cd, Cb, false);
    }
  }
  for (int f = 0; f < p.nf; ++f) {
    for (size_t H = 0; H < p.NH; ++H) assemble_scattering(p, Elem{&p, true, f}, H, sin, sout);
    int cs[2] = {p.fcell[2 * f], p.fcell[2 * f + 1]};
    for (int j = 0; j < 2; ++j) {
      int c = cs[j];
      if (c < 0) continue;
      int o = p.other_cell(f, c);
      if (o < 0) continue;
      Mat Cd = coupling_matrix_in_direction(p, axT, ayT, o, c);
      Mat Cb = coupling_matrix_in_direction(p, bxT, byT, o, c);
      for (size_t H = 0; H < p.NH; ++H) assemble_streaming(p, c, f, H, Cd, Cb, true);
    }
  }
}

// ---------------------------------------------------------------------------
// a10: viennashe/she/eliminate.hpp:40-68 (combine_lines), 80-214
// ---------------------------------------------------------------------------
static void combine_lines(Mat &A, std::vector<double> &rhs, size_t line1, size_t line_to_add, size_t col0) {
  const double s = A.at(line1, col0) / A.at(line_to_add, line_to_add);
  if (!s) return;
  Row &add = A.r[line_to_add];
  rhs[line1] = rhs[line1] - rhs[line_to_add] * s;
  for (auto &e : add) {
    if (!e.second) continue;
    A.at(line1, e.first) -= e.second * s;
  }
  A.r[line1].erase(col0);
}
static void erase_zeros_from(Mat &A, size_t first) {
  for (size_t i = first; i < A.size(); ++i)
    for (auto it = A.r[i].begin(); it != A.r[i].end();) {
      if (!it->second) it = A.r[i].erase(it);
      else ++it;
    }
}
static void diagonalise_odd2odd(Mat &A, std::vector<double> &rhs, size_t ne) {
  const size_t N = rhs.size();
  for (size_t i = ne + 1; i < N; ++i) {
    for (auto it = A.r[i].begin(); it != A.r[i].end(); ++it) {
      size_t c = it->first;
      if (c >= i) break;
      if (c < ne) continue;
      combine_lines(A, rhs, i, c, c);
      break;
    }
  }
  if (ne >= 1) erase_zeros_from(A, ne - 1);
  for (size_t i = N - 1; N > 0 && i >= ne; --i) {
    for (auto it = A.r[i].begin(); it != A.r[i].end(); ++it) {
      size_t c = it->first;
      if (c < i && c >= ne) throw std::runtime_error("values left of the S^oo diagonal");
      if (c < ne) continue;
      if (c == i) continue;
      combine_lines(A, rhs, i, c, c);
      break;
    }
    if (i == 0) break;
  }
  if (ne >= 1) erase_zeros_from(A, ne - 1);
}

// a11: viennashe/she/eliminate.hpp:226-293
static void eliminate_odd(Mat &A, const std::vector<double> &rhs, Mat &C, std::vector<double> &crhs) {
  size_t ne = C.size();
  for (size_t i = 0; i < ne; ++i) {
    crhs[i] = rhs[i];
    for (auto &e : A.r[i]) {
      if (e.first < ne) { C.at(i, e.first) += e.second; continue; }
      double d = -1.0;
      Row &orow = A.r[e.first];
      for (auto &o : orow) if (e.first == o.first) { d = o.second; break; }
      if (d <= 0.0) throw std::runtime_error("eliminate_odd_unknowns(): Diagonal entry not positive or not existing!");
      for (auto &o : orow)
        if (o.first < ne) C.at(i, o.first) -= e.second * o.second / d;
      crhs[i] -= e.second * rhs[e.first] / d;
    }
  }
}

// a18: viennashe/she/eliminate.hpp:305-354
static std::vector<double> recover_odd(const Mat &A, const std::vector<double> &rhs, const std::vector<double> &xe) {
  std::vector<double> x(rhs.size());
  size_t ne = xe.size();
  for (size_t i = 0; i < A.size(); ++i) {
    if (i < ne) { x[i] = xe[i]; continue; }
    double d = 0.0;
    x[i] = rhs[i];
    for (auto &e : A.r[i]) {
      if (e.first < ne) x[i] -= e.second * x[e.first];
      else if (i == e.first) d = e.second;
    }
    x[i] /= d;
  }
  return x;
}

// a12: viennashe/she/rescaling.hpp:50-107
static void setup_scaling(Problem &p) {
  p.scaling.assign(size_t(p.n_even), 1.0);
  for (int c = 0; c < p.nc; ++c) {
    for (size_t H = 0; H < p.NH; ++H) {
      long base = p.idx_c[c * p.NH + H];
      if (base < 0) continue;
      long num = even_unknowns_on_node(long(p.ord_c[c * p.NH + H]));
      for (long i = 0; i < num; ++i) {
        if (p.cfg.scaling_type == VSHE_SCALING_KINETIC_ENERGY)
          p.scaling[size_t(base + i)] = std::exp(-p.ekin_c(c, H) / (KB * p.T));
        else
          p.scaling[size_t(base + i)] = std::exp(-p.Hval[H] / (KB * p.T));
      }
    }
  }
}
static void rescale(Mat &A, const std::vector<double> &s) {
  for (auto &row : A.r)
    for (auto &e : row) e.second *= s[e.first];
}

// a13: viennashe/math/linalg_util.hpp:202-282 (the non-const diagonal access inserts (i,i))
static std::vector<double> row_normalize(Mat &A, std::vector<double> &rhs) {
  std::vector<double> sf(rhs.size(), 1.0);
  Mat Ac = A.trans();
  for (size_t i = 0; i < Ac.size(); ++i) {
    Row &col = Ac.r[i];
    double nrm = 0.0;
    for (auto &e : col) nrm += std::log(std::fabs(e.second));
    nrm = std::exp(nrm / double(col.size()));
    if (Ac.at(i, i) < 0.0) nrm *= -1.0;
    for (auto &e : col) e.second /= nrm;
    sf[i] /= nrm;
  }
  A = Ac.trans();
  for (size_t i = 0; i < A.size(); ++i) {
    Row &row = A.r[i];
    double nrm = 0.0;
    for (auto &e : row) nrm += e.second * e.second;
    nrm = std::sqrt(nrm);
    if (A.at(i, i) < 0.0) nrm *= -1.0;
    for (auto &e : row) e.second /= nrm;
    rhs[i] /= nrm;
  }
  return sf;
}

// a14: viennashe/she/linear_solver.hpp:44-83
static void fill_block_indices(Problem &p) {
  p.blocks.assign(p.NH, {0, 0});
  size_t last = 0;
  for (size_t H = 0; H < p.blocks.size(); ++H) {
    p.blocks[H].first = last;
    for (int c = 0; c < p.nc; ++c) {
      if (p.idx_c[c * p.NH + H] > -1) {
        last = size_t(p.idx_c[c * p.NH + H]);
        p.blocks[H].first = last;
        if (H > 0) p.blocks[H - 1].second = last;
        break;
      }
    }
    if (p.blocks[H].second < p.blocks[H].first) p.blocks[H].second = p.blocks[H].first;
  }
  p.blocks.back().second = size_t(p.n_even);
}

// ---------------------------------------------------------------------------
// CSR helpers and solvers (published algorithms)
// ---------------------------------------------------------------------------
struct CSR { int64_t n = 0; std::vector<int64_t> rp; std::vector<int32_t> ci; std::vector<double> v; };

static CSR to_csr(const Mat &A) {  // src/solvers/viennacl/serial_linear_solver.hpp:52-89 (map order = ascending columns)
  CSR c; c.n = int64_t(A.size()); c.rp.resize(A.size() + 1);
  size_t k = 0;
  for (size_t i = 0; i < A.size(); ++i) {
    c.rp[i] = int64_t(k);
    for (auto &e : A.r[i]) { c.ci.push_back(int32_t(e.first)); c.v.push_back(e.second); ++k; }
  }
  c.rp[A.size()] = int64_t(k);
  return c;
}

static void spmv(int64_t n, const int64_t *rp, const int32_t *ci, const double *v, const double *x, double *y) {
  for (int64_t i = 0; i < n; ++i) {
    double s = 0.0;
    for (int64_t k = rp[i]; k < rp[i + 1]; ++k) s += v[k] * x[ci[k]];
    y[i] = s;
  }
}
static double dot(const std::vector<double> &a, const std::vector<double> &b) {
  double s = 0; for (size_t i = 0; i < a.size(); ++i) s += a[i] * b[i]; return s;
}
static double nrm2(const std::vector<double> &a) { return std::sqrt(dot(a, a)); }

// Incomplete factorisation in CSR form: L (unit, strictly lower) and U (with diagonal).
struct ILU {
  int64_t n = 0;
  std::vector<int64_t> lrp, urp; std::vector<int32_t> lci, uci; std::vector<double> lv, uv;
  void apply(const double *b, double *x) const {  // solve L U x = b
    for (int64_t i = 0; i < n; ++i) {
      double s = b[i];
      for (int64_t k = lrp[i]; k < lrp[i + 1]; ++k) s -= lv[k] * x[lci[k]];
      x[i] = s;
    }
    for (int64_t i = n - 1; i >= 0; --i) {
      double s = x[i];
      int64_t k0 = urp[i];  // first entry is the diagonal
      for (int64_t k = k0 + 1; k < urp[i + 1]; ++k) s -= uv[k] * x[uci[k]];
      x[i] = s / uv[k0];
    }
  }
};

// block id of a row for the block-ILU variants (blocks given as [ptr[b], ptr[b+1]))
static std::vector<int32_t> row_blocks(int64_t n, int64_t nb, const int64_t *bptr) {
  std::vector<int32_t> b(size_t(n), 0);
  if (nb <= 0 || !bptr) return b;
  for (int64_t k = 0; k < nb; ++k)
    for (int64_t i = bptr[k]; i < bptr[k + 1]; ++i) b[size_t(i)] = int32_t(k);
  return b;
}

// ILU(0), Saad Alg. 10.4 (IKJ), restricted to within-block entries when blocks are given.
// Returns the factor values in the pattern of A (entries coupling different blocks are left 0).
static void ilu0_values(int64_t n, const int64_t *rp, const int32_t *ci, const double *v,
                        const std::vector<int32_t> &blk, std::vector<double> &lu, std::vector<int64_t> &diag) {
  lu.assign(v, v + rp[n]);
  diag.assign(size_t(n), -1);
  for (int64_t i = 0; i < n; ++i)
    for (int64_t k = rp[i]; k < rp[i + 1]; ++k) {
      if (blk[size_t(ci[k])] != blk[size_t(i)]) lu[size_t(k)] = 0.0;
      if (ci[k] == i) diag[size_t(i)] = k;
    }
  std::vector<int64_t> pos(size_t(n), -1);
  for (int64_t i = 0; i < n; ++i) {
    if (diag[size_t(i)] < 0) throw std::runtime_error("ILU0: missing diagonal");
    for (int64_t k = rp[i]; k < rp[i + 1]; ++k) pos[size_t(ci[k])] = k;
    for (int64_t k = rp[i]; k < rp[i + 1]; ++k) {
      int64_t c = ci[k];
      if (c >= i) break;
      if (blk[size_t(c)] != blk[size_t(i)]) continue;
      double piv = lu[size_t(diag[size_t(c)])];
      lu[size_t(k)] /= piv;
      double lik = lu[size_t(k)];
      for (int64_t kk = diag[size_t(c)] + 1; kk < rp[c + 1]; ++kk) {
        int64_t j = ci[kk];
        if (blk[size_t(j)] != blk[size_t(i)]) continue;
        int64_t pj = pos[size_t(j)];
        if (pj >= 0) lu[size_t(pj)] -= lik * lu[size_t(kk)];
      }
    }
    for (int64_t k = rp[i]; k < rp[i + 1]; ++k) pos[size_t(ci[k])] = -1;
  }
}

static ILU ilu0(int64_t n, const int64_t *rp, const int32_t *ci, const double *v, int64_t nb, const int64_t *bptr) {
  std::vector<int32_t> blk = row_blocks(n, nb, bptr);
  std::vector<double> lu; std::vector<int64_t> diag;
  ilu0_values(n, rp, ci, v, blk, lu, diag);
  ILU f; f.n = n; f.lrp.assign(1, 0); f.urp.assign(1, 0);
  for (int64_t i = 0; i < n; ++i) {
    for (int64_t k = rp[i]; k < rp[i + 1]; ++k) {
      int64_t j = ci[k];
      if (blk[size_t(j)] != blk[size_t(i)]) continue;
      if (j < i) { f.lci.push_back(int32_t(j)); f.lv.push_back(lu[size_t(k)]); }
    }
    f.uci.push_back(int32_t(i)); f.uv.push_back(lu[size_t(diag[size_t(i)])]);
    for (int64_t k = rp[i]; k < rp[i + 1]; ++k) {
      int64_t j = ci[k];
      if (blk[size_t(j)] != blk[size_t(i)]) continue;
      if (j > i) { f.uci.push_back(int32_t(j)); f.uv.push_back(lu[size_t(k)]); }
    }
    f.lrp.push_back(int64_t(f.lci.size())); f.urp.push_back(int64_t(f.uci.size()));
  }
  return f;
}

// ILU(k) by levels of fill (Saad, Alg. 10.5): the symbolic phase gives every entry of row i a
// level, 0 for A's entries and lev(i,k) + lev(k,j) + 1 for the fill created by eliminating
// with row k; entries of level <= k are kept.  Fill stays inside the row's block when blocks
// are given.  The numeric phase is the IKJ elimination of ILU(0) on the resulting pattern.
// Returns the pattern (rp, ci, sorted columns) with A's values scattered into it (fill 0).
static void iluk_pattern(int64_t n, const int64_t *rp, const int32_t *ci, const double *v, int lev_fill,
                         const std::vector<int32_t> &blk, std::vector<int64_t> &erp, std::vector<int32_t> &eci,
                         std::vector<int32_t> &elev, std::vector<double> &ev) {
  erp.assign(size_t(n) + 1, 0);
  eci.clear(); elev.clear(); ev.clear();
  std::vector<int> lev(size_t(n), -1);
  std::vector<double> val(size_t(n), 0.0);
  for (int64_t i = 0; i < n; ++i) {
    std::set<int32_t> cols;
    for (int64_t k = rp[i]; k < rp[i + 1]; ++k) { cols.insert(ci[k]); lev[size_t(ci[k])] = 0; val[size_t(ci[k])] = v[k]; }
    for (auto it = cols.begin(); it != cols.end() && *it < i; ++it) {
      const int32_t k = *it;
      if (blk[size_t(k)] != blk[size_t(i)]) continue;
      const int lik = lev[size_t(k)];
      for (int64_t kk = erp[size_t(k)]; kk < erp[size_t(k) + 1]; ++kk) {
        const int32_t j = eci[size_t(kk)];
        if (j <= k || blk[size_t(j)] != blk[size_t(i)]) continue;
        const int l = lik + elev[size_t(kk)] + 1;
        if (l > lev_fill) continue;
        if (lev[size_t(j)] < 0) { lev[size_t(j)] = l; val[size_t(j)] = 0.0; cols.insert(j); }
        else if (l < lev[size_t(j)]) lev[size_t(j)] = l;
      }
    }
    for (int32_t j : cols) { eci.push_back(j); elev.push_back(lev[size_t(j)]); ev.push_back(val[size_t(j)]); lev[size_t(j)] = -1; val[size_t(j)] = 0.0; }
    erp[size_t(i) + 1] = int64_t(eci.size());
  }
}

static ILU iluk(int64_t n, const int64_t *rp, const int32_t *ci, const double *v, int lev_fill, int64_t nb, const int64_t *bptr) {
  std::vector<int32_t> blk = row_blocks(n, nb, bptr);
  std::vector<int64_t> erp; std::vector<int32_t> eci, elev; std::vector<double> ev;
  iluk_pattern(n, rp, ci, v, lev_fill, blk, erp, eci, elev, ev);
  std::vector<double> lu; std::vector<int64_t> diag;
  ilu0_values(n, erp.data(), eci.data(), ev.data(), blk, lu, diag);
  ILU f; f.n = n; f.lrp.assign(1, 0); f.urp.assign(1, 0);
  for (int64_t i = 0; i < n; ++i) {
    for (int64_t k = erp[size_t(i)]; k < erp[size_t(i) + 1]; ++k) {
      int64_t j = eci[size_t(k)];
      if (blk[size_t(j)] != blk[size_t(i)]) continue;
      if (j < i) { f.lci.push_back(int32_t(j)); f.lv.push_back(lu[size_t(k)]); }
    }
    f.uci.push_back(int32_t(i)); f.uv.push_back(lu[size_t(diag[size_t(i)])]);
    for (int64_t k = erp[size_t(i)]; k < erp[size_t(i) + 1]; ++k) {
      int64_t j = eci[size_t(k)];
      if (blk[size_t(j)] != blk[size_t(i)]) continue;
      if (j > i) { f.uci.push_back(int32_t(j)); f.uv.push_back(lu[size_t(k)]); }
    }
    f.lrp.push_back(int64_t(f.lci.size())); f.urp.push_back(int64_t(f.uci.size()));
  }
  return f;
}

// ILUT(p, tau), Saad Alg. 10.6 (row-wise, dual dropping).
// With blk (a block id per row), the factorisation is restricted to the blocks, as the library's
// slab-restricted ILUT: a row is not eliminated with rows of other blocks and takes no fill from
// them; tau * ||a_i|| uses the whole row, and the entries of other blocks take part in the
// p-largest rule of L and of U, but are not part of the factor.
static ILU ilut(int64_t n, const int64_t *rp, const int32_t *ci, const double *v, int p, double tau,
                std::vector<std::vector<int32_t>> *passed = nullptr, const std::vector<int32_t> *blk = nullptr) {
  ILU f; f.n = n; f.lrp.assign(1, 0); f.urp.assign(1, 0);
  std::vector<double> w(size_t(n), 0.0);
  std::vector<char> nz(size_t(n), 0);
  std::vector<int64_t> udiag;  // position of each row's diagonal in uv
  for (int64_t i = 0; i < n; ++i) {
    std::vector<int32_t> cols;
    double rn = 0;
    for (int64_t k = rp[i]; k < rp[i + 1]; ++k) {
      int32_t j = ci[k]; w[j] = v[k]; if (!nz[j]) { nz[j] = 1; cols.push_back(j); }
      rn += v[k] * v[k];
    }
    const double ti = tau * std::sqrt(rn);
    if (!nz[i]) { nz[i] = 1; w[i] = 0.0; cols.push_back(int32_t(i)); }
    // eliminate lower entries in increasing column order (the set grows with fill)
    std::vector<int32_t> heap;
    for (int32_t j : cols) if (j < i) heap.push_back(j);
    std::make_heap(heap.begin(), heap.end(), std::greater<int32_t>());
    while (!heap.empty()) {
      std::pop_heap(heap.begin(), heap.end(), std::greater<int32_t>());
      int32_t k = heap.back(); heap.pop_back();
      if (blk && (*blk)[size_t(k)] != (*blk)[size_t(i)]) continue;  // another block: no elimination
      double wk = w[k] / f.uv[size_t(f.urp[k])];
      if (std::fabs(wk) < ti) { w[k] = 0.0; continue; }
      w[k] = wk;
      for (int64_t kk = f.urp[k] + 1; kk < f.urp[k + 1]; ++kk) {
        int32_t j = f.uci[size_t(kk)];
        if (blk && (*blk)[size_t(j)] != (*blk)[size_t(i)]) continue;
        if (!nz[j]) { nz[j] = 1; w[j] = 0.0; cols.push_back(j); if (j < i) { heap.push_back(j); std::push_heap(heap.begin(), heap.end(), std::greater<int32_t>()); } }
        w[j] -= wk * f.uv[size_t(kk)];
      }
    }
    std::vector<std::pair<double, int32_t>> lo, up;
    double d = w[i];
    for (int32_t j : cols) {
      if (j == i) continue;
      if (std::fabs(w[j]) < ti || w[j] == 0.0) continue;
      if (j < i) lo.push_back({std::fabs(w[j]), j}); else up.push_back({std::fabs(w[j]), j});
    }
    auto keep = [&](std::vector<std::pair<double, int32_t>> &s) {
      if (int(s.size()) > p) {
        std::nth_element(s.begin(), s.begin() + p, s.end(), [](const std::pair<double, int32_t> &a, const std::pair<double, int32_t> &b) { return a.first > b.first; });
        s.resize(size_t(p));
      }
      std::sort(s.begin(), s.end(), [](const std::pair<double, int32_t> &a, const std::pair<double, int32_t> &b) { return a.second < b.second; });
    };
    if (passed) {  // the entries that passed the tau test, before the p-largest rule
      auto &ps = (*passed)[size_t(i)];
      for (auto &e : lo) ps.push_back(e.second);
      for (auto &e : up) ps.push_back(e.second);
      std::sort(ps.begin(), ps.end());
    }
    keep(lo); keep(up);
    if (blk) {  // entries of other blocks are ranked above but are not part of the factor
      auto other = [&](const std::pair<double, int32_t> &e) { return (*blk)[size_t(e.second)] != (*blk)[size_t(i)]; };
      lo.erase(std::remove_if(lo.begin(), lo.end(), other), lo.end());
      up.erase(std::remove_if(up.begin(), up.end(), other), up.end());
    }
    for (auto &e : lo) { f.lci.push_back(e.second); f.lv.push_back(w[e.second]); }
    if (d == 0.0) d = (ti > 0 ? ti : 1.0);  // guard a zero pivot
    f.uci.push_back(int32_t(i)); f.uv.push_back(d);
    for (auto &e : up) { f.uci.push_back(e.second); f.uv.push_back(w[e.second]); }
    f.lrp.push_back(int64_t(f.lci.size())); f.urp.push_back(int64_t(f.uci.size()));
    for (int32_t j : cols) { nz[j] = 0; w[j] = 0.0; }
  }
  return f;
}

struct SolveStats { int iters = 0; double relres = 0; int status = 0; double t_setup = 0, t_iter = 0; };

// BiCGStab (van der Vorst 1992), right preconditioning; stops on ||r_k|| / ||b|| < tol.
static int bicgstab(int64_t n, const int64_t *rp, const int32_t *ci, const double *v, const double *b, double *x,
                    const ILU *M, double tol, int maxit, SolveStats &st) {
  const size_t N = size_t(n);
  std::vector<double> r(N), rh, p(N, 0.0), vv(N, 0.0), s(N), t(N), ph(N), sh(N);
  std::vector<double> xv(x, x + n), bv(b, b + n);
  spmv(n, rp, ci, v, xv.data(), r.data());
  for (int64_t i = 0; i < n; ++i) r[size_t(i)] = bv[size_t(i)] - r[size_t(i)];
  rh = r;
  double nb = nrm2(bv);
  if (nb == 0.0) { std::fill(x, x + n, 0.0); st.iters = 0; st.relres = 0; return 0; }
  double rho_old = 1, alpha = 1, omega = 1;
  double res = nrm2(r) / nb;
  st.relres = res;
  if (res < tol) { st.iters = 0; return 0; }
  for (int it = 1; it <= maxit; ++it) {
    double rho = dot(rh, r);
    if (rho == 0.0) { st.status = -1; st.iters = it; return -1; }
    if (it == 1) p = r;
    else {
      double beta = (rho / rho_old) * (alpha / omega);
      for (int64_t i = 0; i < n; ++i) p[size_t(i)] = r[size_t(i)] + beta * (p[size_t(i)] - omega * vv[size_t(i)]);
    }
    if (M) M->apply(p.data(), ph.data()); else ph = p;
    spmv(n, rp, ci, v, ph.data(), vv.data());
    double rv = dot(rh, vv);
    if (rv == 0.0) { st.status = -1; st.iters = it; return -1; }
    alpha = rho / rv;
    for (int64_t i = 0; i < n; ++i) s[size_t(i)] = r[size_t(i)] - alpha * vv[size_t(i)];
    double sn = nrm2(s) / nb;
    if (sn < tol) {
      for (int64_t i = 0; i < n; ++i) xv[size_t(i)] += alpha * ph[size_t(i)];
      st.iters = it; st.relres = sn;
      std::copy(xv.begin(), xv.end(), x);
      return 0;
    }
    if (M) M->apply(s.data(), sh.data()); else sh = s;
    spmv(n, rp, ci, v, sh.data(), t.data());
    double tt = dot(t, t);
    omega = tt == 0.0 ? 0.0 : dot(t, s) / tt;
    for (int64_t i = 0; i < n; ++i) {
      xv[size_t(i)] += alpha * ph[size_t(i)] + omega * sh[size_t(i)];
      r[size_t(i)] = s[size_t(i)] - omega * t[size_t(i)];
    }
    res = nrm2(r) / nb;
    st.iters = it; st.relres = res;
    if (res < tol) { std::copy(xv.begin(), xv.end(), x); return 0; }
    if (omega == 0.0) { st.status = -1; std::copy(xv.begin(), xv.end(), x); return -1; }
    rho_old = rho;
  }
  std::copy(xv.begin(), xv.end(), x);
  st.status = 1;  // not converged
  return 1;
}

// Dense Gauss with partial pivoting: src/solvers/native/dense_linear_solver.hpp:77-133
static int dense_solve(int64_t n, const int64_t *rp, const int32_t *ci, const double *v, const double *b, double *x) {
  std::vector<double> A(size_t(n * n), 0.0), rhs(b, b + n);
  for (int64_t i = 0; i < n; ++i)
    for (int64_t k = rp[i]; k < rp[i + 1]; ++k) A[size_t(i * n + ci[k])] += v[k];
  for (int64_t c = 0; c < n; ++c) {
    int64_t piv = c; double best = std::fabs(A[size_t(c * n + c)]);
    for (int64_t r = c + 1; r < n; ++r) if (std::fabs(A[size_t(r * n + c)]) > best) { best = std::fabs(A[size_t(r * n + c)]); piv = r; }
    if (best == 0.0) return -1;
    if (piv != c) { for (int64_t j = 0; j < n; ++j) std::swap(A[size_t(c * n + j)], A[size_t(piv * n + j)]); std::swap(rhs[size_t(c)], rhs[size_t(piv)]); }
    for (int64_t r = c + 1; r < n; ++r) {
      double f = A[size_t(r * n + c)] / A[size_t(c * n + c)];
      if (f == 0.0) continue;
      for (int64_t j = c; j < n; ++j) A[size_t(r * n + j)] -= f * A[size_t(c * n + j)];
      rhs[size_t(r)] -= f * rhs[size_t(c)];
    }
  }
  for (int64_t i = n - 1; i >= 0; --i) {
    double s = rhs[size_t(i)];
    for (int64_t j = i + 1; j < n; ++j) s -= A[size_t(i * n + j)] * x[j];
    x[i] = s / A[size_t(i * n + i)];
  }
  return 0;
}

// ---------------------------------------------------------------------------
// post-processing: viennashe/she/postproc/carrier_density.hpp:68-130,
// current_density.hpp:66-131, viennashe/postproc/terminal_current.hpp:47-105
// ---------------------------------------------------------------------------
static void density(const Problem &p, const std::vector<double> &xf, double *out) {
  for (int c = 0; c < p.nc; ++c) {
    Elem e{&p, false, c};
    double d = 0;
    const double es = 0.0, ee = 1.0;
    for (size_t H = 1; H < p.NH - 1; ++H) {
      double lo = std::max((p.ekin_c(c, H - 1) + p.ekin_c(c, H)) / 2.0, es);
      double up = std::min((p.ekin_c(c, H + 1) + p.ekin_c(c, H)) / 2.0, ee);
      if (p.mask_c[c]) {
        long u = p.idx_c[c * p.NH + H];
        if (u < 0) continue;
        if (up >= 0 && lo < up) d += xf[size_t(u)] * averaged_dos(e, H) * box_height(e, H);
      } else {
        if (up >= 0 && lo < up) d += p.bnd_c[c * p.NH + H] * averaged_dos(e, H) * box_height(e, H);
      }
    }
    out[c] = d * SYMMETRY;
  }
}
static double current_on_facet(const Problem &p, const std::vector<double> &xf, int f) {
  int c1 = p.fcell[2 * f], c2 = p.fcell[2 * f + 1];
  if (c2 < 0) return 0;
  double nrm[2] = {0, 0}, len = 0;
  for (int d = 0; d < p.dim; ++d) { nrm[d] = p.cen[c2 * p.dim + d] - p.cen[c1 * p.dim + d]; len += nrm[d] * nrm[d]; }
  len = std::sqrt(len);
  for (int d = 0; d < p.dim; ++d) nrm[d] /= len;
  double vn = 0, pol = -1.0;
  double mt = m_trans(), md = m_dos();
  // L = 1 coupling entries a_{x,y}(0, 1..3)
  double ax1 = p.ax.get(0, 1), ax2 = p.ax.get(0, 2), ax3 = p.ax.get(0, 3);
  double ay1 = p.ay.get(0, 1), ay2 = p.ay.get(0, 2), ay3 = p.ay.get(0, 3);
  Elem fe{&p, true, f};
  for (size_t H = 1; H < p.NH - 1; ++H) {
    long u = p.idx_f[f * p.NH + H];
    if (u < 0) continue;
    double factor = integral_vZ(fe, H) * SYMMETRY;
    const double *val = &xf[size_t(u)];
    vn += (ax1 * val[0] + ax2 * val[1] + ax3 * val[2]) * factor * std::sqrt(md / mt) * nrm[0];
    if (p.dim > 1) vn += (ay1 * val[0] + ay2 * val[1] + ay3 * val[2]) * factor * std::sqrt(md / mt) * nrm[1];
  }
  // Y_00 as spherical_harmonics.hpp:102-119 evaluates it: normalisation * P_0^0 / sqrt(2)
  const double Y00 = std::sqrt((2.0 * 0 + 1.0) * 1.0 / (2.0 * PI * 1.0)) * 1.0 / std::sqrt(2.0);
  return -pol * Q * vn / Y00;
}
static void terminal_currents(const Problem &p, const std::vector<double> &xf, int ncontacts, double *out) {
  for (int k = 0; k < ncontacts; ++k) out[k] = 0.0;
  for (int c = 0; c < p.nc; ++c) {
    int k = p.contact[c];
    if (k < 0 || k >= ncontacts) continue;
    for (int j = p.cf_ptr[c]; j < p.cf_ptr[c + 1]; ++j) {
      int f = p.cf_idx[j];
      int o = p.other_cell(f, c);
      if (o < 0 || !p.is_semi(o)) continue;  // interface between the terminal and the semiconductor
      double conn[2] = {0, 0}, len = 0;
      for (int d = 0; d < p.dim; ++d) { conn[d] = p.cen[o * p.dim + d] - p.cen[c * p.dim + d]; len += conn[d] * conn[d]; }
      len = std::sqrt(len);
      double sgn = (p.fcell[2 * f] == c) ? 1.0 : -1.0, dt = 0;
      for (int d = 0; d < p.dim; ++d) dt += sgn * p.fnorm[f * p.dim + d] * conn[d] / len;
      double wa = p.fvol[f] * dt;
      double J = current_on_facet(p, xf, f);
      if (p.fcell[2 * f] == c) out[k] += J * wa;
      else out[k] -= J * wa;
    }
  }
}

}  // namespace vsheo

using namespace vsheo;

struct vsheo_handle {
  Problem p;
};

static void set_err(char *err, int n, const std::string &s) {
  if (err && n > 0) { std::strncpy(err, s.c_str(), size_t(n - 1)); err[n - 1] = 0; }
}

static void load_coupling(Problem &p, const vshe_coupling_tables *ct) {
  const int D = (ct->L + 1) * (ct->L + 1);
  Mat *m[6] = {&p.ax, &p.ay, &p.az, &p.bx, &p.by, &p.bz};
  for (int t = 0; t < 6; ++t) {
    *m[t] = Mat(size_t(D));
    for (int i = 0; i < D; ++i)
      for (int j = 0; j < D; ++j) {
        double x = ct->data[size_t(t) * D * D + size_t(i) * D + j];
        if (x != 0.0) m[t]->at(size_t(i), size_t(j)) = x;
      }
  }
}

static void csr_out(const Mat &A, int64_t *rp, int32_t *ci, double *v) {
  size_t k = 0;
  for (size_t i = 0; i < A.size(); ++i) {
    if (rp) rp[i] = int64_t(k);
    for (auto &e : A.r[i]) { if (ci) ci[k] = int32_t(e.first); if (v) v[k] = e.second; ++k; }
  }
  if (rp) rp[A.size()] = int64_t(k);
}

extern "C" {

// Runs setup, assembly, odd elimination, scaling and normalisation (everything
// she::solve does before the linear solver).  Returns NULL on error.
void *vsheo_create(const vshe_device_desc *d, const vshe_she_config *cfg, const vshe_coupling_tables *ct, char *err, int errlen) {
  std::unique_ptr<vsheo_handle> h(new vsheo_handle);
  Problem &p = h->p;
  try {
    p.dim = d->dim; p.nc = d->n_cells; p.nf = d->n_facets; p.T = d->temperature;
    p.mat.assign(d->cell_material, d->cell_material + p.nc);
    p.vol.assign(d->cell_volume, d->cell_volume + p.nc);
    p.cen.assign(d->cell_centroid, d->cell_centroid + size_t(p.nc) * p.dim);
    p.nd.assign(d->doping_n, d->doping_n + p.nc);
    p.na.assign(d->doping_p, d->doping_p + p.nc);
    p.phi.assign(d->potential, d->potential + p.nc);
    p.contact.assign(d->contact_id, d->contact_id + p.nc);
    p.fcell.assign(d->facet_cells, d->facet_cells + 2 * size_t(p.nf));
    p.fvol.assign(d->facet_volume, d->facet_volume + p.nf);
    p.fnorm.assign(d->facet_normal, d->facet_normal + size_t(p.nf) * p.dim);
    p.cf_ptr.assign(d->cell_facet_ptr, d->cell_facet_ptr + p.nc + 1);
    p.cf_idx.assign(d->cell_facet_idx, d->cell_facet_idx + p.cf_ptr[p.nc]);
    p.cfg = *cfg;
    p.L = cfg->max_expansion_order;
    if (ct->L != p.L) throw std::runtime_error("coupling table order differs from max_expansion_order");
    load_coupling(p, ct);
    snap_phonon_energy(p);
    setup_energies(p);
    distribute_expansion_orders(p);
    write_boundary_conditions(p);
    create_mapping(p);
    assemble(p);
    // she::solve: viennashe/she/linear_solver.hpp:100-189
    p.A_diag = p.A_full; p.b_diag = p.b_full;
    diagonalise_odd2odd(p.A_diag, p.b_diag, size_t(p.n_even));
    p.A_red0 = Mat(size_t(p.n_even)); p.b_red0.assign(size_t(p.n_even), 0.0);
    eliminate_odd(p.A_diag, p.b_diag, p.A_red0, p.b_red0);
    p.A_red = p.A_red0; p.b_red = p.b_red0;
    p.scaling.assign(size_t(p.n_even), 1.0);
    if (p.cfg.scale) { setup_scaling(p); rescale(p.A_red, p.scaling); }
    p.scale_factors = row_normalize(p.A_red, p.b_red);
    fill_block_indices(p);
  } catch (std::exception &e) {
    set_err(err, errlen, e.what());
    return nullptr;
  }
  return h.release();
}

void vsheo_destroy(void *h) { delete static_cast<vsheo_handle *>(h); }

// out: [NH, n_even, n_odd, nnz_full, nnz_diag, nnz_red0, nnz_red, n_cells, n_facets]
void vsheo_info(void *hh, int64_t *out) {
  Problem &p = static_cast<vsheo_handle *>(hh)->p;
  out[0] = int64_t(p.NH); out[1] = p.n_even; out[2] = p.n_odd;
  out[3] = int64_t(p.A_full.nnz()); out[4] = int64_t(p.A_diag.nnz());
  out[5] = int64_t(p.A_red0.nnz()); out[6] = int64_t(p.A_red.nnz());
  out[7] = p.nc; out[8] = p.nf;
}

void vsheo_energies(void *hh, double *H, double *shift_c, double *shift_f, double *hbar_omega) {
  Problem &p = static_cast<vsheo_handle *>(hh)->p;
  std::copy(p.Hval.begin(), p.Hval.end(), H);
  std::copy(p.shift_c.begin(), p.shift_c.end(), shift_c);
  std::copy(p.shift_f.begin(), p.shift_f.end(), shift_f);
  *hbar_omega = p.hbar_omega;
}

void vsheo_mapping(void *hh, int64_t *idx_c, int64_t *idx_f, int32_t *ord_c, int32_t *ord_f, double *bnd_c) {
  Problem &p = static_cast<vsheo_handle *>(hh)->p;
  for (size_t i = 0; i < p.idx_c.size(); ++i) { idx_c[i] = p.idx_c[i]; ord_c[i] = int32_t(p.ord_c[i]); bnd_c[i] = p.bnd_c[i]; }
  for (size_t i = 0; i < p.idx_f.size(); ++i) { idx_f[i] = p.idx_f[i]; ord_f[i] = int32_t(p.ord_f[i]); }
}

// which: 0 = assembled A_full, 1 = after diagonalise (used by recovery),
//        2 = A_red after elimination, 3 = A_red after scaling + normalisation
int vsheo_matrix(void *hh, int which, int64_t *rp, int32_t *ci, double *v, double *rhs) {
  Problem &p = static_cast<vsheo_handle *>(hh)->p;
  const Mat *A = nullptr; const std::vector<double> *b = nullptr;
  switch (which) {
    case 0: A = &p.A_full; b = &p.b_full; break;
    case 1: A = &p.A_diag; b = &p.b_diag; break;
    case 2: A = &p.A_red0; b = &p.b_red0; break;
    case 3: A = &p.A_red; b = &p.b_red; break;
    default: return -1;
  }
  csr_out(*A, rp, ci, v);
  if (rhs) std::copy(b->begin(), b->end(), rhs);
  return 0;
}

void vsheo_scaling(void *hh, double *scaling, double *scale_factors) {
  Problem &p = static_cast<vsheo_handle *>(hh)->p;
  std::copy(p.scaling.begin(), p.scaling.end(), scaling);
  std::copy(p.scale_factors.begin(), p.scale_factors.end(), scale_factors);
}

// energy-slab block boundaries (fill_block_indices), NH + 1 entries: [first_0, first_1, ..., n_even]
void vsheo_blocks(void *hh, int64_t *bptr) {
  Problem &p = static_cast<vsheo_handle *>(hh)->p;
  for (size_t i = 0; i < p.blocks.size(); ++i) bptr[i] = int64_t(p.blocks[i].first);
  bptr[p.blocks.size()] = p.n_even;
}

// From the solution of the normalised reduced system: unscale, recover the odd
// unknowns, full-system residual, carrier density per cell, terminal currents.
int vsheo_finish(void *hh, const double *x_red, double *x_full, double *dens, double *currents, int ncontacts, double *full_res) {
  Problem &p = static_cast<vsheo_handle *>(hh)->p;
  std::vector<double> xe(x_red, x_red + p.n_even);
  if (p.cfg.scale)
    for (size_t i = 0; i < xe.size(); ++i) xe[i] *= p.scaling[i] * p.scale_factors[i];
  std::vector<double> xf = recover_odd(p.A_diag, p.b_diag, xe);
  std::copy(xf.begin(), xf.end(), x_full);
  // linear_solver.hpp:183-186
  std::vector<double> Ax(xf.size());
  CSR c = to_csr(p.A_diag);
  spmv(c.n, c.rp.data(), c.ci.data(), c.v.data(), xf.data(), Ax.data());
  double num = 0, den = 0;
  for (size_t i = 0; i < Ax.size(); ++i) { double t = Ax[i] - p.b_diag[i]; num += t * t; den += p.b_diag[i] * p.b_diag[i]; }
  *full_res = std::sqrt(num) / std::sqrt(den);
  if (dens) density(p, xf, dens);
  if (currents) terminal_currents(p, xf, ncontacts, currents);
  return 0;
}

// ---- CSR-level solvers (the reference's solvers::solve backends, restated) ----

// precond: 0 none, 1 ILU0, 2 ILUT(p, tau), 3 block ILU0 over [bptr[k], bptr[k+1])
int vsheo_csr_solve(int64_t n, const int64_t *rp, const int32_t *ci, const double *v, const double *b, double *x,
                    int precond, int ilut_p, double ilut_tau, int64_t nb, const int64_t *bptr,
                    double tol, int maxit, int *iters, double *relres, double *t_setup, double *t_solve) {
  try {
    auto t0 = std::chrono::steady_clock::now();
    ILU M; const ILU *pm = nullptr;
    if (precond == 1) { M = ilu0(n, rp, ci, v, 0, nullptr); pm = &M; }
    else if (precond == 2) {
      const std::vector<int32_t> blk = row_blocks(n, nb, bptr);
      M = ilut(n, rp, ci, v, ilut_p, ilut_tau, nullptr, nb > 0 ? &blk : nullptr);
      pm = &M;
    }
    else if (precond == 3) { M = ilu0(n, rp, ci, v, nb, bptr); pm = &M; }
    else if (precond == 4) { M = iluk(n, rp, ci, v, ilut_p, nb, bptr); pm = &M; }
    auto t1 = std::chrono::steady_clock::now();
    SolveStats st;
    std::fill(x, x + n, 0.0);
    int rc = bicgstab(n, rp, ci, v, b, x, pm, tol, maxit, st);
    auto t2 = std::chrono::steady_clock::now();
    if (iters) *iters = st.iters;
    if (relres) *relres = st.relres;
    if (t_setup) *t_setup = std::chrono::duration<double>(t1 - t0).count();
    if (t_solve) *t_solve = std::chrono::duration<double>(t2 - t1).count();
    return rc;
  } catch (std::exception &) {
    return -2;
  }
}

// ILU(k) factor in CSR (pattern of levels of fill <= k, block-restricted when nb > 0): call with
// erp == NULL to get the entry count in *nnz_out, then with arrays of that size.
int vsheo_iluk_csr(int64_t n, const int64_t *rp, const int32_t *ci, const double *v, int32_t lev_fill, int64_t nb, const int64_t *bptr,
                   int64_t *nnz_out, int64_t *erp_out, int32_t *eci_out, double *lu_out) {
  try {
    std::vector<int32_t> blk = row_blocks(n, nb, bptr);
    std::vector<int64_t> erp; std::vector<int32_t> eci, elev; std::vector<double> ev;
    iluk_pattern(n, rp, ci, v, lev_fill, blk, erp, eci, elev, ev);
    *nnz_out = erp[size_t(n)];
    if (!erp_out) return 0;
    std::vector<double> lu; std::vector<int64_t> diag;
    ilu0_values(n, erp.data(), eci.data(), ev.data(), blk, lu, diag);
    std::copy(erp.begin(), erp.end(), erp_out);
    std::copy(eci.begin(), eci.end(), eci_out);
    std::copy(lu.begin(), lu.end(), lu_out);
    return 0;
  } catch (...) { return -1; }
}

// ILUT(p, tau) factor as one CSR (L strictly lower, then U with its diagonal, columns ascending):
// call with rp_out == NULL for the entry count, then with arrays of that size.
int vsheo_ilut_csr(int64_t n, const int64_t *rp, const int32_t *ci, const double *v, int32_t p, double tau,
                   int64_t nb, const int64_t *bptr, int64_t *nnz_out, int64_t *rp_out, int32_t *ci_out, double *lu_out) {
  try {
    const std::vector<int32_t> blk = row_blocks(n, nb, bptr);
    ILU f = ilut(n, rp, ci, v, p, tau, nullptr, nb > 0 ? &blk : nullptr);
    *nnz_out = int64_t(f.lci.size() + f.uci.size());
    if (!rp_out) return 0;
    int64_t q = 0;
    rp_out[0] = 0;
    for (int64_t i = 0; i < n; ++i) {
      for (int64_t k = f.lrp[size_t(i)]; k < f.lrp[size_t(i) + 1]; ++k) { ci_out[q] = f.lci[size_t(k)]; lu_out[q++] = f.lv[size_t(k)]; }
      for (int64_t k = f.urp[size_t(i)]; k < f.urp[size_t(i) + 1]; ++k) { ci_out[q] = f.uci[size_t(k)]; lu_out[q++] = f.uv[size_t(k)]; }
      rp_out[i + 1] = q;
    }
    return 0;
  } catch (...) { return -1; }
}

// Per row, the columns whose entries passed ILUT's tau test (before its p-largest rule), as a
// CSR pattern: call with rp_out == NULL for the count.
int vsheo_ilut_passed(int64_t n, const int64_t *rp, const int32_t *ci, const double *v, int32_t p, double tau,
                      int64_t nb, const int64_t *bptr, int64_t *nnz_out, int64_t *rp_out, int32_t *ci_out) {
  try {
    std::vector<std::vector<int32_t>> passed((size_t)n);
    const std::vector<int32_t> blk = row_blocks(n, nb, bptr);
    ilut(n, rp, ci, v, p, tau, &passed, nb > 0 ? &blk : nullptr);
    int64_t q = 0;
    for (auto &r : passed) q += int64_t(r.size());
    *nnz_out = q;
    if (!rp_out) return 0;
    q = 0;
    rp_out[0] = 0;
    for (int64_t i = 0; i < n; ++i) {
      for (int32_t j : passed[size_t(i)]) ci_out[q++] = j;
      rp_out[i + 1] = q;
    }
    return 0;
  } catch (...) { return -1; }
}

// ILU0 factor values in the pattern of A (block-restricted when nb > 0).
int vsheo_ilu0_values(int64_t n, const int64_t *rp, const int32_t *ci, const double *v, int64_t nb, const int64_t *bptr, double *lu) {
  try {
    std::vector<int32_t> blk = row_blocks(n, nb, bptr);
    std::vector<double> f; std::vector<int64_t> diag;
    ilu0_values(n, rp, ci, v, blk, f, diag);
    std::copy(f.begin(), f.end(), lu);
    return 0;
  } catch (std::exception &) {
    return -1;
  }
}

// Apply (L U)^{-1} for the factor values returned by vsheo_ilu0_values.
int vsheo_ilu0_apply(int64_t n, const int64_t *rp, const int32_t *ci, const double *lu, int64_t nb, const int64_t *bptr, const double *b, double *x) {
  std::vector<int32_t> blk = row_blocks(n, nb, bptr);
  std::vector<double> y(b, b + n);
  for (int64_t i = 0; i < n; ++i) {
    double s = y[size_t(i)];
    for (int64_t k = rp[i]; k < rp[i + 1]; ++k) {
      int64_t j = ci[k];
      if (j >= i) break;
      if (blk[size_t(j)] != blk[size_t(i)]) continue;
      s -= lu[k] * y[size_t(j)];
    }
    y[size_t(i)] = s;
  }
  for (int64_t i = n - 1; i >= 0; --i) {
    double s = y[size_t(i)], d = 0;
    for (int64_t k = rp[i]; k < rp[i + 1]; ++k) {
      int64_t j = ci[k];
      if (j < i) continue;
      if (j == i) { d = lu[k]; continue; }
      if (blk[size_t(j)] != blk[size_t(i)]) continue;
      s -= lu[k] * y[size_t(j)];
    }
    y[size_t(i)] = s / d;
  }
  std::copy(y.begin(), y.end(), x);
  return 0;
}

// The oracle's scalar physics at given arguments, numbered like oracle/ref_physics.cpp's probe
// of the reference's own headers (tests/test_oracle_ref.py compares the two): 0 DOS(in[0]);
// 1 velocity(in[0]); 2 optical phonon number(in[0], T = in[1]); 3 built-in potential(T, N_D, N_A);
// 4 ohmic contact electron density(T, N_D, N_A); 5 acoustic rate(T = in[0], fit factor in[1]);
// 6 optical processes(spacing in[0], T in[1], kinetic energy in[2], fit factor in[3]) -> the rates
// of emission, emission into the state, absorption, absorption into the state, and the snapped
// phonon energy; 7 band weight(T).
int vsheo_physics_probe(int what, const double *in, double *out) {
  Problem p;
  switch (what) {
    case 0: out[0] = dos(in[0]); return 0;
    case 1: out[0] = velocity(in[0]); return 0;
    case 2: out[0] = optical_phonon_number(in[0], in[1]); return 0;
    case 3: out[0] = built_in_potential(in[0], in[1], in[2]); return 0;
    case 4: out[0] = contact_carrier_ohm_n(in[0], in[1], in[2]); return 0;
    case 5:
      p.T = in[0]; p.cfg.acoustic_fit_factor = in[1];
      out[0] = acoustic_rate(p);
      return 0;
    case 6: {
      p.cfg.energy_spacing = in[0]; p.T = in[1]; p.cfg.optical_fit_factor = in[3];
      snap_phonon_energy(p);
      const double r = optical_rate(p), N = optical_phonon_number(p.hbar_omega, p.T);
      out[0] = r * (N + 1.0); out[1] = r * (N + 1.0); out[2] = r * N; out[3] = r * N;
      out[4] = p.hbar_omega;
      return 0;
    }
    case 7: out[0] = band_weight(in[0]); return 0;
  }
  return -1;
}

// Spherical-harmonics index sequence of an iterator type (0 all, 1 even, 2 odd) up to order L.
int vsheo_harmonics(int L, int type, int64_t *out, int cap) {
  int k = 0;
  for (HarmIter it(L, type); it.valid(); it.next()) { if (k < cap) out[k] = *it; ++k; }
  return k;
}

int vsheo_dense_solve(int64_t n, const int64_t *rp, const int32_t *ci, const double *v, const double *b, double *x) {
  return dense_solve(n, rp, ci, v, b, x);
}

void vsheo_spmv(int64_t n, const int64_t *rp, const int32_t *ci, const double *v, const double *x, double *y) {
  spmv(n, rp, ci, v, x, y);
}

// Timed sample of the serial solver on a CSR system: ILU0 factorisation plus
// `iters` BiCGStab iterations (no convergence test), for the CPU baseline.
int vsheo_bench_serial(int64_t n, const int64_t *rp, const int32_t *ci, const double *v, const double *b,
                       int iters, double *t_factor, double *t_per_iter, double *relres) {
  auto t0 = std::chrono::steady_clock::now();
  ILU M = ilu0(n, rp, ci, v, 0, nullptr);
  auto t1 = std::chrono::steady_clock::now();
  std::vector<double> x(size_t(n), 0.0);
  SolveStats st;
  bicgstab(n, rp, ci, v, b, x.data(), &M, 0.0, iters, st);
  auto t2 = std::chrono::steady_clock::now();
  *t_factor = std::chrono::duration<double>(t1 - t0).count();
  *t_per_iter = std::chrono::duration<double>(t2 - t1).count() / (st.iters > 0 ? st.iters : 1);
  *relres = st.relres;
  return st.iters;
}

}  // extern "C"

// poisson_oracle.cpp -- TEST INFRASTRUCTURE, not product code.
//
// CPU restatement (FP64, single-threaded) of the reference's Gummel-linearised Poisson system,
// the checker of the device's vshe_poisson_* path.  Only tests/ call it.
//
//   viennashe/assemble.hpp:165-345   assemble_poisson: per non-Dirichlet cell, per facet to
//                                    another cell, the harmonic-mean permittivity flux term
//                                    (or the Dirichlet term towards a contact cell); then the
//                                    Gummel term q (n + p) / V_T on the diagonal and the charge
//                                    q (n - N_D - p + N_A) in the rhs of semiconductor cells
//   viennashe/materials/all.hpp:45-232  material ids and permittivities
//   viennashe/physics/constants.hpp:60-80, physics/physics.hpp:61-64  q, kB, eps_0, V_T
//
// The matrix is kept as the reference's container keeps it (viennashe/math/linalg_util.hpp:
// one ordered map per row, entries created on first access), so the pattern is the reference's.
// Unknowns are the cells that are not contacts, numbered in cell order (the reference numbers
// the potential's unknowns over the cell range and skips the Dirichlet cells).  The mesh is the
// flat vshe_device_desc; facet centres come from the caller (viennagrid::centroid of a facet).

#include "../include/vshe_types.h"

#include <cmath>
#include <cstdint>
#include <map>
#include <vector>

namespace {

const double kQ = 1.602176565e-19;
const double kKB = 1.3806488e-23;
const double kEps0 = 1.0e7 / (4.0 * 3.1415926535897932384626433832795 * 299792458.0 * 299792458.0);

// materials/all.hpp:49-232; metal (id 100) has no permittivity in the reference (it throws)
double permittivity(int32_t m) {
  switch (m) {
    case 0: return 11.9 * kEps0;
    case 1: return 3.9 * kEps0;
    case 2: return 25.0 * kEps0;
    case 3: return 10.0 * kEps0;
    case 4: return 1.0 * kEps0;
    default: return NAN;
  }
}

double norm(const double *a, const double *b, int dim) {  // |a - b|_2
  double s = 0.0;
  for (int k = 0; k < dim; ++k) s += (a[k] - b[k]) * (a[k] - b[k]);
  return std::sqrt(s);
}

}  // namespace

extern "C" {

// Assembles A (CSR, columns ascending) and b of the Gummel step for the current potential psi
// and densities n, p (all n_cells).  Returns the number of unknowns; *nnz the entries; the
// arrays must hold n_cells + 1 row offsets and max_nnz entries.  -1 on a capacity or material
// error.
int64_t vsheo_poisson_assemble(const vshe_device_desc *d, const double *facet_centroid, const double *psi, const double *n,
                               const double *p, int64_t max_nnz, int64_t *row_ptr, int32_t *col, double *val, double *rhs,
                               int64_t *nnz) {
  const int dim = d->dim;
  const int32_t nc = d->n_cells;
  std::vector<int64_t> unk((size_t)nc, -1);
  int64_t nu = 0;
  for (int32_t c = 0; c < nc; ++c)
    if (d->contact_id[c] < 0) unk[(size_t)c] = nu++;
  std::vector<std::map<int64_t, double>> A((size_t)nu);
  std::vector<double> b((size_t)nu, 0.0);
  const double VT = (kKB * d->temperature) / kQ;  // physics.hpp:61-64
  for (int32_t c = 0; c < nc; ++c) {
    const int64_t row = unk[(size_t)c];
    if (row < 0) continue;  // Dirichlet (contact) cell
    const double *cc = d->cell_centroid + (size_t)c * dim;
    const double potential_center = psi[c];
    const double permittivity_center = permittivity(d->cell_material[c]);
    if (std::isnan(permittivity_center)) return -1;
    b[(size_t)row] = 0;
    A[(size_t)row][row] = 0;
    for (int32_t k = d->cell_facet_ptr[c]; k < d->cell_facet_ptr[c + 1]; ++k) {
      const int32_t f = d->cell_facet_idx[k];
      const int32_t c1 = d->facet_cells[2 * f], c2 = d->facet_cells[2 * f + 1];
      const int32_t o = c1 == c ? c2 : c1;
      if (o < 0) continue;  // boundary of the domain: homogeneous Neumann
      const double *co = d->cell_centroid + (size_t)o * dim;
      double conn[3], nrm[3];
      for (int q = 0; q < dim; ++q) conn[q] = co[q] - cc[q];
      const double len = norm(co, cc, dim);
      double ip = 0.0;
      for (int q = 0; q < dim; ++q) {
        nrm[q] = (c1 == c ? 1.0 : -1.0) * d->facet_normal[(size_t)f * dim + q];  // outer normal of c
        ip += nrm[q] * (conn[q] / len);
      }
      const double weighted_interface_area = d->facet_volume[f] * ip;
      const int64_t col_index = unk[(size_t)o];
      const double potential_outer = psi[o];
      if (col_index >= 0) {
        const double *fc = facet_centroid + (size_t)f * dim;
        const double in_cell = norm(fc, cc, dim), in_other = norm(fc, co, dim);
        const double permittivity_mean = (in_cell + in_other) / (in_cell / permittivity_center + in_other / permittivity(d->cell_material[o]));
        A[(size_t)row][col_index] = permittivity_mean * weighted_interface_area / len;
        A[(size_t)row][row] -= permittivity_mean * weighted_interface_area / len;
        b[(size_t)row] -= permittivity_mean * weighted_interface_area * (potential_outer - potential_center) / len;
      } else {
        // the contact cell's boundary value is its potential in the description
        A[(size_t)row][row] -= permittivity_center * weighted_interface_area / len;
        b[(size_t)row] -= permittivity_center * weighted_interface_area / len * (d->potential[o] - potential_center);
      }
    }
    const double cell_volume = d->cell_volume[c];
    if (d->cell_material[c] == VSHE_MATERIAL_SI) {
      A[(size_t)row][row] -= cell_volume * kQ * (n[c] + p[c]) / VT;
      b[(size_t)row] += cell_volume * kQ * (n[c] - d->doping_n[c] - p[c] + d->doping_p[c]);
    }
  }
  int64_t e = 0;
  row_ptr[0] = 0;
  for (int64_t r = 0; r < nu; ++r) {
    for (auto &kv : A[(size_t)r]) {
      if (e >= max_nnz) return -1;
      col[e] = int32_t(kv.first);
      val[e] = kv.second;
      ++e;
    }
    row_ptr[r + 1] = e;
    rhs[r] = b[(size_t)r];
  }
  *nnz = e;
  return nu;
}

}  // extern "C"

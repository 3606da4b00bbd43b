// she_host.h -- host-side setup of the (x, H) space for one SHE problem:
// energies, expansion orders, unknown mapping, boundary values and the
// direction-resolved coupling blocks the device assembly reads.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

#include "../../include/vshe_types.h"

namespace vshe {

// physical constants and silicon/electron parameters (viennashe/physics/constants.hpp:59-76,
// viennashe/materials/all.hpp:58-99)
struct SheConst {
  static constexpr double PI = 3.1415926535897932384626433832795;
  static constexpr double Q = 1.602176565e-19;
  static constexpr double KB = 1.3806488e-23;
  static constexpr double M0 = 9.10938291e-31;
};

// Everything the device kernels need about one problem, in flat host arrays.
struct SheSetup {
  // device description (copied)
  int dim = 1, nc = 0, nf = 0;
  double T = 300.0;
  std::vector<int32_t> mat, contact, fcell, cf_ptr, cf_idx;
  std::vector<double> vol, cen, nd, na, phi, fvol, fnorm;
  vshe_she_config cfg{};
  int L = 1;
  // (x, H) space
  int32_t NH = 0;
  double hbar_omega = 0.0;
  std::vector<double> Hval, shift_c, shift_f, bnd_c;
  std::vector<int32_t> ord_c, ord_f;      // [elem * NH + H]
  std::vector<int64_t> idx_c, idx_f;      // [elem * NH + H], -1 = no unknown
  std::vector<char> mask_c;
  int64_t n_even = 0, n_odd = 0;
  std::vector<int32_t> even_nodes, odd_nodes;   // pairs (elem, H) in unknown order
  std::vector<int64_t> slab_ptr;                // energy-slab row blocks of the reduced system (NH + 1)
  // harmonics
  int D = 4;                                    // (L+1)^2
  std::vector<int32_t> even_harm, odd_harm;     // index sequences for order L (prefixes give lower orders)
  // coupling blocks per incidence direction: dirs[k] = unit vector; blocks [k][4][D][D]:
  // 0 = diffusion, even rows (a . n), 1 = drift, even rows (b . n),
  // 2 = diffusion, odd rows (a^T . n), 3 = drift, odd rows (b^T . n)
  std::vector<double> dirs;
  std::vector<double> cblocks;
  std::vector<int32_t> inc_dir_even;   // per cell-facet incidence (cf_idx position): block set for the even rows
  std::vector<int32_t> inc_dir_odd;    // per facet * 2 + side: block set for the odd rows of the facet via that cell
  double a_x01[3] = {0, 0, 0}, a_y01[3] = {0, 0, 0};  // L = 1 entries a_{x,y}(0, 1..3) for the current density

  std::string build(const vshe_device_desc &d, const vshe_she_config &c, const vshe_coupling_tables &ct);

  bool is_semi(int c) const { return mat[c] == VSHE_MATERIAL_SI; }
  bool is_metal(int c) const { return mat[c] == VSHE_MATERIAL_METAL; }
  int other_cell(int f, int c) const {
    int c1 = fcell[2 * f], c2 = fcell[2 * f + 1];
    if (c2 < 0) return -1;
    return c1 == c ? c2 : c1;
  }
  double ekin_c(int c, int H) const { return Hval[H] - shift_c[c]; }
  double ekin_f(int f, int H) const { return Hval[H] - shift_f[f]; }
};

// The multicolour order of the reduced rows (SHE problems with ordering = multicolor and no
// caller permutation): perm[t] = reduced row at position t; colour (optional) receives every
// row's colour.
void node_colour_order(const SheSetup &H, int fill_level, std::vector<int32_t> &perm, std::vector<int32_t> *colour);

// Density of states of the Modena dispersion for silicon electrons at kinetic energy eps (J),
// per unit volume and energy (viennashe/physics/dispersion.hpp:207-286); 0 for eps <= 0.
double density_of_states(double eps);

// Spherical-harmonics coupling tables a_{x,y,z}, b_{x,y,z} of order L computed by
// quadrature of the integrals that define them (viennashe/she/harmonics_coupling.hpp:39-200,
// 216-278): out has 6 * D * D entries, values below 1e-8 in magnitude set to 0.
void coupling_quadrature(int L, double *out);

}  // namespace vshe

// gummel.cpp -- the self-consistent electron SHE + Poisson Gummel loop (vshe_gummel_solve),
// written on the public C ABI: the Gummel update of the potential (vshe_poisson_*) and the device
// SHE pipeline (vshe_she_*), with the reference's damping and stopping rules.
//
// Reference: viennashe/simulator.hpp:895-1130 (the loop, its norms and its stopping rules),
// :560-577 (logarithmic damping of the density), solvers/config.hpp:256-257 (tolerance 1e-8,
// 100 iterations, damping 0.3).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>
#include "../../include/vshe_gpu.h"
#include "host_internal.h"

extern "C" int vshe_gummel_solve(vshe_ctx *ctx, const vshe_device_desc *dev, const double *facet_centroid,
                                 const vshe_she_config *cfg, const vshe_coupling_tables *coupling,
                                 const vshe_solve_opts *she_opts, const vshe_gummel_opts *gopts, const double *density0,
                                 const double *p0, double *potential_out, double *density_out, double *currents_out,
                                 double *history, vshe_gummel_stats *stats) {
  if (!ctx || !dev || !facet_centroid || !cfg || !coupling || !density0 || !p0) return VSHE_E_INVALID_ARGUMENT;
  vshe_gummel_opts g{100, 1e-8, 0.3};
  if (gopts) g = *gopts;
  if (g.max_iters <= 0 || !(g.damping > 0.0 && g.damping <= 1.0) || !(g.tol >= 0.0)) return VSHE_E_INVALID_ARGUMENT;
  const size_t nc = size_t(dev->n_cells);
  int ncont = 0;
  for (size_t c = 0; c < nc; ++c) ncont = std::max(ncont, dev->contact_id[c] + 1);
  std::vector<double> psi(dev->potential, dev->potential + nc), n(density0, density0 + nc), p(p0, p0 + nc);
  std::vector<double> psi_new(nc), n_she(nc), cur((size_t)std::max(ncont, 1), 0.0);
  vshe_gummel_stats st{};
  int64_t ph = 0;
  int rc = vshe_poisson_create(ctx, dev, facet_centroid, nullptr, &ph);
  if (rc) return rc;
  bool no_damping = false, break_after = false;
  double initial = 0.0;
  for (int it = 1; it <= g.max_iters; ++it) {
    if (it == g.max_iters) no_damping = true;
    const double alpha = no_damping ? 1.0 : g.damping;
    // spatial quantity: the potential
    vshe_poisson_stats ps{};
    rc = vshe_poisson_update(ctx, ph, psi.data(), n.data(), p.data(), alpha, psi_new.data(), &ps);
    if (rc) break;
    psi.swap(psi_new);
    // SHE quantity: the electron distribution for the new potential, and the density
    vshe_device_desc d = *dev;
    d.potential = psi.data();
    int64_t sh = 0;
    rc = vshe_she_create(ctx, &d, cfg, coupling, she_opts, &sh);
    if (rc) break;
    vshe_solve_stats ss{};
    double full_res = 0.0;
    rc = vshe_she_run(ctx, sh, &ss, &full_res);
    if (!rc) rc = vshe_she_results(ctx, sh, nullptr, n_she.data(), cur.data());
    vshe_she_free(ctx, sh);
    if (rc) break;
    st.she_iterations += ss.iterations;
    for (size_t c = 0; c < nc; ++c) {
      if (dev->contact_id[c] >= 0 || dev->cell_material[c] != VSHE_MATERIAL_SI) continue;
      if (no_damping) { n[c] = n_she[c]; continue; }
      const double nv = std::max(n_she[c], n[c] * 1e-10);
      n[c] = std::pow(n[c], 1.0 - alpha) * std::pow(nv, alpha);
    }
    const double res = ps.rhs_norm;
    st.iterations = it;
    st.potential_increment = ps.update_norm;
    st.rhs_norm = res;
    if (history) {
      history[3 * (it - 1)] = res;
      history[3 * (it - 1) + 1] = ps.update_norm;
      history[3 * (it - 1) + 2] = ss.iterations;
    }
    if (break_after) break;
    if (res == 0.0) break;  // equilibrium: nothing to iterate
    if (it == 1) {
      initial = res;
      st.initial_rhs_norm = res;
    } else if (res / initial < 1e-10 || ps.update_norm < g.tol) {
      no_damping = true;
      break_after = true;
    }
  }
  vshe_poisson_free(ctx, ph);
  if (rc) return rc;
  st.status = (break_after || st.rhs_norm == 0.0) ? VSHE_OK : VSHE_E_NOT_CONVERGED;
  if (potential_out) std::memcpy(potential_out, psi.data(), sizeof(double) * nc);
  if (density_out) std::memcpy(density_out, n.data(), sizeof(double) * nc);
  if (currents_out && ncont > 0) std::memcpy(currents_out, cur.data(), sizeof(double) * size_t(ncont));
  if (stats) *stats = st;
  return st.status;
}

// adapter_check.cpp -- test harness for the drop-in adapter (viennashe-dev_b200/adapter/
// vshe_gpu_solver.hpp), compiled against the reference's own headers (viennashe/forwards.h,
// math/linalg_util.hpp, solvers/config.hpp, util/exception.hpp, log/log.hpp) with
// -DVIENNASHE_HAVE_GPU_SOLVER, and linked to libvshe_b200.so.  It builds the reference's
// sparse_matrix and linear_solver_config from a CSR system and makes the two calls solve_impl
// makes under the define (src/solvers/solve.hpp:77-82): the unqualified gpu-slot call, found by
// argument-dependent lookup, and the qualified AMGX call.  Test infrastructure only.
#define VIENNASHE_HAVE_GPU_SOLVER
#include "vshe_gpu_solver.hpp"

#include <cstring>
#include <exception>
#include <utility>

namespace {
void set_msg(char *msg, int len, const char *s) {
  if (msg && len > 0) { std::strncpy(msg, s, size_t(len) - 1); msg[len - 1] = 0; }
}

viennashe::math::sparse_matrix<double> to_matrix(int64_t n, const int64_t *rp, const int32_t *ci, const double *v) {
  viennashe::math::sparse_matrix<double> A(static_cast<size_t>(n), static_cast<size_t>(n));
  for (int64_t i = 0; i < n; ++i)
    for (int64_t k = rp[i]; k < rp[i + 1]; ++k) A(size_t(i), size_t(ci[k])) = v[k];
  return A;
}

viennashe::solvers::linear_solver_config to_config(double tol, int64_t max_iters, int64_t nslab, const int64_t *slab_ptr) {
  viennashe::solvers::linear_solver_config cfg;
  cfg.set(std::string("gpu_parallel_linear_solver"));
  cfg.tolerance(tol);
  cfg.max_iters(size_t(max_iters));
  for (int64_t s = 0; s < nslab; ++s)
    cfg.block_preconditioner_boundaries().push_back(std::make_pair(size_t(slab_ptr[s]), size_t(slab_ptr[s + 1])));
  return cfg;
}
}  // namespace

extern "C" {

// The gpu-slot solve through the adapter.  Returns 0 (x filled), 1 a linear_solver_exception
// (its text in msg), 2 another exception, 3 the configuration does not select the slot.
int adapter_check_solve(int64_t n, const int64_t *rp, const int32_t *ci, const double *v, const double *b, int64_t nslab,
                        const int64_t *slab_ptr, double tol, int64_t max_iters, double *x, char *msg, int msglen) {
  try {
    viennashe::math::sparse_matrix<double> A = to_matrix(n, rp, ci, v);
    viennashe::solvers::linear_solver_config cfg = to_config(tol, max_iters, nslab, slab_ptr);
    if (cfg.id() != viennashe::solvers::linear_solver_config::gpu_parallel_linear_solver) return 3;
    std::vector<double> rhs(b, b + n);
    using namespace viennashe::solvers;
    std::vector<double> r = solve(A, rhs, cfg, gpu_parallel_linear_solver_tag());
    for (int64_t i = 0; i < n; ++i) x[i] = r[size_t(i)];
    return 0;
  } catch (viennashe::util::linear_solver_exception &e) {
    set_msg(msg, msglen, e.what());
    return 1;
  } catch (std::exception &e) {
    set_msg(msg, msglen, e.what());
    return 2;
  }
}

// The options the adapter derives from a configuration with these slabs (no GPU needed):
// out[0] = precond, out[1] = ordering, out[2] = fill_level, out[3] = n_blocks.
int adapter_check_options(int64_t n, int64_t nslab, const int64_t *slab_ptr, int32_t *out) {
  viennashe::solvers::linear_solver_config cfg = to_config(1e-10, 1000, nslab, slab_ptr);
  std::vector<int64_t> blocks;
  vshe_solve_opts o;
  viennashe::solvers::detail::vshe_gpu_options(cfg, size_t(n), blocks, o);
  out[0] = o.precond; out[1] = o.ordering; out[2] = o.fill_level; out[3] = int32_t(o.n_blocks);
  return 0;
}

// The AMGX case the define also enables: returns 1 when it throws the reference's
// invalid_linear_solver_exception, 0 otherwise.
int adapter_check_amgx(void) {
  viennashe::math::sparse_matrix<double> A(2, 2);
  A(0, 0) = 1.0; A(1, 1) = 1.0;
  std::vector<double> rhs(2, 1.0);
  viennashe::solvers::linear_solver_config cfg;
  try {
    viennashe::solvers::solve(A, rhs, cfg, viennashe::solvers::petsc_amgx_solver_tag());
  } catch (viennashe::solvers::invalid_linear_solver_exception &) {
    return 1;
  }
  return 0;
}

}  // extern "C"

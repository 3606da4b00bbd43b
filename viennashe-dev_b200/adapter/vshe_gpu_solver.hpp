// vshe_gpu_solver.hpp -- the drop-in adapter that binds ViennaSHE's reserved
// gpu_parallel_linear_solver slot to this library (libvshe_b200.so, include/vshe_gpu.h).
//
// A ViennaSHE build adds this header as src/solvers/gpu/vshe_gpu_solver.hpp, includes it in
// src/solvers/solve.hpp beside the other backends (before solve_impl, src/solvers/solve.hpp:44),
// compiles with -DVIENNASHE_HAVE_GPU_SOLVER and links libvshe_b200.so into libshesolvers
// (src/CMakeLists.txt:1-11).  The define enables two dispatch cases in solve_impl
// (src/solvers/solve.hpp:77-82): gpu_parallel_linear_solver, served here, and
// petsc_parallel_AMGX_solver, whose overload the reference does not define anywhere; this header
// defines it so that the reference compiles with the define, and it throws the reference's
// invalid_linear_solver_exception (viennashe/solvers/exception.hpp) as solve_impl's default case
// does for any solver the build does not provide.  The AMGX call in solve_impl is qualified, so
// its overload must be declared before solve_impl: hence the include in solve.hpp.
//
// Reference interfaces used (paths inside viennashe-dev): sparse_matrix
// (viennashe/math/linalg_util.hpp:68-196), linear_solver_config (viennashe/solvers/config.hpp:56-232),
// the solver tags (viennashe/forwards.h:200-217), linear_solver_exception
// (viennashe/util/exception.hpp:38), log::warning (viennashe/log/log.hpp).
#ifndef VSHE_GPU_SOLVER_HPP
#define VSHE_GPU_SOLVER_HPP

#include <cstdint>
#include <string>
#include <vector>

#include "viennashe/forwards.h"
#include "viennashe/log/log.hpp"
#include "viennashe/math/linalg_util.hpp"
#include "viennashe/solvers/config.hpp"
#include "viennashe/solvers/exception.hpp"
#include "viennashe/util/exception.hpp"

#include "vshe_gpu.h"

namespace viennashe {
namespace solvers {

namespace detail {
// One context per process on device 0, created on first use; the library keeps the schedule of
// the last pattern it analysed, so consecutive Gummel steps on an unchanged pattern upload only
// values and right-hand side.
inline vshe_ctx *vshe_gpu_context() {
  static vshe_ctx *ctx = nullptr;
  if (!ctx && vshe_create(&ctx, 0, 0) != VSHE_OK)
    throw viennashe::util::linear_solver_exception("gpu_parallel_linear_solver: no usable CUDA device");
  return ctx;
}

// Solver options from the reference's configuration: tolerance, iteration cap and ILUT
// parameters as given; the preconditioner from the energy-slab bounds that she::solve puts into
// the configuration (she/linear_solver.hpp:160, fill_block_indices :44-83).  With slabs spanning
// the system whose widest one holds at least 4096 rows (2D and 3D meshes), block-ILU(1) per slab
// over a greedy distance-2 colouring inside each slab (the fastest measured on the 2D bar);
// otherwise (1D meshes, whose slabs hold a few hundred rows, and a configuration without slabs)
// natural-order ILU(0) over the whole system, the reference's serial_linear_solver choice:
// per-slab blocks and colourings lose the transport direction there and stall.
inline void vshe_gpu_options(linear_solver_config const &config, std::size_t n, std::vector<int64_t> &blocks,
                             vshe_solve_opts &o) {
  vshe_default_opts(&o);
  o.precision = VSHE_PRECISION_MIXED;
  o.precond = VSHE_PRECOND_ILU0;
  o.ordering = VSHE_ORDER_NATURAL;
  o.tol = config.tolerance();
  o.max_iters = int32_t(config.max_iters());
  o.ilut_entries = int32_t(config.ilut_entries());
  o.ilut_drop = config.ilut_drop_tolerance();
  blocks.clear();
  linear_solver_config::block_preconditioner_boundaries_container const &slabs = config.block_preconditioner_boundaries();
  std::size_t widest = 0;
  for (std::size_t k = 0; k < slabs.size(); ++k)
    if (slabs[k].second > slabs[k].first && slabs[k].second - slabs[k].first > widest) widest = slabs[k].second - slabs[k].first;
  if (!slabs.empty() && slabs.front().first == 0 && slabs.back().second == n && widest >= 4096) {
    for (std::size_t k = 0; k < slabs.size(); ++k) blocks.push_back(int64_t(slabs[k].first));
    blocks.push_back(int64_t(slabs.back().second));
    o.precond = VSHE_PRECOND_BLOCK_ILU0;
    o.n_blocks = int64_t(blocks.size() - 1);
    o.block_ptr = blocks.data();
    o.ordering = VSHE_ORDER_MULTICOLOR;
    o.fill_level = 1;
  }
}
}  // namespace detail

// Overload picked by solve_impl for linear_solver_ids::gpu_parallel_linear_solver.
template <typename NumericT, typename VectorType>
VectorType solve(viennashe::math::sparse_matrix<NumericT> const &A, VectorType const &b, linear_solver_config const &config,
                 gpu_parallel_linear_solver_tag) {
  // std::map rows -> CSR, columns ascending (map order), as serial_linear_solver's copy
  // (src/solvers/viennacl/serial_linear_solver.hpp:52-89)
  const std::size_t n = A.size1();
  std::vector<int64_t> row_ptr(n + 1, 0);
  std::vector<int32_t> col;
  std::vector<double> val;
  col.reserve(A.nnz());
  val.reserve(A.nnz());
  for (std::size_t i = 0; i < n; ++i) {
    typedef typename viennashe::math::sparse_matrix<NumericT>::const_iterator2 It;
    for (It it = A.row(i).begin(); it != A.row(i).end(); ++it) {
      col.push_back(int32_t(it->first));
      val.push_back(double(it->second));
    }
    row_ptr[i + 1] = int64_t(col.size());
  }
  std::vector<int64_t> blocks;
  vshe_solve_opts o;
  detail::vshe_gpu_options(config, n, blocks, o);
  std::vector<double> rhs(b.begin(), b.end()), x(n, 0.0);
  vshe_solve_stats st;
  vshe_ctx *ctx = detail::vshe_gpu_context();
  const int rc = vshe_solve_csr(ctx, int64_t(n), int64_t(col.size()), row_ptr.data(), col.data(), val.data(), rhs.data(), &o,
                                x.data(), &st);
  if (rc == VSHE_E_NOT_CONVERGED)  // the native solvers log and return the last iterate
    viennashe::log::warning() << "gpu_parallel_linear_solver: not converged, relative residual " << st.rel_residual << std::endl;
  else if (rc != VSHE_OK)
    throw viennashe::util::linear_solver_exception(std::string("gpu_parallel_linear_solver: ") + vshe_last_error(ctx));
  VectorType result(n);
  for (std::size_t i = 0; i < n; ++i) result[i] = x[i];
  return result;
}

// The second case the define enables in solve_impl; this backend provides no AMGX solver.
template <typename NumericT, typename VectorType>
VectorType solve(viennashe::math::sparse_matrix<NumericT> const &, VectorType const &, linear_solver_config const &,
                 petsc_amgx_solver_tag) {
  throw invalid_linear_solver_exception();
}

}  // namespace solvers
}  // namespace viennashe

#endif

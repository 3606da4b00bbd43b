/*
 * vshe_gpu.h -- C ABI of the B200 SHE linear-solve backend (libvshe_b200.so).
 *
 * This is the library a ViennaSHE build binds for its reserved
 * gpu_parallel_linear_solver slot.  Every entry point takes plain pointers and
 * sizes; no C++, CUDA or PyTorch types cross the boundary.  All functions
 * return VSHE_OK (0) on success and a negative VSHE_E* code on failure; the
 * message of the last failure on a context is available from vshe_last_error().
 *
 * Reference interfaces this library replaces (paths inside viennashe-dev):
 *   - viennashe::solvers::solve(sparse_matrix<double>&, std::vector<double> const&,
 *     linear_solver_config const&) with config.id() == gpu_parallel_linear_solver
 *       src/solver.cpp:34-38, dispatched at src/solvers/solve.hpp:68-86, slot
 *       reserved at viennashe/solvers/config.hpp:46 / viennashe/forwards.h:215-216
 *       -> vshe_solve_csr / vshe_system_*
 *   - viennashe::she::assemble(...)   viennashe/she/assemble_all.hpp:46-424
 *   - viennashe::she::solve(...)      viennashe/she/linear_solver.hpp:100-189
 *       -> vshe_she_*
 *   - error codes: libviennashe/include/error.h:25-31 (int codes, 0 = success)
 */
#ifndef VSHE_GPU_H
#define VSHE_GPU_H

#include "vshe_types.h"

#ifdef __cplusplus
extern "C" {
#endif

/* ---- error codes (0 = success, as viennasheErrorCode) ---- */
#define VSHE_OK                   0
#define VSHE_E_INVALID_ARGUMENT  -1   /* bad size, null pointer, bad option */
#define VSHE_E_EMPTY_ROW         -2   /* src/solvers/solve.hpp:54-58 (matrix_consistency_check) */
#define VSHE_E_NAN               -3   /* NaN/Inf in rhs or matrix (util/checks.hpp:111-130) */
#define VSHE_E_ODD_DIAGONAL      -4   /* non-positive S^oo diagonal (she/eliminate.hpp:265-270) */
#define VSHE_E_BREAKDOWN         -5   /* BiCGStab breakdown (rho or (r^,v) == 0) */
#define VSHE_E_NOT_CONVERGED     -6   /* iteration limit reached above tolerance */
#define VSHE_E_OUT_OF_MEMORY     -7   /* device allocation failed */
#define VSHE_E_BUDGET            -8   /* request exceeds the context's HBM budget */
#define VSHE_E_CUDA              -9   /* CUDA runtime error */
#define VSHE_E_TIMEOUT          -10   /* a device-side wait ran out of iterations */
#define VSHE_E_ZERO_PIVOT       -11   /* zero pivot in the incomplete factorisation */
#define VSHE_E_NOT_FOUND        -12   /* unknown handle */
#define VSHE_E_UNSUPPORTED      -13   /* option not available in this build */
#define VSHE_E_CAPACITY         -14   /* size beyond a fixed capacity (vshe_csr_residual_noalloc) */

/* ---- solver options ---- */
#define VSHE_PRECISION_FP64   0   /* FP64 BiCGStab, FP64 ILU(0) factors and triangular solves */
#define VSHE_PRECISION_MIXED  1   /* FP64 BiCGStab (SpMV, dots, updates), ILU(0) factors stored in
                                     FP32 and read into FP64 triangular solves; convergence on the
                                     true FP64 residual */

#define VSHE_PRECOND_NONE        0
#define VSHE_PRECOND_ILU0        1   /* ILU(0) on the whole system (serial_linear_solver's choice) */
#define VSHE_PRECOND_BLOCK_ILU0  2   /* ILU(0) per block (energy slabs: block_preconditioner_boundaries) */
#define VSHE_PRECOND_ILUT        3   /* ILUT(ilut_entries, ilut_drop) (Saad Alg. 10.6): the host finds, from the
                                        values at system creation, every position whose entry passes the drop
                                        tolerance; the factorisation of every solve runs on the device inside
                                        that pattern with ILUT's two dropping rules (multipliers and entries
                                        below tol * ||a_i||, then the ilut_entries largest of L and of U).
                                        With n_blocks / block_ptr the factorisation stays inside the blocks
                                        (energy slabs): no elimination with, and no fill from, rows of other
                                        blocks; tol * ||a_i|| uses the whole row */

#define VSHE_ORDER_NATURAL     0   /* the caller's row order (the reference's) */
#define VSHE_ORDER_MULTICOLOR  1   /* greedy colouring of the matrix graph, rows grouped by colour */

#define VSHE_SHADOW_DENSE     0   /* fixed dense pseudo-random r^ in [0.5, 1.5) */
#define VSHE_SHADOW_R0        1   /* r^ = r_0 */

#define VSHE_TRSV_AUTO        0
#define VSHE_TRSV_PERSISTENT  1   /* one cooperative launch per triangular solve, grid barrier per level */
#define VSHE_TRSV_PER_LEVEL   2   /* one launch per level */
#define VSHE_TRSV_PER_SYSTEM  3   /* one CTA per system walks the system's levels (CTA barrier per level,
                                     factor slices staged through shared memory); AUTO picks it for
                                     systems with many short levels (1D devices) */
#define VSHE_TRSV_FLOW        4   /* one cooperative launch per triangular solve without level barriers:
                                     each row polls the rows it reads; same results, measured 2-3x
                                     slower than VSHE_TRSV_PERSISTENT, so AUTO never picks it */
#define VSHE_TRSV_PER_BLOCK   5   /* one CTA per preconditioner block (energy slab of BLOCK_ILU0) walks
                                     the block's levels with a CTA barrier per level, the factor slices
                                     staged through shared memory by bulk copies; AUTO picks it for
                                     block-ILU systems with at least two blocks of at most 2^18 rows */

typedef struct vshe_solve_opts {
  int32_t precision;        /* VSHE_PRECISION_* */
  int32_t precond;          /* VSHE_PRECOND_* */
  int32_t ordering;         /* VSHE_ORDER_* */
  double  tol;              /* FP64 relative residual ||b - A x|| / ||b|| to reach (e.g. 1e-10) */
  int32_t max_iters;        /* cap on BiCGStab iterations (all refinement sweeps together) */
  double  inner_tol;        /* reserved */
  int32_t max_refinements;  /* reserved */
  int64_t n_blocks;         /* BLOCK_ILU0: number of blocks; 0 = one block per ... see block_ptr */
  const int64_t *block_ptr; /* n_blocks + 1 row offsets (block_preconditioner_boundaries) */
  int32_t trsv_mode;        /* VSHE_TRSV_* */
  int32_t check_every;      /* iterations between host-side convergence checks (0 = default 8) */
  const int32_t *perm;      /* optional symmetric permutation for the preconditioner: perm[i] is the
                               original row placed at position i (overrides ordering); NULL = none */
  int32_t shadow;           /* BiCGStab shadow residual: VSHE_SHADOW_DENSE (default) or
                               VSHE_SHADOW_R0 (r^ = r_0, as the reference's ViennaCL bicgstab) */
  int32_t fill_level;       /* ILU0 / BLOCK_ILU0: 0 = ILU(0); k > 0 = ILU(k), the factor keeps the fill
                               of levels <= k (Saad Alg. 10.5), inside the row's block */
  int32_t ilut_entries;     /* ILUT: largest entries kept per row in L and in U (linear_solver_config::
                               ilut_entries(); 0 = its default 60, viennashe/solvers/config.hpp:63) */
  double  ilut_drop;        /* ILUT: relative drop tolerance (ilut_drop_tolerance(); 0 = its default 1e-4) */
} vshe_solve_opts;

typedef struct vshe_solve_stats {
  int32_t status;           /* VSHE_OK or an error code */
  int32_t iterations;       /* BiCGStab iterations (all sweeps) */
  int32_t refinements;      /* residual replacements: restarts from r = b - A x (FP64) after the
                               recursive residual met tol but the true one did not */
  double  rel_residual;     /* final FP64 ||b - A x|| / ||b|| */
  double  setup_ms;         /* factorisation time (device) */
  double  solve_ms;         /* Krylov time incl. residual checks (device) */
  int32_t levels_L;         /* level-schedule depth of the L and U solves */
  int32_t levels_U;
  int64_t bytes_device;     /* device memory held by the system */
  int32_t sweep_ctas;       /* CTAs of the grid-wide triangular sweep (autotuned; 0 = none); for a
                               member swept per task, the CTAs per task (1 = staged single CTA) */
  int32_t tile_rows;        /* rows per reduction tile of this system (autotuned) */
  int32_t sweep_mode;       /* grid-wide sweep used: VSHE_TRSV_PERSISTENT, _PER_LEVEL or _FLOW (0 = none) */
} vshe_solve_stats;

/* Fills opts with the defaults: mixed precision, ILU0, natural order, tol 1e-10,
 * max_iters 1000, persistent triangular solves. */
void vshe_default_opts(vshe_solve_opts *opts);

/* ---- context ---- */
typedef struct vshe_ctx vshe_ctx;

/* Creates a context on CUDA device `device`; hbm_budget_bytes = 0 means 150 GB. */
int vshe_create(vshe_ctx **ctx, int device, size_t hbm_budget_bytes);
int vshe_destroy(vshe_ctx *ctx);
const char *vshe_errstr(int code);
const char *vshe_last_error(vshe_ctx *ctx);
/* Bytes of device memory currently held by the context's systems and SHE problems. */
size_t vshe_bytes_in_use(vshe_ctx *ctx);
/* Per-kernel-class device timing (CUDA events around every launch of the next
 * solves; off by default).  vshe_get_profile returns, for the last solve, ms spent
 * in [0] SpMV, [1] triangular solves, [2] vector updates, [3] unused (0),
 * [4] factorisation, and counts[0] SpMV launches, counts[1] triangular-solve launches. */
int vshe_set_profiling(vshe_ctx *ctx, int32_t on);
/* Polls every bounded device-side wait of this context's solves makes (grid barriers, the flow
 * sweep's polls, the staged sweep's copy barriers) before it gives up: the solve then returns
 * VSHE_E_TIMEOUT and the context stays usable.  0 restores the default (20,000,000 polls, about
 * 1-2 s).  No reference counterpart: failure handling of the device-side waits. */
int vshe_set_spin_limit(vshe_ctx *ctx, uint64_t polls);
/* Host threads the library uses for its host work (the layout of a pattern: colouring, symbolic
 * ILU(k) per block, levels, pattern conversions; the drop-in call's value checks and pattern
 * comparison), for every context of the process: 0 (default) up to 16, limited by the cores.
 * Every choice gives the same layout and results.  No reference counterpart. */
int vshe_set_host_threads(int32_t threads);
/* Sweep kernel of the members swept one task per CTA or cluster (VSHE_TRSV_PER_BLOCK,
 * VSHE_TRSV_PER_SYSTEM and their AUTO cases): -1 (default) times the candidates on each batch's
 * own factors before its first iteration and keeps the fastest; 0 one CTA per task with the
 * factor slices staged through shared memory by bulk copies; 2, 4 or 8 one thread-block cluster
 * of that many CTAs per task with a cluster barrier per level.  Every choice gives bitwise the same
 * results.  No reference counterpart: scheduling control of the triangular sweeps. */
int vshe_set_task_sweep(vshe_ctx *ctx, int32_t kernel);
int vshe_get_profile(vshe_ctx *ctx, double *ms, int64_t *counts);
/* Autotuner record: the rows per reduction tile chosen for systems of n's size class
 * (floor(log2 n)) on this context, and ms[0..3] = the timed FP64 SpMV for 512, 1024, 2048 and
 * 4096-row tiles.  VSHE_E_NOT_FOUND until a system of that class was solved.  No reference
 * counterpart: instrumentation of the tile autotuner. */
int vshe_autotune_info(vshe_ctx *ctx, int64_t n, int64_t *tile_rows, double *ms);
/* Number of this library's own kernel launches in the process so far (all
 * contexts; library kernels such as CUB scans are not counted).  No reference
 * counterpart: instrumentation. */
int64_t vshe_kernel_launches(void);

/* ---- drop-in linear solve: viennashe::solvers::solve(A, b, config), gpu slot ----
 * A is n x n CSR (int64 row offsets, int32 column indices ascending per row,
 * FP64 values), rhs and x are host arrays of length n.  Checks, in the
 * reference's order (src/solvers/solve.hpp:54-66): empty rows -> VSHE_E_EMPTY_ROW,
 * non-finite rhs -> VSHE_E_NAN, ||rhs|| == 0 -> x = 0.  Host buffers are copied
 * in and out inside the call.  The context keeps the system of the last call resident (its
 * solver order, schedules and device buffers; counted in vshe_bytes_in_use): a following call
 * with the same row offsets, columns and options (a Gummel loop's next step) uploads only the
 * values and rhs.  Not kept for VSHE_PRECOND_ILUT, whose pattern depends on the values.
 * vshe_solve_csr_release frees the kept system (vshe_destroy does too). */
int vshe_solve_csr(vshe_ctx *ctx, int64_t n, int64_t nnz, const int64_t *row_ptr, const int32_t *col,
                   const double *val, const double *rhs, const vshe_solve_opts *opts, double *x,
                   vshe_solve_stats *stats);
int vshe_solve_csr_release(vshe_ctx *ctx);

/* ---- resident systems: upload once, refactor/solve many times ----
 * vshe_system_create copies the CSR (host) to the device and builds the
 * preconditioner's schedule for `opts`.  The pattern is fixed for the life of
 * the handle; vshe_system_set_values replaces values and rhs (host arrays). */
int vshe_system_create(vshe_ctx *ctx, int64_t n, int64_t nnz, const int64_t *row_ptr, const int32_t *col,
                       const double *val, const double *rhs, const vshe_solve_opts *opts, int64_t *handle);
int vshe_system_set_values(vshe_ctx *ctx, int64_t handle, const double *val, const double *rhs);
/* Factorises and solves on the device; x (host, may be NULL) receives the solution. */
int vshe_system_solve(vshe_ctx *ctx, int64_t handle, double *x, vshe_solve_stats *stats);
/* Solves several resident systems together (one batched pass; per-system
 * Krylov scalars, so each result equals the one it would get alone). */
int vshe_batch_solve(vshe_ctx *ctx, int32_t count, const int64_t *handles, vshe_solve_stats *stats);
int vshe_system_get_x(vshe_ctx *ctx, int64_t handle, double *x);
int vshe_system_free(vshe_ctx *ctx, int64_t handle);

/* Kernel-level entry points on a resident system (used by parity tests and
 * the bench): y = A x, host x/y of length n (precision must be VSHE_PRECISION_FP64: the
 * SpMV is FP64 in every solver mode); the incomplete factor values in A's pattern (FP64,
 * host array of length nnz). */
int vshe_system_spmv(vshe_ctx *ctx, int64_t handle, int32_t precision, const double *x, double *y);
int vshe_system_factor_values(vshe_ctx *ctx, int64_t handle, double *lu);
/* Device-timed kernel throughput on a resident system: runs `reps` SpMVs in the
 * given precision (FP64 only) and returns the mean time per SpMV (ms) from CUDA events. */
int vshe_system_time_spmv(vshe_ctx *ctx, int64_t handle, int32_t precision, int32_t reps, double *ms);

/* ---- residual without device allocation ----
 * No counterpart in the reference: an entry point for callers that cannot call cudaMalloc,
 * because another component (a framework's caching allocator, a fixed arena) owns all device
 * memory, or because the call sits in a loop where cudaMalloc/cudaFree would synchronise the
 * device.  Computes r = b - A x and norms2[0] = ||r||^2, norms2[1] = ||b||^2 for an n x n CSR
 * matrix (int64 row offsets, int32 columns, FP64 values); every pointer is a caller-owned
 * DEVICE buffer (d_r of n doubles, d_norms2 of 2) on the current CUDA device.  The kernel is
 * queued on `stream` (a cudaStream_t; NULL = the default stream) and the call returns without
 * waiting.  Its scratch (one partial-sum pair per 2048 rows) is a fixed 512 KiB array in the
 * library's device image, so n is limited to 64 Mi rows (67,108,864): larger n returns
 * VSHE_E_CAPACITY.  The first call on each device looks up that array's address and clears its
 * ticket counter, so it synchronises the device once and should come before any stream capture.  All calls share
 * the array: calls whose kernels overlap on the GPU (other streams or threads on the same
 * device) race on it.  Nothing is allocated or freed by this call. */
int vshe_csr_residual_noalloc(int64_t n, int64_t nnz, const int64_t *d_row_ptr, const int32_t *d_col,
                              const double *d_val, const double *d_x, const double *d_b, double *d_r,
                              double *d_norms2, void *stream);

/* ---- host-only layout inspection (no GPU needed) ----
 * The solver order and the SELL-32 tables a resident system built from (A, opts) uses, for
 * tests of the ordering and layout logic (val: the values, read for VSHE_PRECOND_ILUT only, else
 * may be NULL).  No reference counterpart: the reference's
 * ViennaCL solvers keep the caller's CSR.  The solver order q = 0..n-1 lists the caller's rows
 * (perm[q]) sorted by forward-sweep level; forward level k is rows [lvr[k], lvr[k+1]).  A
 * SELL-32 slice j spans slots [off[j], off[j+1]) = 32 x width; entry k of the slice's row
 * `lane` sits in slot off[j] + 32 k + lane.  Columns are solver-order rows; padding slots point
 * at column n and map to entry -1.  vshe_layout_sizes fills sizes[0..9] = slices_A, slots_A,
 * slices_L, slots_L, slices_U, slots_U, levels_L, levels_U, nnz_L, nnz_U.  vshe_layout_export
 * fills caller arrays of those sizes (any pointer may be NULL): perm[n], lvr[levels_L + 1],
 * aoff[slices_A + 1], acol / amap_a[slots_A] (caller entry index of each slot), lrow0 /
 * loff[slices_L + 1] (first solver row / slot offset of each L slice, plus the end), lcol /
 * lmap[slots_L], uslot0 / uoff[slices_U + 1], ucol / umap[slots_U], urow[n] (solver row of each
 * backward-sweep slot). */
int vshe_layout_sizes(int64_t n, int64_t nnz, const int64_t *row_ptr, const int32_t *col, const double *val,
                      const vshe_solve_opts *opts, int64_t *sizes);
int vshe_layout_export(int64_t n, int64_t nnz, const int64_t *row_ptr, const int32_t *col, const double *val,
                       const vshe_solve_opts *opts,
                       int32_t *perm, int64_t *lvr, int64_t *aoff, int32_t *acol, int64_t *amap_a,
                       int32_t *lrow0, int64_t *loff, int32_t *lcol, int64_t *lmap,
                       int32_t *uslot0, int64_t *uoff, int32_t *ucol, int64_t *umap, int32_t *urow);
/* The sweep plan of that system alone, as a batch of one on a device of num_sms SMs (0: 148):
 * - counts[0..3]: tasks, chunks, slice descriptors, and the system's sweep (0 grid-wide, 1 one
 *   task for the system, 2 tasks of preconditioner blocks).
 * - tasks[6 t ..]: system, first and end chunk of the forward sweep, first and end chunk of the
 *   backward sweep, 0.
 * - chunks[10 c ..]: first and end slice, flags (1: last chunk of its level, 2: read from global
 *   memory), factor slots, first slot, first slice descriptor, first and end row operand, the
 *   consumer rotation, and the bytes the chunk occupies in a 64 KiB shared-memory stage.
 * - sdesc[4 d ..]: slot offset in the chunk, width, first row (L) or slot (U), and rows.
 * Call once with NULL arrays for the counts, then with arrays of those sizes.  Host only; this
 * is the plan the task sweeps (k_trsv_task) stage from, so tests check the stage bounds on it. */
int vshe_layout_sweep_plan(int64_t n, int64_t nnz, const int64_t *row_ptr, const int32_t *col, const double *val,
                           const vshe_solve_opts *opts, int32_t num_sms, int64_t *counts, int32_t *tasks,
                           int64_t *chunks, int32_t *sdesc);

/* ---- SHE path on the device: she::assemble + she::solve (secondary boundary) ----
 * vshe_she_create runs the host setup of the (x, H) space (energies, expansion
 * orders, unknown mapping, boundary values: viennashe/she/setup_energies.hpp:61-153,
 * expansion_order.hpp:262-364, mapping.hpp:97-393, boundary_conditions.hpp:57-134),
 * then builds the patterns of the full and the reduced system on the device and
 * the preconditioner schedule for `opts` (BLOCK_ILU0 with no block_ptr uses one
 * block per energy slab, as fill_block_indices, linear_solver.hpp:44-83).
 * `coupling` carries the spherical-harmonics coupling tables a_{x,y,z}, b_{x,y,z}
 * of order cfg->max_expansion_order (fill_coupling_matrices,
 * viennashe/she/harmonics_coupling.hpp:1050-1073); vshe_coupling_tables_compute
 * fills them by quadrature when the caller has none. */
typedef struct vshe_she_info {
  int32_t n_energies;       /* N_H */
  int64_t n_even, n_odd;    /* unknowns (even = reduced system size) */
  int64_t nnz_full, nnz_reduced;
  int32_t n_cells, n_facets, n_contacts;
  double  hbar_omega;       /* optical phonon energy snapped to the grid, J */
  int64_t bytes_device;
  int32_t levels_L, levels_U;
  int64_t nnz_factor;       /* strict lower + upper entries the ILU(0) preconditioner keeps */
  int64_t bytes_estimate;   /* the upper bound of bytes_device computed from the host set-up alone, which
                               vshe_she_create and the server compare with the HBM budget before allocating */
} vshe_she_info;

/* 6 * ((L+1)^2)^2 doubles, layout of vshe_coupling_tables.data; no GPU needed. */
int vshe_coupling_tables_compute(int32_t L, double *out);
/* The host set-up of a SHE problem alone, no GPU needed (capacity planning before a request is
 * submitted): fills n_energies, n_even, n_odd, n_cells, n_facets, n_contacts, hbar_omega and
 * bytes_estimate (the footprint bound vshe_she_create and the server admit by) of *info, the
 * other fields 0.  opts may be NULL (the defaults). */
int vshe_she_plan(const vshe_device_desc *dev, const vshe_she_config *cfg, const vshe_coupling_tables *coupling,
                  const vshe_solve_opts *opts, vshe_she_info *info);
/* The (x, H) space of the same set-up, no GPU needed, so that a caller can read the unknowns of
 * x_full (vshe_she_results) per cell and energy -- the quantity the reference's distribution
 * function wrappers look up (viennashe/she/df_wrappers.hpp:45-90, 230-260): the N_H total
 * energies (J); per cell and energy, at [cell * N_H + H], the index in x_full of the node's first
 * even unknown (-1: no unknown there; the node's harmonics follow in the order of
 * spherical_harmonics.hpp:213-252), its expansion order, the kinetic energy H - E_c(cell) (J) and
 * the density of states there (Modena dispersion, viennashe/physics/dispersion.hpp:207-286); per
 * facet and energy, at [facet * N_H + H], the first odd unknown's index and the order.  Sizes are
 * vshe_she_plan's n_energies, n_cells and n_facets.  Any output pointer may be NULL. */
int vshe_she_space(const vshe_device_desc *dev, const vshe_she_config *cfg, const vshe_coupling_tables *coupling,
                   double *energies, int64_t *even_index, int32_t *even_order, double *kinetic_energy,
                   double *density_of_states, int64_t *odd_index, int32_t *odd_order);
/* The multicolour order of the reduced rows that vshe_she_create uses when opts->ordering is
 * VSHE_ORDER_MULTICOLOR and opts->perm is NULL, no GPU needed: every (cell, H) node takes a colour,
 * and all harmonics of a node share it.  The cell part is a greedy colouring of the mesh graph (at
 * distance 2 for fill_level > 0).  The energy part is H / n_op in 2 classes (3 for fill_level >
 * 0), since in-scattering couples H with H +- n_op.  perm[t] is the reduced row at position t, by
 * colour and then by row; colour[row] is each row's colour.  Both hold n_even entries
 * (vshe_she_plan); either may be NULL. */
int vshe_she_node_order(const vshe_device_desc *dev, const vshe_she_config *cfg, const vshe_coupling_tables *coupling,
                        int32_t fill_level, int32_t *perm, int32_t *colour);
int vshe_she_create(vshe_ctx *ctx, const vshe_device_desc *dev, const vshe_she_config *cfg,
                    const vshe_coupling_tables *coupling, const vshe_solve_opts *opts, int64_t *handle);
int vshe_she_info_get(vshe_ctx *ctx, int64_t handle, vshe_she_info *info);
/* Device assembly with the current potential-independent tables: upto = 1 assembles the
 * full even+odd system (assemble_all.hpp:46-424), 2 also eliminates the odd unknowns
 * (eliminate.hpp:80-293), 3 also scales and normalises (rescaling.hpp:50-107,
 * linalg_util.hpp:202-282) -- the state vshe_she_solve needs. */
int vshe_she_assemble(vshe_ctx *ctx, int64_t handle, int32_t upto);
/* ILU(0)/BiCGStab (FP64 or mixed) on the reduced system, on the device. */
int vshe_she_solve(vshe_ctx *ctx, int64_t handle, vshe_solve_stats *stats);
/* Unscale, recover the odd unknowns, full-system residual (linear_solver.hpp:172-186,
 * eliminate.hpp:305-354), carrier density per cell and terminal current per contact
 * (carrier_density.hpp:68-130, terminal_current.hpp:47-105), on the device. */
int vshe_she_finish(vshe_ctx *ctx, int64_t handle, double *full_residual);
/* assemble(3) + solve + finish. */
int vshe_she_run(vshe_ctx *ctx, int64_t handle, vshe_solve_stats *stats, double *full_residual);
/* Device-timed throughput of vshe_she_run: `warmup` untimed runs, then `steps` runs each
 * bracketed by a device synchronisation and timed with CUDA events on the library's
 * stream; step_ms[k] receives the duration of run k, *last the stats of the last run. */
int vshe_she_bench(vshe_ctx *ctx, int64_t handle, int32_t warmup, int32_t steps, double *step_ms, vshe_solve_stats *last);
/* Bias sweep / many devices in one solve: assembles every problem, solves all reduced
 * systems as one batch (shared launches; each system's iterates are the same as when it is
 * solved alone) and finishes each.  The problems must share precision and preconditioner
 * kind.  stats[k] and full_residuals[k] (either may be NULL) belong to handles[k];
 * *device_ms (may be NULL) receives the CUDA-event time of the whole call on the library's
 * stream.  The batch schedule is built on first use of a handle set and reused.  The
 * reference solves such sweeps one system at a time (simulator::run per bias point). */
int vshe_she_run_batch(vshe_ctx *ctx, int32_t count, const int64_t *handles, vshe_solve_stats *stats,
                       double *full_residuals, double *device_ms);
/* Host copies of the results (any pointer may be NULL): x_full (n_even + n_odd),
 * density (n_cells), currents (n_contacts). */
int vshe_she_results(vshe_ctx *ctx, int64_t handle, double *x_full, double *density, double *currents);
/* Host copy of the current full (which = 0) or reduced (which = 1) system, CSR + rhs. */
int vshe_she_export(vshe_ctx *ctx, int64_t handle, int32_t which, int64_t *row_ptr, int32_t *col, double *val, double *rhs);
/* Unknown scaling s and column scale factors of the reduced system (length n_even). */
int vshe_she_scaling(vshe_ctx *ctx, int64_t handle, double *scaling, double *scale_factors);
/* Energy-slab row blocks of the reduced system (n_energies + 1 row offsets; slab H = rows
 * [block_ptr[H], block_ptr[H+1]), empty for the end slabs): what fill_block_indices
 * (viennashe/she/linear_solver.hpp:44-83) puts into linear_solver_config::block_preconditioner_boundaries(). */
int vshe_she_blocks(vshe_ctx *ctx, int64_t handle, int64_t *block_ptr);
int vshe_she_free(vshe_ctx *ctx, int64_t handle);

/* ---- served stream: continuous batching of SHE solves ----
 * No reference counterpart: the reference solves one device at a time (simulator::run).  A
 * server owns a worker thread that admits submitted requests in arrival order while the device
 * memory of its resident problems stays within hbm_budget and at most max_active are resident
 * (with problems resident, a quarter second of set-up per scheduling step at most, and the host
 * layout of a request of 262,144 or more reduced unknowns on a thread of its own, so that the
 * residents keep iterating while a long queue is set up), iterates all resident problems together (one batch, chunks of check_every iterations), and
 * retires each one as soon as it converges, its place taken by the next request.  A served
 * result equals the result of the same request solved alone (per-system reductions in a fixed
 * order).  The server makes its GPU calls on ctx under ctx's lock; other calls on the same
 * context interleave with it step by step.  Every request shares the precision and the
 * preconditioner kind of opts->solve (and its tol, max_iters, check_every); the ordering and
 * the preconditioner variant may differ per request. */
typedef struct vshe_server vshe_server;
typedef struct vshe_server_opts {
  size_t  hbm_budget;       /* bytes the resident problems may hold (0: the context's budget) */
  int32_t max_active;       /* resident problems at most (0: 256) */
  vshe_solve_opts solve;    /* default solver options of a request */
  int32_t stagnation_iters; /* a request whose recursive residual has not halved within this many
                               iterations ends early with VSHE_E_NOT_CONVERGED, freeing its slot
                               (0: 400; negative: never, only max_iters ends it) */
} vshe_server_opts;
typedef struct vshe_server_result {
  int32_t status;           /* VSHE_OK or the error of this request */
  int32_t iterations;
  int32_t refinements;      /* residual replacements */
  double  rel_residual;     /* FP64 relative residual of the reduced system */
  double  full_residual;    /* relative residual of the full (even + odd) system */
  double  queue_ms;         /* submission -> admission (host clock) */
  double  latency_ms;       /* submission -> result ready (host clock) */
  int64_t n_unknowns;       /* reduced-system size */
} vshe_server_result;

int vshe_server_create(vshe_ctx *ctx, const vshe_server_opts *opts, vshe_server **server);
/* Queues one solve: the arrays of dev, cfg and coupling are copied, so they may be released
 * on return.  opts may be NULL (the server's defaults).  *ticket identifies the request. */
int vshe_server_submit(vshe_server *server, const vshe_device_desc *dev, const vshe_she_config *cfg,
                       const vshe_coupling_tables *coupling, const vshe_solve_opts *opts, int64_t *ticket);
/* Waits for a request (timeout_ms < 0: without limit; VSHE_E_TIMEOUT if it is not done in
 * time) and copies its result, densities (n_cells) and terminal currents (one per contact);
 * any pointer may be NULL.  Returns the request's status and forgets the ticket. */
int vshe_server_wait(vshe_server *server, int64_t ticket, double timeout_ms, vshe_server_result *result,
                     double *density, double *currents);
/* Finishes the resident requests, drops the queued ones and joins the worker. */
int vshe_server_destroy(vshe_server *server);

/* ---- outer loop: Gummel update of the electrostatic potential ----
 * One spatial step of the reference's Gummel iteration (viennashe/simulator.hpp:1029-1052) on
 * the device: the linearised Poisson system of viennashe/assemble.hpp:165-345 (finite volumes
 * on the cell mesh, harmonic-mean permittivity across facets, homogeneous Neumann at the domain
 * boundary, Dirichlet at contact cells with the description's potential there, the Gummel term
 * q (n + p) / V_T on the diagonal of semiconductor cells, the charge q (n - N_D - p + N_A) in the
 * rhs; no fixed or trapped charge), solved for the update in FP64, then the damped update of
 * simulator.hpp:606-647: psi <- (1 - alpha) psi + alpha (psi + dpsi) (contact cells keep their
 * value).  The unknowns are the non-contact cells, in cell order.  Every cell that is not a
 * contact needs a non-metal material.  facet_centroid (n_facets * dim) gives the facet centres
 * the permittivity mean weights by (viennagrid::centroid of the facet in the reference). */
typedef struct vshe_poisson_stats {
  int32_t status;            /* of the linear solve */
  int32_t iterations;
  double  rel_residual;      /* of the linear solve */
  double  rhs_norm;          /* ||b||_2: the reference's current_residual_norm term */
  double  update_norm;       /* ||dpsi||_2: the reference's potential_norm_increment */
  int64_t n_unknowns;
} vshe_poisson_stats;
/* opts: FP64 solver options (NULL: ILU(0) in natural order, tol 1e-12, 10000 iterations;
 * the precision is always FP64). */
int vshe_poisson_create(vshe_ctx *ctx, const vshe_device_desc *dev, const double *facet_centroid,
                        const vshe_solve_opts *opts, int64_t *handle);
/* potential (n_cells, host) is the current iterate; n and p (n_cells, host, m^-3) the carrier
 * densities; the damped new potential goes to potential_out (n_cells, host; may alias
 * potential).  damping in (0, 1]. */
int vshe_poisson_update(vshe_ctx *ctx, int64_t handle, const double *potential, const double *n, const double *p,
                        double damping, double *potential_out, vshe_poisson_stats *stats);
/* The last assembled system: row offsets (n_unknowns + 1), columns and values (nnz), rhs
 * (n_unknowns); NULL pointers are skipped; *nnz receives the entry count. */
int vshe_poisson_export(vshe_ctx *ctx, int64_t handle, int64_t *row_ptr, int32_t *col, double *val, double *rhs,
                        int64_t *nnz);
int vshe_poisson_free(vshe_ctx *ctx, int64_t handle);

/* The self-consistent electron SHE + Poisson Gummel loop of simulator::run
 * (viennashe/simulator.hpp:895-1130, electrons only, the SHE equation for electrons): each
 * iteration takes the Gummel update of the potential for the current electron and hole
 * densities (vshe_poisson_update), then solves the SHE for the new potential on the device
 * (vshe_she_create / _run / _results) and updates the electron density with logarithmic damping,
 * n <- n^(1 - alpha) n_SHE^alpha with n_SHE >= 1e-10 n (simulator.hpp:560-577).  The holes stay
 * at their initial density (hole equation off).  The loop ends, as the reference's does, after
 * one more undamped update once the Poisson rhs norm has fallen below 1e-10 of its first value
 * or the potential increment below tol, or at max_iters (the last iteration undamped).  The SHE
 * rhs is not part of the residual norm here (the reference adds ||b_SHE||).  Each iteration
 * builds the SHE problem for its potential on the host (energies, orders, mapping). */
typedef struct vshe_gummel_opts {
  int32_t max_iters;   /* the reference's default 100 (solvers/config.hpp:256-257) */
  double  tol;         /* on ||dpsi||_2, default 1e-8 */
  double  damping;     /* default 0.3 */
} vshe_gummel_opts;
typedef struct vshe_gummel_stats {
  int32_t status;
  int32_t iterations;          /* Gummel iterations done */
  double  potential_increment; /* ||dpsi||_2 of the last iteration */
  double  rhs_norm;            /* ||b_Poisson||_2 of the last iteration */
  double  initial_rhs_norm;    /* ... of the first */
  int64_t she_iterations;      /* BiCGStab iterations over all SHE solves */
} vshe_gummel_stats;
/* density0 / p0: initial electron and hole densities (n_cells, m^-3).  The potential starts at
 * the description's.  Outputs (n_cells / one per contact, host, may be NULL): the final
 * potential, electron density and terminal currents of the last SHE solve.  history, if not NULL,
 * receives per iteration (||b_Poisson||, ||dpsi||, SHE iterations), 3 * max_iters doubles. */
int vshe_gummel_solve(vshe_ctx *ctx, const vshe_device_desc *dev, const double *facet_centroid, const vshe_she_config *cfg,
                      const vshe_coupling_tables *coupling, const vshe_solve_opts *she_opts, const vshe_gummel_opts *gopts,
                      const double *density0, const double *p0, double *potential_out, double *density_out,
                      double *currents_out, double *history, vshe_gummel_stats *stats);

#ifdef __cplusplus
}
#endif

#endif /* VSHE_GPU_H */

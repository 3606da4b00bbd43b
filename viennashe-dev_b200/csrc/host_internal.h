// host_internal.h -- C++ host objects of the solver backend (not part of the C ABI).
#pragma once
#include <cstdint>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/vshe_gpu.h"
#include "kernels.h"
#include "solver_kernels.cuh"

namespace vshe {

const char *errstr(int code);

// polls of a device-side wait before it gives up with VSHE_E_TIMEOUT (about 1-2 s with backoff)
constexpr unsigned long long kDefaultSpinLimit = 20000000ull;
// Entries allocated past n in the Krylov vectors and in urow / udinv: the per-task sweep stages
// row ranges rounded up to a multiple of 4 entries, which may reach up to 3 entries past n.
constexpr int64_t kVecPad = 8;

// Device allocations owned by one object, freed together.
struct DevArena {
  std::vector<void *> ptrs;
  size_t total = 0;
  void *alloc(size_t bytes, cudaError_t &e);
  void release();
  ~DevArena() { release(); }
};

struct Ctx;

// Host-side solver layout of one system (no CUDA): the solver order, the solver-order CSR used
// by the factorisation, and the SELL-32 tables of A, L and U (solver_kernels.cuh).
struct Layout {
  std::vector<int32_t> perm, blk;
  std::vector<int64_t> lvr, lvsL, lvsU;
  int32_t nlevL = 0, nlevU = 0;
  int64_t nslA = 0, nslL = 0, nslU = 0, padA = 0, padL = 0, padU = 0, nnzL = 0, nnzU = 0;
  int64_t nnzF = 0;                      // entries of the factor pattern (A's + ILU(k) fill)
  std::vector<int64_t> prp, pdiag, amap;
  std::vector<int32_t> pci;
  std::vector<int64_t> aoff, astart, amapS;
  std::vector<int32_t> acol;
  std::vector<int64_t> fmap, dpos, loff, uoff, lstart, ustart;
  std::vector<int32_t> lcol, ucol, urow;
  // (level, block) groups of the L and U slices: group g = slices [grp_s0[g], grp_s0[g+1]) of
  // level grp_lev[g] and preconditioner block grp_blk[g], ordered by level, then block
  std::vector<int64_t> lgrp_s0, ugrp_s0;
  std::vector<int32_t> lgrp_lev, lgrp_blk, ugrp_lev, ugrp_blk;
  // values (caller order, host) are read only for the ILUT pattern and may be NULL otherwise
  int build(int64_t n, int64_t nnz, const std::vector<int64_t> &rp, const std::vector<int32_t> &ci,
            const vshe_solve_opts &opts, const double *values, std::string &err);
};

// One resident linear system.  The caller's CSR (and rhs) stay in the caller's order; the
// solver works in a level-sorted solver order (perm[q] = caller row of solver row q) on
// SELL-32 copies of A and of the incomplete factors (solver_kernels.cuh).
struct System {
  int64_t n = 0, nnz = 0;
  vshe_solve_opts opts{};
  bool mixed = true;     // FP32-stored ILU(0) factors (Krylov and triangular-solve arithmetic in FP64 either way)
  bool borrowed = false;  // A and b live in the caller's device memory
  bool has_pc = true;
  double bnorm_host = 0.0;
  // host: pattern and schedules
  std::vector<int64_t> rp;
  std::vector<int32_t> ci;
  std::vector<int32_t> perm, blk;       // perm[q] = caller row of solver row q; blk in solver order
  std::vector<int64_t> lvr;             // forward level k = solver rows [lvr[k], lvr[k+1])
  std::vector<int64_t> lvsL, lvsU;      // forward / backward level k = L / U slices [lvs[k], lvs[k+1])
  std::vector<int64_t> lgrp_s0, ugrp_s0;  // (level, block) slice groups (Layout)
  std::vector<int32_t> lgrp_lev, lgrp_blk, ugrp_lev, ugrp_blk;
  std::vector<int64_t> loff_h, uoff_h;    // SELL slot offsets of the L and U slices (host copies)
  std::vector<int64_t> lrow0_h, uslot0_h; // first solver row / slot of every L / U slice (host copies)
  int32_t nlevL = 0, nlevU = 0;
  int64_t nslA = 0, nslL = 0, nslU = 0;     // SELL slices
  int64_t padA = 0, padL = 0, padU = 0;     // SELL slots (incl. padding)
  int64_t nnzL = 0, nnzU = 0;               // factor entries (excl. padding)
  int64_t nnzF = 0;                         // entries of the factor pattern (A's + ILU(k) fill)
  // device
  DevArena arena;
  int64_t *d_rp = nullptr; int32_t *d_ci = nullptr;
  double *d_av64 = nullptr;   // caller-order values
  double *d_b64 = nullptr;    // caller-order rhs
  double *d_x64 = nullptr;    // caller-order solution
  double *d_bp = nullptr;     // solver-order rhs
  int32_t *d_perm = nullptr, *d_blk = nullptr;
  // SELL A (solver order)
  int64_t *d_aoff = nullptr, *d_amapS = nullptr; int32_t *d_acol = nullptr; double *d_aval = nullptr;
  // solver-order CSR for the factorisation
  int64_t *d_prp = nullptr, *d_pdiag = nullptr, *d_amap = nullptr, *d_fmap = nullptr, *d_dpos = nullptr, *d_lvr = nullptr;
  int32_t *d_pci = nullptr;
  double *d_lu64 = nullptr;
  // SELL factors
  int32_t *d_lrow0 = nullptr, *d_uslot0 = nullptr, *d_urow = nullptr, *d_lcol = nullptr, *d_ucol = nullptr;
  int64_t *d_loff = nullptr, *d_uoff = nullptr, *d_lvsL = nullptr, *d_lvsU = nullptr;
  void *d_lval = nullptr, *d_uval = nullptr, *d_udinv = nullptr;
  double *d_ytmp = nullptr;
  void *kv[9] = {nullptr};  // x r rh p v s t ph sh (FP64, solver order, n + kVecPad entries; entry n stays 0)
  int64_t tile_rows = 0;    // rows per reduction tile (0: not chosen yet; see Batch::autotune_tiles)

  int create(Ctx &ctx, int64_t n, int64_t nnz, const int64_t *rp, const int32_t *ci, const double *v,
             const double *rhs, const vshe_solve_opts &o);
  // A system whose CSR and rhs already live on the device (owned by the caller): the host
  // pattern is used for the schedules, values are read from the device at solve time.
  int create_borrowed(Ctx &ctx, int64_t n, int64_t nnz, const int64_t *rp, const int32_t *ci, int64_t *d_rp_,
                      int32_t *d_ci_, double *d_val, double *d_rhs, const vshe_solve_opts &o, const double *host_val = nullptr);
  int set_values(Ctx &ctx, const double *v, const double *rhs);
  int setup_pattern(Ctx &ctx, const double *host_val);  // ordering, schedules, device buffers
  // the two halves of create_borrowed: the host copies of the pattern and the device pointers,
  // and (after Layout::build on those copies, which needs no device) the device buffers
  int init_borrowed(Ctx &ctx, int64_t n, int64_t nnz, const int64_t *rp, const int32_t *ci, int64_t *d_rp_,
                    int32_t *d_ci_, double *d_val, double *d_rhs, const vshe_solve_opts &o);
  int setup_from_layout(Ctx &ctx, const Layout &Lt);
  void adopt_layout(const Layout &Lt);  // the host fields of setup_from_layout, no device work
  // gathers the caller-order values and rhs into the solver-order SELL A, the factorisation
  // CSR and b_p (on the context's stream)
  void prepare(Ctx &ctx);
  void fill_sysdev(void *out) const;
};

// Several systems solved together.
// Sweep plan of a batch: per member 0 (grid-wide sweep), 1 (one task for the system) or 2 (tasks of
// preconditioner blocks); the tasks, the chunks of their levels, the chunks' slice descriptors,
// and the level slice ranges of the cluster sweeps.
struct SweepPlan {
  std::vector<char> on_task;
  std::vector<TaskDev> tasks;
  std::vector<ChunkDev> chunks;
  std::vector<SliceDesc> sdesc;
  std::vector<ClusterTask> ctasks;
  std::vector<int64_t> clv;
  int64_t tune_key_tasks = 0;
  bool has_tune_key = false;
};
void plan_sweep_tasks(const std::vector<System *> &sys, bool mixed, bool has_pc, int64_t num_sms, SweepPlan &plan);

struct Batch {
  std::vector<System *> sys;
  int nsys = 0;
  bool mixed = true, has_pc = true;
  int ntiles = 0;
  int32_t nlevL = 0, nlevU = 0;   // merged levels of the grid-wide sweeps
  int32_t nlevF = 0;              // merged levels of the factorisation (all members)
  int trsv_grid = 148, ilu_grid = 148, num_sms = 148;
  // sweep tasks (k_trsv_task: one CTA per preconditioner block or per system, TaskDev / ChunkDev
  // tables, ordered by decreasing work); members not swept as tasks share the merged level
  // schedule of the grid-wide sweep (grid_group)
  int ntasks = 0;
  std::vector<int32_t> task_kind;  // per member: 0 grid-wide sweep, 1 one task per system, 2 one task per block
  void *d_tasks = nullptr, *d_chunks = nullptr, *d_ctasks = nullptr, *d_sdesc = nullptr;
  int64_t *d_clv = nullptr;
  int task_kernel = 4;                 // 0 staged single CTA per task, K > 0 cluster of K CTAs per task
  bool tasks_tuned = false;
  int64_t tune_key_tasks = -1, tune_key_grid = -1;  // shape classes of the task and grid-wide sweeps
  std::vector<double> task_tune_ms;    // ms per apply: staged, clusters of 2, 4, 8
  int launch_tasks(Ctx &ctx, int which);
  int autotune_tasks(Ctx &ctx);
  bool grid_group = true;
  // the BiCGStab iteration chunk (check_every iterations) captured once as a CUDA graph and
  // replayed; graph_failed: capture was refused (then the chunk is launched directly)
  cudaGraphExec_t chunk_exec = nullptr;
  int chunk_every = 0;
  long long chunk_launches = 0;
  bool graph_failed = false;
  ~Batch() { if (chunk_exec) cudaGraphExecDestroy(chunk_exec); }
  // row tiles: every member's own tile_rows rows per tile, rebuilt by set_tiles
  DevArena tile_arena;
  DevArena arena;
  int32_t *d_tile_sys = nullptr, *d_sys_tile0 = nullptr, *d_active = nullptr, *d_counters = nullptr, *d_err = nullptr;
  int64_t *d_tile_r0 = nullptr, *d_tile_r1 = nullptr;
  double *d_partials = nullptr, *d_rnorm2 = nullptr, *d_bnorm2 = nullptr;
  unsigned *d_bar = nullptr;
  void *d_sysdev = nullptr, *d_state = nullptr, *d_refdev = nullptr, *d_factdev = nullptr;
  // triangular-solve schedules (per level: the (system, slice) entries of every member)
  int64_t *d_cptrL = nullptr, *d_cptrU = nullptr;
  int32_t *d_csL = nullptr, *d_cqL = nullptr, *d_csU = nullptr, *d_cqU = nullptr;
  // factorisation schedule of a multi-system batch (per level: rows of every system)
  int64_t *d_fptr = nullptr;
  int32_t *d_fsys = nullptr, *d_frow = nullptr;
  VkTiles tiles{};
  VkLevels levL{}, levU{}, levF{};
  std::vector<char> last_state;
  // per-kernel-class device time of the last solve (CUDA events), when profiling is on
  bool profile = false;
  double t_spmv = 0, t_trsv = 0, t_vec = 0, t_reliable = 0, t_factor = 0;
  int64_t n_spmv = 0, n_trsv = 0;

  int build(Ctx &ctx, const std::vector<System *> &members);
  unsigned long long bar_limit = 0;  // poll limit last written to d_bar[2..3]
  int sync_spin_limit(Ctx &ctx);
  // only_member >= 0: tiles of that member alone, with `rows` rows (the autotuner's trial tiles)
  int set_tiles(Ctx &ctx, int only_member = -1, int64_t rows = 0);
  int autotune_tiles(Ctx &ctx);
  int autotune_trsv(Ctx &ctx);
  bool trsv_tuned = false;
  int trsv_bps_max = 4;
  std::vector<double> trsv_tune_ms;  // ms per apply for 1, 2, ... CTAs per SM (barrier sweeps, then flow sweeps)
  int trsv_kernel = 1;               // grid-wide sweep launched: 1 barrier per level, 3 flow (vk_trsv modes)
  int factor(Ctx &ctx);
  int bicgstab(Ctx &ctx, double tol, int max_iter, bool resume, int &iters_out);
  int start(Ctx &ctx, double tol, int max_iter, bool resume);
  int run_chunk(Ctx &ctx, int every);
  int read_states(Ctx &ctx, std::vector<char> &out);
  int write_states(Ctx &ctx, const std::vector<char> &in);
  std::vector<int32_t> act_host;  // host copy of the active flags
  int residual(Ctx &ctx, std::vector<double> &rel);
  int set_active(Ctx &ctx, const std::vector<int32_t> &act);
  int solve(Ctx &ctx, std::vector<vshe_solve_stats> &stats);
  int check_err(Ctx &ctx, const char *what);
  int state_of(int k, int32_t &status, int32_t &iter) const;
};

struct Ctx {
  int device = 0;
  size_t budget = 0;
  cudaStream_t stream = nullptr;
  std::string last_error;
  std::mutex mu;
  int64_t next_handle = 0;
  bool profile = false;
  // polls of a device-side wait (grid barrier, flow poll, stage barrier) before it gives up
  // with VSHE_E_TIMEOUT
  unsigned long long spin_limit = kDefaultSpinLimit;
  // task sweep of one-CTA/cluster-per-task members: -1 autotuned per batch, 0 one CTA with staged
  // factor slices, K = 2, 4, 8 a cluster of K CTAs
  int task_sweep = -1;
  std::map<int64_t, std::unique_ptr<System>> systems;
  // vshe_solve_csr's pattern cache: the system of its last call (0 = none) and the options it was
  // created with (with copies of the option arrays)
  int64_t csr_cache = 0;
  vshe_solve_opts csr_cache_opts{};
  std::vector<int64_t> csr_cache_blocks;
  std::vector<int32_t> csr_cache_perm;
  std::map<std::vector<int64_t>, std::unique_ptr<Batch>> batches;
  // kernel-class timings of the last profiled solve (ms): spmv, trsv, vector, reliable, factor
  double prof[5] = {0, 0, 0, 0, 0};
  int64_t prof_counts[2] = {0, 0};
  // autotuned rows per reduction tile, per system size class (floor(log2 n)); the first system
  // of a class is timed, later ones reuse the choice, so a system's reduction order (and its
  // iterates) does not depend on the batch it is solved in
  std::map<int, int64_t> tile_choice;
  std::map<int, std::vector<double>> tile_timings;  // ms per SpMV for 512, 1024, 2048, 4096 rows
  // autotuned sweep choices per batch shape class (Batch::tune_key_*): a later batch of the same
  // class (a served batch rebuilt on an admission, say) reuses the choice instead of timing again;
  // every choice gives bitwise the same results
  std::map<int64_t, int> task_choice;
  std::map<int64_t, std::pair<int, int>> trsv_choice;  // (grid, kernel)
  int fail(int code, const std::string &msg);
  int cuda_fail(cudaError_t e, const char *what);
};

// releases the SHE problems of a context (she_pipeline.cpp)
void she_release_all(Ctx *ctx);
// device memory held by the context's SHE problems (she_pipeline.cpp)
size_t she_bytes(Ctx *ctx);
void poisson_release_all(Ctx *ctx);
size_t poisson_bytes(Ctx *ctx);

}  // namespace vshe

struct vshe_ctx : public vshe::Ctx {};

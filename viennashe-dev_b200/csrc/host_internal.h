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

template <typename T>
using BiStateHost = BiState<T>;
typedef RefDev RefHost;
typedef FactDev FactHost;

// Device allocations owned by one object, freed together.
struct DevArena {
  std::vector<void *> ptrs;
  size_t total = 0;
  void *alloc(size_t bytes, cudaError_t &e);
  void release();
  ~DevArena() { release(); }
};

struct Ctx;

// One resident linear system.
struct System {
  int64_t n = 0, nnz = 0;
  vshe_solve_opts opts{};
  bool mixed = true;
  bool factored = false;
  double bnorm_host = 0.0;
  // host copies of the pattern and schedules
  std::vector<int64_t> rp, diag, lrp, urp;
  std::vector<int32_t> ci, blk, lci, uci, levL, levU;
  int32_t nlevL = 0, nlevU = 0;
  int spmv_group = 8, trsv_group = 4;
  // device
  DevArena arena;
  int64_t *d_rp = nullptr; int32_t *d_ci = nullptr;
  double *d_av64 = nullptr; float *d_av32 = nullptr;
  double *d_b64 = nullptr, *d_x64 = nullptr, *d_r64 = nullptr;
  double *d_lu64 = nullptr; int64_t *d_diag = nullptr; int32_t *d_blk = nullptr;
  int64_t *d_lrp = nullptr, *d_urp = nullptr; int32_t *d_lci = nullptr, *d_uci = nullptr;
  void *d_lv = nullptr, *d_uv = nullptr, *d_dinv = nullptr;
  void *kv[9] = {nullptr};  // x r rh p v s t ph sh in the Krylov precision

  int create(Ctx &ctx, int64_t n, int64_t nnz, const int64_t *rp, const int32_t *ci, const double *v,
             const double *rhs, const vshe_solve_opts &o);
  int set_values(Ctx &ctx, const double *v, const double *rhs);
  void fill_sysdev(void *out) const;
};

// Several systems solved together.
struct Batch {
  std::vector<System *> sys;
  int nsys = 0;
  bool mixed = true, has_pc = true;
  int ntiles = 0;
  int32_t nlevL = 0, nlevU = 0;
  int spmv_group = 8, trsv_group = 4, trsv_grid = 148, ilu_grid = 148, num_sms = 148;
  DevArena arena;
  int32_t *d_tile_sys = nullptr, *d_sys_tile0 = nullptr, *d_active = nullptr, *d_counters = nullptr, *d_err = nullptr;
  int64_t *d_tile_r0 = nullptr, *d_tile_r1 = nullptr;
  double *d_partials = nullptr, *d_rnorm2 = nullptr, *d_bnorm2 = nullptr;
  unsigned *d_bar = nullptr;
  void *d_sysdev = nullptr, *d_state = nullptr, *d_refdev = nullptr, *d_factdev = nullptr;
  int64_t *d_lptrL = nullptr, *d_lptrU = nullptr;
  int32_t *d_esL = nullptr, *d_erL = nullptr, *d_esU = nullptr, *d_erU = nullptr;
  VkTiles tiles{};
  VkLevels levL{}, levU{};
  std::vector<char> last_state;

  int build(Ctx &ctx, const std::vector<System *> &members);
  int factor(Ctx &ctx);
  int bicgstab(Ctx &ctx, double tol, int max_iter, int &iters_out);
  int residual(Ctx &ctx, std::vector<double> &rel);
  int set_active(Ctx &ctx, const std::vector<int32_t> &act);
  int solve(Ctx &ctx, std::vector<vshe_solve_stats> &stats);
  int check_err(Ctx &ctx, const char *what);
  int state_of(int k, int32_t &status, int32_t &iter, double &res) const;
};

struct Ctx {
  int device = 0;
  size_t budget = 0;
  cudaStream_t stream = nullptr;
  std::string last_error;
  std::mutex mu;
  int64_t next_handle = 0;
  std::map<int64_t, std::unique_ptr<System>> systems;
  std::map<std::vector<int64_t>, std::unique_ptr<Batch>> batches;
  int fail(int code, const std::string &msg);
  int cuda_fail(cudaError_t e, const char *what);
};

}  // namespace vshe

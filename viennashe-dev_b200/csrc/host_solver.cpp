// host_solver.cpp -- C++ host side of the SHE linear-solve backend.
//
// Owns resident systems (CSR on the device, incomplete factors, Krylov
// vectors), builds their level schedules and tiles, merges several systems
// into one batch, and drives the batched BiCGStab / FP64 iterative refinement
// through the thin kernel launchers of kernels.h.  Exposes the public C ABI
// of include/vshe_gpu.h.
//
// Reference semantics mirrored here:
//   * input checks of src/solvers/solve.hpp:54-66 (empty rows, non-finite
//     rhs, ||b|| = 0 -> x = 0);
//   * tolerance / max_iters / block boundaries of linear_solver_config
//     (viennashe/solvers/config.hpp:56-232);
//   * ILU(0) + BiCGStab of the serial backend
//     (src/solvers/viennacl/serial_linear_solver.hpp:101-156), and the
//     per-energy-slab block ILU(0) the parallel backend intends
//     (src/solvers/viennacl/parallel_linear_solver.hpp:82-93).

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/vshe_gpu.h"
#include "kernels.h"
#include "host_internal.h"

namespace vshe {

const char *errstr(int code) {
  switch (code) {
    case VSHE_OK: return "ok";
    case VSHE_E_INVALID_ARGUMENT: return "invalid argument";
    case VSHE_E_EMPTY_ROW: return "solve(): Found empty row in system_matrix.";
    case VSHE_E_NAN: return "non-finite entry in matrix or right hand side";
    case VSHE_E_ODD_DIAGONAL: return "eliminate_odd_unknowns(): Diagonal entry not positive or not existing!";
    case VSHE_E_BREAKDOWN: return "BiCGStab breakdown";
    case VSHE_E_NOT_CONVERGED: return "iteration limit reached above tolerance";
    case VSHE_E_OUT_OF_MEMORY: return "device out of memory";
    case VSHE_E_BUDGET: return "request exceeds the HBM budget";
    case VSHE_E_CUDA: return "CUDA runtime error";
    case VSHE_E_TIMEOUT: return "device-side wait timed out";
    case VSHE_E_ZERO_PIVOT: return "zero pivot in incomplete factorisation";
    case VSHE_E_NOT_FOUND: return "unknown handle";
    case VSHE_E_UNSUPPORTED: return "unsupported option";
  }
  return "unknown error";
}

int Ctx::fail(int code, const std::string &msg) {
  last_error = std::string(errstr(code)) + (msg.empty() ? "" : ": " + msg);
  return code;
}

int Ctx::cuda_fail(cudaError_t e, const char *what) {
  if (e == cudaErrorMemoryAllocation) return fail(VSHE_E_OUT_OF_MEMORY, what);
  return fail(VSHE_E_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

static int group_for(double avg) {
  if (avg <= 2.5) return 2;
  if (avg <= 6.0) return 4;
  if (avg <= 12.0) return 8;
  if (avg <= 24.0) return 16;
  return 32;
}
static int trsv_group_for(double avg) {
  if (avg <= 1.5) return 1;
  if (avg <= 3.0) return 2;
  if (avg <= 6.0) return 4;
  return 8;
}

// ---------------------------------------------------------------- DevBuf
void *DevArena::alloc(size_t bytes, cudaError_t &e) {
  if (bytes == 0) bytes = 16;
  void *p = nullptr;
  e = cudaMalloc(&p, bytes);
  if (e != cudaSuccess) return nullptr;
  ptrs.push_back(p);
  total += bytes;
  return p;
}
void DevArena::release() {
  for (void *p : ptrs) cudaFree(p);
  ptrs.clear();
  total = 0;
}

// ------------------------------------------------------------- schedules
// Level of each row in the forward (L) and backward (U) solves of a
// block-restricted incomplete factorisation with A's pattern.
static void compute_levels(int64_t n, const std::vector<int64_t> &rp, const std::vector<int32_t> &ci,
                           const std::vector<int32_t> &blk, std::vector<int32_t> &levL, std::vector<int32_t> &levU,
                           int32_t &nL, int32_t &nU) {
  levL.assign(size_t(n), 0);
  levU.assign(size_t(n), 0);
  nL = 0; nU = 0;
  for (int64_t i = 0; i < n; ++i) {
    int32_t m = -1;
    for (int64_t k = rp[i]; k < rp[i + 1]; ++k) {
      int32_t j = ci[k];
      if (j >= i) break;
      if (blk[j] == blk[i] && levL[j] > m) m = levL[j];
    }
    levL[i] = m + 1;
    nL = std::max(nL, m + 2);
  }
  for (int64_t i = n - 1; i >= 0; --i) {
    int32_t m = -1;
    for (int64_t k = rp[i + 1] - 1; k >= rp[i]; --k) {
      int32_t j = ci[k];
      if (j <= i) break;
      if (blk[j] == blk[i] && levU[j] > m) m = levU[j];
    }
    levU[i] = m + 1;
    nU = std::max(nU, m + 2);
  }
}

// ----------------------------------------------------------------- System
int System::create(Ctx &ctx, int64_t n_, int64_t nnz_, const int64_t *rp_, const int32_t *ci_, const double *v,
                   const double *rhs, const vshe_solve_opts &o) {
  n = n_; nnz = nnz_; opts = o;
  if (n <= 0 || nnz <= 0 || !rp_ || !ci_ || !v || !rhs) return ctx.fail(VSHE_E_INVALID_ARGUMENT, "empty system or null pointer");
  if (n >= (int64_t(1) << 31)) return ctx.fail(VSHE_E_INVALID_ARGUMENT, "more than 2^31 rows");
  if (rp_[0] != 0 || rp_[n] != nnz) return ctx.fail(VSHE_E_INVALID_ARGUMENT, "row_ptr does not span nnz");
  rp.assign(rp_, rp_ + n + 1);
  ci.assign(ci_, ci_ + nnz);
  // src/solvers/solve.hpp:54-58: empty rows are an error
  for (int64_t i = 0; i < n; ++i) {
    if (rp[i + 1] < rp[i]) return ctx.fail(VSHE_E_INVALID_ARGUMENT, "row_ptr not monotone");
    if (rp[i + 1] == rp[i]) return ctx.fail(VSHE_E_EMPTY_ROW, "row " + std::to_string(i));
  }
  diag.assign(size_t(n), -1);
  for (int64_t i = 0; i < n; ++i) {
    int32_t prev = -1;
    for (int64_t k = rp[i]; k < rp[i + 1]; ++k) {
      int32_t j = ci[k];
      if (j < 0 || j >= n) return ctx.fail(VSHE_E_INVALID_ARGUMENT, "column index out of range");
      if (j <= prev) return ctx.fail(VSHE_E_INVALID_ARGUMENT, "columns not strictly ascending in row " + std::to_string(i));
      prev = j;
      if (j == i) diag[size_t(i)] = k;
    }
  }
  for (int64_t k = 0; k < nnz; ++k)
    if (!std::isfinite(v[k])) return ctx.fail(VSHE_E_NAN, "matrix entry " + std::to_string(k));
  for (int64_t i = 0; i < n; ++i)
    if (!std::isfinite(rhs[i])) return ctx.fail(VSHE_E_NAN, "rhs entry " + std::to_string(i));

  const bool has_pc = opts.precond != VSHE_PRECOND_NONE;
  if (has_pc)
    for (int64_t i = 0; i < n; ++i)
      if (diag[size_t(i)] < 0) return ctx.fail(VSHE_E_ZERO_PIVOT, "no diagonal entry in row " + std::to_string(i));

  // block ids
  blk.assign(size_t(n), 0);
  if (opts.precond == VSHE_PRECOND_BLOCK_ILU0 && opts.n_blocks > 0 && opts.block_ptr) {
    const int64_t *bp = opts.block_ptr;
    if (bp[0] != 0 || bp[opts.n_blocks] != n) return ctx.fail(VSHE_E_INVALID_ARGUMENT, "block_ptr must span [0, n]");
    for (int64_t b = 0; b < opts.n_blocks; ++b) {
      if (bp[b + 1] < bp[b]) return ctx.fail(VSHE_E_INVALID_ARGUMENT, "block_ptr not monotone");
      for (int64_t i = bp[b]; i < bp[b + 1]; ++i) blk[size_t(i)] = int32_t(b);
    }
  }
  // factor patterns and level schedules
  if (has_pc) {
    compute_levels(n, rp, ci, blk, levL, levU, nlevL, nlevU);
    lrp.assign(size_t(n) + 1, 0);
    urp.assign(size_t(n) + 1, 0);
    for (int64_t i = 0; i < n; ++i) {
      int64_t nl = 0, nu = 0;
      for (int64_t k = rp[i]; k < rp[i + 1]; ++k) {
        int32_t j = ci[k];
        if (j == i || blk[j] != blk[i]) continue;
        if (j < i) ++nl; else ++nu;
      }
      lrp[i + 1] = lrp[i] + nl;
      urp[i + 1] = urp[i] + nu;
    }
    lci.resize(size_t(lrp[n]));
    uci.resize(size_t(urp[n]));
    for (int64_t i = 0; i < n; ++i) {
      int64_t lp = lrp[i], up = urp[i];
      for (int64_t k = rp[i]; k < rp[i + 1]; ++k) {
        int32_t j = ci[k];
        if (j == i || blk[j] != blk[i]) continue;
        if (j < i) lci[size_t(lp++)] = j; else uci[size_t(up++)] = j;
      }
    }
  }
  mixed = opts.precision == VSHE_PRECISION_MIXED;
  spmv_group = group_for(double(nnz) / double(n));
  trsv_group = has_pc ? trsv_group_for(double(lrp[n] + urp[n]) / (2.0 * double(n))) : 1;

  // ---- device buffers ----
  cudaError_t e;
#define ALLOC(ptr, type, count)                                              \
  ptr = (type *)arena.alloc(sizeof(type) * size_t(count), e);               \
  if (!ptr) return ctx.cuda_fail(e, "cudaMalloc " #ptr);
  ALLOC(d_rp, int64_t, n + 1);
  ALLOC(d_ci, int32_t, nnz);
  ALLOC(d_av64, double, nnz);
  ALLOC(d_b64, double, n);
  ALLOC(d_x64, double, n);
  ALLOC(d_r64, double, n);
  ALLOC(d_blk, int32_t, n);
  if (mixed) { ALLOC(d_av32, float, nnz); }
  const size_t tsz = mixed ? sizeof(float) : sizeof(double);
  for (int k = 0; k < 9; ++k) {
    kv[k] = arena.alloc(tsz * size_t(n), e);
    if (!kv[k]) return ctx.cuda_fail(e, "cudaMalloc krylov");
  }
  if (has_pc) {
    ALLOC(d_lu64, double, nnz);
    ALLOC(d_diag, int64_t, n);
    ALLOC(d_lrp, int64_t, n + 1);
    ALLOC(d_urp, int64_t, n + 1);
    ALLOC(d_lci, int32_t, std::max<int64_t>(lrp[n], 1));
    ALLOC(d_uci, int32_t, std::max<int64_t>(urp[n], 1));
    d_lv = arena.alloc(tsz * size_t(std::max<int64_t>(lrp[n], 1)), e);
    if (!d_lv) return ctx.cuda_fail(e, "cudaMalloc lv");
    d_uv = arena.alloc(tsz * size_t(std::max<int64_t>(urp[n], 1)), e);
    if (!d_uv) return ctx.cuda_fail(e, "cudaMalloc uv");
    d_dinv = arena.alloc(tsz * size_t(n), e);
    if (!d_dinv) return ctx.cuda_fail(e, "cudaMalloc dinv");
  }
#undef ALLOC
  cudaStream_t s = ctx.stream;
#define H2D(dst, src, bytes)                                                             \
  if ((e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s)) != cudaSuccess) \
    return ctx.cuda_fail(e, "upload " #dst);
  H2D(d_rp, rp.data(), sizeof(int64_t) * size_t(n + 1));
  H2D(d_ci, ci.data(), sizeof(int32_t) * size_t(nnz));
  H2D(d_blk, blk.data(), sizeof(int32_t) * size_t(n));
  if (has_pc) {
    H2D(d_diag, diag.data(), sizeof(int64_t) * size_t(n));
    H2D(d_lrp, lrp.data(), sizeof(int64_t) * size_t(n + 1));
    H2D(d_urp, urp.data(), sizeof(int64_t) * size_t(n + 1));
    if (lrp[n]) H2D(d_lci, lci.data(), sizeof(int32_t) * size_t(lrp[n]));
    if (urp[n]) H2D(d_uci, uci.data(), sizeof(int32_t) * size_t(urp[n]));
  }
#undef H2D
  int rc = set_values(ctx, v, rhs);
  if (rc) return rc;
  if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return ctx.cuda_fail(e, "upload");
  return VSHE_OK;
}

int System::set_values(Ctx &ctx, const double *v, const double *rhs) {
  cudaStream_t s = ctx.stream;
  cudaError_t e;
  for (int64_t k = 0; k < nnz; ++k)
    if (!std::isfinite(v[k])) return ctx.fail(VSHE_E_NAN, "matrix entry " + std::to_string(k));
  bnorm_host = 0.0;
  for (int64_t i = 0; i < n; ++i) {
    if (!std::isfinite(rhs[i])) return ctx.fail(VSHE_E_NAN, "rhs entry " + std::to_string(i));
    bnorm_host += rhs[i] * rhs[i];
  }
  bnorm_host = std::sqrt(bnorm_host);
  if ((e = cudaMemcpyAsync(d_av64, v, sizeof(double) * size_t(nnz), cudaMemcpyHostToDevice, s)) != cudaSuccess) return ctx.cuda_fail(e, "upload values");
  if ((e = cudaMemcpyAsync(d_b64, rhs, sizeof(double) * size_t(n), cudaMemcpyHostToDevice, s)) != cudaSuccess) return ctx.cuda_fail(e, "upload rhs");
  if (mixed) vk_cast_f64_f32(nnz, d_av64, d_av32, s);
  factored = false;
  return VSHE_OK;
}

void System::fill_sysdev(void *out) const {
  // SysDev<T> has the same layout for both T (pointers); fill through the float view
  SysDev<float> d;
  d.n = n;
  d.rp = d_rp; d.ci = d_ci;
  d.av = mixed ? d_av32 : (const float *)d_av64;
  d.lrp = d_lrp; d.lci = d_lci; d.lv = (const float *)d_lv;
  d.urp = d_urp; d.uci = d_uci; d.uv = (const float *)d_uv;
  d.dinv = (const float *)d_dinv;
  d.x = (float *)kv[0]; d.r = (float *)kv[1]; d.rh = (float *)kv[2]; d.p = (float *)kv[3];
  d.v = (float *)kv[4]; d.s = (float *)kv[5]; d.t = (float *)kv[6]; d.ph = (float *)kv[7]; d.sh = (float *)kv[8];
  std::memcpy(out, &d, sizeof(d));
}

// ------------------------------------------------------------------ Batch
int Batch::build(Ctx &ctx, const std::vector<System *> &members) {
  sys = members;
  nsys = int(sys.size());
  mixed = sys[0]->mixed;
  has_pc = sys[0]->opts.precond != VSHE_PRECOND_NONE;
  for (System *S : sys) {
    if (S->mixed != mixed || (S->opts.precond != VSHE_PRECOND_NONE) != has_pc)
      return ctx.fail(VSHE_E_INVALID_ARGUMENT, "systems in one batch need the same precision and preconditioner kind");
  }
  // tiles
  const int64_t TILE = 2048;
  std::vector<int32_t> tsys, st0;
  std::vector<int64_t> tr0, tr1;
  for (int s = 0; s < nsys; ++s) {
    st0.push_back(int32_t(tsys.size()));
    for (int64_t a = 0; a < sys[s]->n; a += TILE) {
      tsys.push_back(s);
      tr0.push_back(a);
      tr1.push_back(std::min(a + TILE, sys[s]->n));
    }
  }
  st0.push_back(int32_t(tsys.size()));
  ntiles = int(tsys.size());
  // merged level schedules
  std::vector<int64_t> lptrL, lptrU;
  std::vector<int32_t> esL, erL, esU, erU;
  if (has_pc) {
    auto merge = [&](bool lower, std::vector<int64_t> &lptr, std::vector<int32_t> &es, std::vector<int32_t> &er, int32_t &nlev) {
      nlev = 0;
      for (System *S : sys) nlev = std::max(nlev, lower ? S->nlevL : S->nlevU);
      std::vector<int64_t> cnt(size_t(nlev) + 1, 0);
      for (System *S : sys) {
        const auto &lev = lower ? S->levL : S->levU;
        for (int32_t l : lev) cnt[size_t(l) + 1]++;
      }
      for (size_t k = 1; k < cnt.size(); ++k) cnt[k] += cnt[k - 1];
      lptr = cnt;
      int64_t total = cnt.back();
      es.resize(size_t(total));
      er.resize(size_t(total));
      std::vector<int64_t> pos(cnt.begin(), cnt.end() - 1);
      for (int s = 0; s < nsys; ++s) {
        const auto &lev = lower ? sys[s]->levL : sys[s]->levU;
        if (lower) {
          for (int64_t i = 0; i < sys[s]->n; ++i) { int64_t p = pos[size_t(lev[size_t(i)])]++; es[size_t(p)] = s; er[size_t(p)] = int32_t(i); }
        } else {
          for (int64_t i = sys[s]->n - 1; i >= 0; --i) { int64_t p = pos[size_t(lev[size_t(i)])]++; es[size_t(p)] = s; er[size_t(p)] = int32_t(i); }
        }
      }
    };
    merge(true, lptrL, esL, erL, nlevL);
    merge(false, lptrU, esU, erU, nlevU);
  }
  cudaError_t e;
#define ALLOC(ptr, type, count)                                              \
  ptr = (type *)arena.alloc(sizeof(type) * size_t(count), e);               \
  if (!ptr) return ctx.cuda_fail(e, "cudaMalloc batch " #ptr);
  ALLOC(d_tile_sys, int32_t, ntiles);
  ALLOC(d_tile_r0, int64_t, ntiles);
  ALLOC(d_tile_r1, int64_t, ntiles);
  ALLOC(d_sys_tile0, int32_t, nsys + 1);
  ALLOC(d_active, int32_t, nsys);
  ALLOC(d_counters, int32_t, nsys);
  ALLOC(d_partials, double, size_t(ntiles) * 3);
  ALLOC(d_bar, unsigned, 2);
  ALLOC(d_err, int32_t, 1);
  ALLOC(d_rnorm2, double, nsys);
  ALLOC(d_bnorm2, double, nsys);
  d_sysdev = arena.alloc(vk_sysdev_size_f32() * size_t(nsys), e);
  if (!d_sysdev) return ctx.cuda_fail(e, "cudaMalloc sysdev");
  d_state = arena.alloc(vk_bistate_size_f64() * size_t(nsys), e);
  if (!d_state) return ctx.cuda_fail(e, "cudaMalloc state");
  d_refdev = arena.alloc(vk_refdev_size() * size_t(nsys), e);
  if (!d_refdev) return ctx.cuda_fail(e, "cudaMalloc refdev");
  d_factdev = arena.alloc(vk_factdev_size() * size_t(nsys), e);
  if (!d_factdev) return ctx.cuda_fail(e, "cudaMalloc factdev");
  if (has_pc) {
    ALLOC(d_lptrL, int64_t, lptrL.size());
    ALLOC(d_lptrU, int64_t, lptrU.size());
    ALLOC(d_esL, int32_t, std::max<size_t>(esL.size(), 1));
    ALLOC(d_erL, int32_t, std::max<size_t>(erL.size(), 1));
    ALLOC(d_esU, int32_t, std::max<size_t>(esU.size(), 1));
    ALLOC(d_erU, int32_t, std::max<size_t>(erU.size(), 1));
  }
#undef ALLOC
  cudaStream_t s = ctx.stream;
  std::vector<char> sd(vk_sysdev_size_f32() * size_t(nsys));
  std::vector<char> rd(vk_refdev_size() * size_t(nsys));
  std::vector<char> fd(vk_factdev_size() * size_t(nsys));
  for (int k = 0; k < nsys; ++k) {
    sys[k]->fill_sysdev(sd.data() + vk_sysdev_size_f32() * size_t(k));
    RefHost r{sys[k]->n, sys[k]->d_rp, sys[k]->d_ci, sys[k]->d_av64, sys[k]->d_b64, sys[k]->d_x64, sys[k]->d_r64};
    std::memcpy(rd.data() + vk_refdev_size() * size_t(k), &r, sizeof(r));
    FactHost f{sys[k]->n, sys[k]->d_rp, sys[k]->d_ci, sys[k]->d_lu64, sys[k]->d_diag, sys[k]->d_blk};
    std::memcpy(fd.data() + vk_factdev_size() * size_t(k), &f, sizeof(f));
  }
  std::vector<int32_t> ones(size_t(nsys), 1), zeros(size_t(nsys), 0);
#define H2D(dst, src, bytes)                                                             \
  if ((e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s)) != cudaSuccess) \
    return ctx.cuda_fail(e, "upload batch " #dst);
  H2D(d_tile_sys, tsys.data(), sizeof(int32_t) * tsys.size());
  H2D(d_tile_r0, tr0.data(), sizeof(int64_t) * tr0.size());
  H2D(d_tile_r1, tr1.data(), sizeof(int64_t) * tr1.size());
  H2D(d_sys_tile0, st0.data(), sizeof(int32_t) * st0.size());
  H2D(d_active, ones.data(), sizeof(int32_t) * size_t(nsys));
  H2D(d_counters, zeros.data(), sizeof(int32_t) * size_t(nsys));
  H2D(d_sysdev, sd.data(), sd.size());
  H2D(d_refdev, rd.data(), rd.size());
  H2D(d_factdev, fd.data(), fd.size());
  if (has_pc) {
    H2D(d_lptrL, lptrL.data(), sizeof(int64_t) * lptrL.size());
    H2D(d_lptrU, lptrU.data(), sizeof(int64_t) * lptrU.size());
    if (!esL.empty()) { H2D(d_esL, esL.data(), sizeof(int32_t) * esL.size()); H2D(d_erL, erL.data(), sizeof(int32_t) * erL.size()); }
    if (!esU.empty()) { H2D(d_esU, esU.data(), sizeof(int32_t) * esU.size()); H2D(d_erU, erU.data(), sizeof(int32_t) * erU.size()); }
  }
#undef H2D
  if ((e = cudaMemsetAsync(d_bar, 0, 2 * sizeof(unsigned), s)) != cudaSuccess) return ctx.cuda_fail(e, "memset");
  if ((e = cudaMemsetAsync(d_err, 0, sizeof(int32_t), s)) != cudaSuccess) return ctx.cuda_fail(e, "memset");
  tiles = VkTiles{ntiles, d_tile_sys, d_tile_r0, d_tile_r1, d_sys_tile0};
  levL = VkLevels{nlevL, d_lptrL, nsys > 1 ? d_esL : nullptr, d_erL};
  levU = VkLevels{nlevU, d_lptrU, nsys > 1 ? d_esU : nullptr, d_erU};
  // execution shapes
  int64_t tot_nnz = 0, tot_n = 0, tot_lu = 0;
  for (System *S : sys) { tot_nnz += S->nnz; tot_n += S->n; if (has_pc) tot_lu += S->lrp[S->n] + S->urp[S->n]; }
  spmv_group = group_for(double(tot_nnz) / double(tot_n));
  trsv_group = has_pc ? trsv_group_for(double(tot_lu) / (2.0 * double(tot_n))) : 1;
  int dev = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&num_sms, cudaDevAttrMultiProcessorCount, dev);
  int bps = 0;
  if (mixed) vk_trsv_occupancy_f32(trsv_group, &bps); else vk_trsv_occupancy_f64(trsv_group, &bps);
  trsv_grid = std::max(1, bps) * num_sms;
  int bpf = 0;
  vk_ilu0_occupancy(&bpf);
  ilu_grid = std::max(1, bpf) * num_sms;
  return VSHE_OK;
}

int Batch::check_err(Ctx &ctx, const char *what) {
  int32_t err = 0;
  cudaError_t e = cudaMemcpyAsync(&err, d_err, sizeof(int32_t), cudaMemcpyDeviceToHost, ctx.stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx.stream);
  if (e != cudaSuccess) return ctx.cuda_fail(e, what);
  if (err) {
    cudaMemsetAsync(d_err, 0, sizeof(int32_t), ctx.stream);
    cudaMemsetAsync(d_bar, 0, 2 * sizeof(unsigned), ctx.stream);
    return ctx.fail(err, what);
  }
  return VSHE_OK;
}

int Batch::factor(Ctx &ctx) {
  if (!has_pc) return VSHE_OK;
  cudaStream_t s = ctx.stream;
  cudaError_t e;
  for (System *S : sys)
    if ((e = cudaMemcpyAsync(S->d_lu64, S->d_av64, sizeof(double) * size_t(S->nnz), cudaMemcpyDeviceToDevice, s)) != cudaSuccess)
      return ctx.cuda_fail(e, "copy factor values");
  const int mode = (sys[0]->opts.trsv_mode == VSHE_TRSV_PER_LEVEL) ? 2 : 1;
  int rc = vk_ilu0(mode, mode == 1 ? ilu_grid : std::max(1, num_sms * 8), d_factdev, &levL, d_bar, d_err, s);
  if (rc) return ctx.cuda_fail(cudaError_t(rc), "ilu0 launch");
  for (System *S : sys) {
    if (mixed)
      vk_split_factor_f32(S->n, S->d_rp, S->d_ci, S->d_lu64, S->d_blk, S->d_lrp, (float *)S->d_lv, S->d_urp, (float *)S->d_uv, (float *)S->d_dinv, s);
    else
      vk_split_factor_f64(S->n, S->d_rp, S->d_ci, S->d_lu64, S->d_blk, S->d_lrp, (double *)S->d_lv, S->d_urp, (double *)S->d_uv, (double *)S->d_dinv, s);
  }
  rc = check_err(ctx, "ilu0 factorisation");
  if (rc) return rc;
  for (System *S : sys) S->factored = true;
  return VSHE_OK;
}

// One BiCGStab solve on every active system, rhs in r (precision of the batch),
// to relative tolerance `tol`.  Returns the total iterations of the slowest system.
int Batch::bicgstab(Ctx &ctx, double tol, int max_iter, int &iters_out) {
  cudaStream_t s = ctx.stream;
  const int every = sys[0]->opts.check_every > 0 ? sys[0]->opts.check_every : 8;
  const int mode = (sys[0]->opts.trsv_mode == VSHE_TRSV_PER_LEVEL) ? 2 : 1;
  const int lvl_grid = mode == 1 ? trsv_grid : std::max(1, num_sms * 8);
  // state: tolerance and iteration cap (host writes, before init)
  std::vector<char> stbuf(vk_bistate_size_f64() * size_t(nsys), 0);
  cudaError_t e = cudaMemcpyAsync(stbuf.data(), d_state, stbuf.size(), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return ctx.cuda_fail(e, "read state");
  for (int k = 0; k < nsys; ++k) {
    if (mixed) {
      BiStateHost<float> *b = (BiStateHost<float> *)(stbuf.data() + vk_bistate_size_f32() * size_t(k));
      b->tol = float(tol); b->max_iter = max_iter; b->done = 0;
    } else {
      BiStateHost<double> *b = (BiStateHost<double> *)(stbuf.data() + vk_bistate_size_f64() * size_t(k));
      b->tol = tol; b->max_iter = max_iter; b->done = 0;
    }
  }
  if ((e = cudaMemcpyAsync(d_state, stbuf.data(), stbuf.size(), cudaMemcpyHostToDevice, s)) != cudaSuccess) return ctx.cuda_fail(e, "write state");
  if (mixed) vk_bicg_init_f32(ntiles, d_sysdev, d_state, &tiles, (float *)d_partials, d_counters, d_active, s);
  else vk_bicg_init_f64(ntiles, d_sysdev, d_state, &tiles, d_partials, d_counters, d_active, s);
  int done_iters = 0;
  while (true) {
    for (int it = 0; it < every; ++it) {
      int rc = 0;
      if (mixed) {
        vk_update_p_f32(ntiles, d_sysdev, d_state, &tiles, d_active, s);
        if (has_pc) rc = vk_trsv_f32(mode, trsv_group, lvl_grid, d_sysdev, d_state, d_active, &levL, &levU, 0, d_bar, d_err, s);
        else vk_precond_copy_f32(ntiles, d_sysdev, d_state, &tiles, d_active, 0, s);
        vk_spmv_dot_f32(spmv_group, ntiles, d_sysdev, d_state, &tiles, (float *)d_partials, d_counters, d_active, 0, s);
        vk_update_s_f32(ntiles, d_sysdev, d_state, &tiles, (float *)d_partials, d_counters, d_active, s);
        if (has_pc) rc |= vk_trsv_f32(mode, trsv_group, lvl_grid, d_sysdev, d_state, d_active, &levL, &levU, 1, d_bar, d_err, s);
        else vk_precond_copy_f32(ntiles, d_sysdev, d_state, &tiles, d_active, 1, s);
        vk_spmv_dot_f32(spmv_group, ntiles, d_sysdev, d_state, &tiles, (float *)d_partials, d_counters, d_active, 1, s);
        vk_update_xr_f32(ntiles, d_sysdev, d_state, &tiles, (float *)d_partials, d_counters, d_active, s);
      } else {
        vk_update_p_f64(ntiles, d_sysdev, d_state, &tiles, d_active, s);
        if (has_pc) rc = vk_trsv_f64(mode, trsv_group, lvl_grid, d_sysdev, d_state, d_active, &levL, &levU, 0, d_bar, d_err, s);
        else vk_precond_copy_f64(ntiles, d_sysdev, d_state, &tiles, d_active, 0, s);
        vk_spmv_dot_f64(spmv_group, ntiles, d_sysdev, d_state, &tiles, d_partials, d_counters, d_active, 0, s);
        vk_update_s_f64(ntiles, d_sysdev, d_state, &tiles, d_partials, d_counters, d_active, s);
        if (has_pc) rc |= vk_trsv_f64(mode, trsv_group, lvl_grid, d_sysdev, d_state, d_active, &levL, &levU, 1, d_bar, d_err, s);
        else vk_precond_copy_f64(ntiles, d_sysdev, d_state, &tiles, d_active, 1, s);
        vk_spmv_dot_f64(spmv_group, ntiles, d_sysdev, d_state, &tiles, d_partials, d_counters, d_active, 1, s);
        vk_update_xr_f64(ntiles, d_sysdev, d_state, &tiles, d_partials, d_counters, d_active, s);
      }
      if (rc) return ctx.cuda_fail(cudaError_t(rc), "trsv launch");
    }
    done_iters += every;
    if ((e = cudaMemcpyAsync(stbuf.data(), d_state, stbuf.size(), cudaMemcpyDeviceToHost, s)) != cudaSuccess) return ctx.cuda_fail(e, "read state");
    int rc = check_err(ctx, "bicgstab");
    if (rc) return rc;
    bool all_done = true;
    int maxit = 0;
    for (int k = 0; k < nsys; ++k) {
      int32_t d, it;
      if (mixed) { auto *b = (BiStateHost<float> *)(stbuf.data() + vk_bistate_size_f32() * size_t(k)); d = b->done; it = b->iter; }
      else { auto *b = (BiStateHost<double> *)(stbuf.data() + vk_bistate_size_f64() * size_t(k)); d = b->done; it = b->iter; }
      if (!d) all_done = false;
      maxit = std::max(maxit, it);
    }
    iters_out = maxit;
    if (all_done || done_iters >= max_iter + every) break;
  }
  // per-system status
  last_state.assign(stbuf.begin(), stbuf.end());
  return VSHE_OK;
}

int Batch::state_of(int k, int32_t &status, int32_t &iter, double &res) const {
  if (last_state.empty()) { status = 0; iter = 0; res = 0; return 0; }
  if (mixed) { auto *b = (const BiStateHost<float> *)(last_state.data() + vk_bistate_size_f32() * size_t(k)); status = b->status; iter = b->iter; res = b->res; }
  else { auto *b = (const BiStateHost<double> *)(last_state.data() + vk_bistate_size_f64() * size_t(k)); status = b->status; iter = b->iter; res = b->res; }
  return 0;
}

// FP64 residual r = b - A x for all members; returns per-system ||r|| / ||b||.
int Batch::residual(Ctx &ctx, std::vector<double> &rel) {
  cudaStream_t s = ctx.stream;
  vk_residual64(spmv_group, ntiles, d_refdev, &tiles, d_partials, d_counters, d_active, d_rnorm2, d_bnorm2, s);
  std::vector<double> r2((size_t)nsys), b2((size_t)nsys);
  cudaError_t e = cudaMemcpyAsync(r2.data(), d_rnorm2, sizeof(double) * size_t(nsys), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(b2.data(), d_bnorm2, sizeof(double) * size_t(nsys), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return ctx.cuda_fail(e, "residual");
  rel.resize(size_t(nsys));
  for (int k = 0; k < nsys; ++k) rel[size_t(k)] = b2[size_t(k)] > 0 ? std::sqrt(r2[size_t(k)]) / std::sqrt(b2[size_t(k)]) : 0.0;
  return VSHE_OK;
}

int Batch::set_active(Ctx &ctx, const std::vector<int32_t> &act) {
  cudaError_t e = cudaMemcpyAsync(d_active, act.data(), sizeof(int32_t) * size_t(nsys), cudaMemcpyHostToDevice, ctx.stream);
  if (e != cudaSuccess) return ctx.cuda_fail(e, "active flags");
  return VSHE_OK;
}

// Full solve of every member: factorisation, then FP64 BiCGStab or FP32 BiCGStab
// inside FP64 iterative refinement, to each member's tolerance.
int Batch::solve(Ctx &ctx, std::vector<vshe_solve_stats> &stats) {
  cudaStream_t s = ctx.stream;
  cudaError_t e;
  stats.assign(size_t(nsys), vshe_solve_stats{});
  cudaEvent_t e0, e1, e2;
  cudaEventCreate(&e0); cudaEventCreate(&e1); cudaEventCreate(&e2);
  struct EvGuard { cudaEvent_t a, b, c; ~EvGuard() { cudaEventDestroy(a); cudaEventDestroy(b); cudaEventDestroy(c); } } guard{e0, e1, e2};
  std::vector<int32_t> act(size_t(nsys), 1);
  int rc = set_active(ctx, act);
  if (rc) return rc;
  cudaEventRecord(e0, s);
  rc = factor(ctx);
  if (rc) return rc;
  cudaEventRecord(e1, s);
  const vshe_solve_opts &o = sys[0]->opts;
  std::vector<int32_t> status(size_t(nsys), 0), iters(size_t(nsys), 0), refs(size_t(nsys), 0);
  std::vector<double> rel(size_t(nsys), 1.0);
  // x64 = 0, r64 = b
  for (System *S : sys) {
    if ((e = cudaMemsetAsync(S->d_x64, 0, sizeof(double) * size_t(S->n), s)) != cudaSuccess) return ctx.cuda_fail(e, "memset x");
  }
  // trivial rhs -> x = 0 (src/solvers/solve.hpp:60-66)
  for (int k = 0; k < nsys; ++k)
    if (sys[size_t(k)]->bnorm_host == 0.0) { act[size_t(k)] = 0; rel[size_t(k)] = 0.0; }
  if (!mixed) {
    for (int k = 0; k < nsys; ++k) {
      System *S = sys[size_t(k)];
      if ((e = cudaMemcpyAsync(S->kv[1], S->d_b64, sizeof(double) * size_t(S->n), cudaMemcpyDeviceToDevice, s)) != cudaSuccess) return ctx.cuda_fail(e, "rhs");
    }
    if ((rc = set_active(ctx, act))) return rc;
    int it = 0;
    rc = bicgstab(ctx, o.tol, o.max_iters, it);
    if (rc) return rc;
    for (int k = 0; k < nsys; ++k) {
      System *S = sys[size_t(k)];
      int32_t stt, itk; double res;
      state_of(k, stt, itk, res);
      status[size_t(k)] = act[size_t(k)] ? stt : 0;
      iters[size_t(k)] = act[size_t(k)] ? itk : 0;
      if (act[size_t(k)] && (e = cudaMemcpyAsync(S->d_x64, S->kv[0], sizeof(double) * size_t(S->n), cudaMemcpyDeviceToDevice, s)) != cudaSuccess) return ctx.cuda_fail(e, "x");
    }
    std::vector<int32_t> all(size_t(nsys), 1);
    if ((rc = set_active(ctx, all))) return rc;
    if ((rc = residual(ctx, rel))) return rc;
  } else {
    std::vector<int32_t> all(size_t(nsys), 1);
    const int max_ref = o.max_refinements > 0 ? o.max_refinements : 10;
    const double inner = o.inner_tol > 0 ? o.inner_tol : 1e-5;
    for (int sweep = 0; sweep <= max_ref; ++sweep) {
      if ((rc = set_active(ctx, all))) return rc;
      if ((rc = residual(ctx, rel))) return rc;  // r64 = b - A x64
      bool any = false;
      for (int k = 0; k < nsys; ++k) {
        if (sys[size_t(k)]->bnorm_host == 0.0) { act[size_t(k)] = 0; rel[size_t(k)] = 0.0; continue; }
        act[size_t(k)] = (rel[size_t(k)] >= o.tol && status[size_t(k)] == 0 && iters[size_t(k)] < o.max_iters) ? 1 : 0;
        if (act[size_t(k)]) any = true;
      }
      if (!any || sweep == max_ref) break;
      if ((rc = set_active(ctx, act))) return rc;
      vk_scale_to_f32(ntiles, d_refdev, d_sysdev, &tiles, d_active, d_rnorm2, s);
      int it = 0;
      int budget = 0;
      for (int k = 0; k < nsys; ++k) if (act[size_t(k)]) budget = std::max(budget, o.max_iters - iters[size_t(k)]);
      rc = bicgstab(ctx, inner, std::max(1, budget), it);
      if (rc) return rc;
      vk_accumulate_x(ntiles, d_refdev, d_sysdev, &tiles, d_active, d_rnorm2, s);
      for (int k = 0; k < nsys; ++k) {
        if (!act[size_t(k)]) continue;
        int32_t stt, itk; double res;
        state_of(k, stt, itk, res);
        iters[size_t(k)] += itk;
        refs[size_t(k)] += 1;
        // an inner breakdown / stall is not fatal while refinement still makes progress
        if (stt == VSHE_E_BREAKDOWN && itk <= 1) status[size_t(k)] = VSHE_E_BREAKDOWN;
      }
    }
  }
  cudaEventRecord(e2, s);
  if ((e = cudaEventSynchronize(e2)) != cudaSuccess) return ctx.cuda_fail(e, "solve");
  float ms_setup = 0, ms_solve = 0;
  cudaEventElapsedTime(&ms_setup, e0, e1);
  cudaEventElapsedTime(&ms_solve, e1, e2);
  for (int k = 0; k < nsys; ++k) {
    vshe_solve_stats &st = stats[size_t(k)];
    System *S = sys[size_t(k)];
    st.iterations = iters[size_t(k)];
    st.refinements = refs[size_t(k)];
    st.rel_residual = rel[size_t(k)];
    st.setup_ms = ms_setup;
    st.solve_ms = ms_solve;
    st.levels_L = S->nlevL;
    st.levels_U = S->nlevU;
    st.bytes_device = int64_t(S->arena.total);
    int32_t code = status[size_t(k)];
    if (code == 0 && rel[size_t(k)] >= o.tol) code = VSHE_E_NOT_CONVERGED;
    if (code == VSHE_E_BREAKDOWN && rel[size_t(k)] < o.tol) code = 0;
    st.status = code;
  }
  return VSHE_OK;
}

}  // namespace vshe

// =======================================================================
// public C ABI
// =======================================================================
using namespace vshe;

struct vshe_ctx : public vshe::Ctx {};

extern "C" {

void vshe_default_opts(vshe_solve_opts *o) {
  std::memset(o, 0, sizeof(*o));
  o->precision = VSHE_PRECISION_MIXED;
  o->precond = VSHE_PRECOND_ILU0;
  o->ordering = VSHE_ORDER_NATURAL;
  o->tol = 1e-10;
  o->max_iters = 1000;
  o->inner_tol = 1e-5;
  o->max_refinements = 10;
  o->trsv_mode = VSHE_TRSV_AUTO;
  o->check_every = 8;
}

const char *vshe_errstr(int code) { return vshe::errstr(code); }

int vshe_create(vshe_ctx **ctx, int device, size_t budget) {
  if (!ctx) return VSHE_E_INVALID_ARGUMENT;
  *ctx = nullptr;
  int ndev = 0;
  cudaError_t e = cudaGetDeviceCount(&ndev);
  if (e != cudaSuccess || ndev == 0) return VSHE_E_CUDA;
  if (device < 0 || device >= ndev) return VSHE_E_INVALID_ARGUMENT;
  if ((e = cudaSetDevice(device)) != cudaSuccess) return VSHE_E_CUDA;
  std::unique_ptr<vshe_ctx> c(new vshe_ctx);
  c->device = device;
  c->budget = budget ? budget : size_t(150) * 1000 * 1000 * 1000;
  if ((e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking)) != cudaSuccess) return VSHE_E_CUDA;
  *ctx = c.release();
  return VSHE_OK;
}

int vshe_destroy(vshe_ctx *ctx) {
  if (!ctx) return VSHE_E_INVALID_ARGUMENT;
  cudaSetDevice(ctx->device);
  cudaStreamSynchronize(ctx->stream);
  ctx->batches.clear();
  ctx->systems.clear();
  cudaStreamDestroy(ctx->stream);
  delete ctx;
  return VSHE_OK;
}

const char *vshe_last_error(vshe_ctx *ctx) { return ctx ? ctx->last_error.c_str() : "no context"; }

size_t vshe_bytes_in_use(vshe_ctx *ctx) {
  if (!ctx) return 0;
  size_t t = 0;
  for (auto &kv : ctx->systems) t += kv.second->arena.total;
  for (auto &kv : ctx->batches) t += kv.second->arena.total;
  return t;
}

int vshe_system_create(vshe_ctx *ctx, int64_t n, int64_t nnz, const int64_t *rp, const int32_t *ci, const double *v,
                       const double *rhs, const vshe_solve_opts *opts, int64_t *handle) {
  if (!ctx || !handle) return VSHE_E_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lk(ctx->mu);
  cudaSetDevice(ctx->device);
  vshe_solve_opts o;
  if (opts) o = *opts; else vshe_default_opts(&o);
  // admission against the HBM budget (upper estimate of the system's footprint)
  const size_t est = size_t(nnz) * (4 + 8 + 8 + 4 + 16) + size_t(n) * (8 * 8 + 9 * 8 + 16);
  if (vshe_bytes_in_use(ctx) + est > ctx->budget) return ctx->fail(VSHE_E_BUDGET, std::to_string(est) + " bytes requested");
  std::unique_ptr<System> S(new System);
  int rc = S->create(*ctx, n, nnz, rp, ci, v, rhs, o);
  if (rc) return rc;
  int64_t h = ++ctx->next_handle;
  ctx->systems[h] = std::move(S);
  *handle = h;
  return VSHE_OK;
}

int vshe_system_set_values(vshe_ctx *ctx, int64_t h, const double *v, const double *rhs) {
  if (!ctx) return VSHE_E_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lk(ctx->mu);
  auto it = ctx->systems.find(h);
  if (it == ctx->systems.end()) return ctx->fail(VSHE_E_NOT_FOUND, "");
  cudaSetDevice(ctx->device);
  return it->second->set_values(*ctx, v, rhs);
}

static Batch *get_batch(vshe_ctx *ctx, const std::vector<int64_t> &hs, int &rc) {
  rc = VSHE_OK;
  auto it = ctx->batches.find(hs);
  if (it != ctx->batches.end()) return it->second.get();
  std::vector<System *> mem;
  for (int64_t h : hs) {
    auto f = ctx->systems.find(h);
    if (f == ctx->systems.end()) { rc = ctx->fail(VSHE_E_NOT_FOUND, std::to_string(h)); return nullptr; }
    mem.push_back(f->second.get());
  }
  std::unique_ptr<Batch> B(new Batch);
  rc = B->build(*ctx, mem);
  if (rc) return nullptr;
  Batch *p = B.get();
  ctx->batches[hs] = std::move(B);
  return p;
}

static void drop_batches_with(vshe_ctx *ctx, int64_t h) {
  for (auto it = ctx->batches.begin(); it != ctx->batches.end();) {
    if (std::find(it->first.begin(), it->first.end(), h) != it->first.end()) it = ctx->batches.erase(it);
    else ++it;
  }
}

int vshe_batch_solve(vshe_ctx *ctx, int32_t count, const int64_t *handles, vshe_solve_stats *stats) {
  if (!ctx || count <= 0 || !handles) return VSHE_E_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lk(ctx->mu);
  cudaSetDevice(ctx->device);
  std::vector<int64_t> hs(handles, handles + count);
  int rc;
  Batch *B = get_batch(ctx, hs, rc);
  if (!B) return rc;
  std::vector<vshe_solve_stats> st;
  rc = B->solve(*ctx, st);
  if (rc) return rc;
  int worst = VSHE_OK;
  for (int k = 0; k < count; ++k) {
    if (stats) stats[k] = st[size_t(k)];
    if (st[size_t(k)].status) worst = st[size_t(k)].status;
  }
  if (worst) ctx->fail(worst, "");
  return worst;
}

int vshe_system_solve(vshe_ctx *ctx, int64_t h, double *x, vshe_solve_stats *stats) {
  int rc = vshe_batch_solve(ctx, 1, &h, stats);
  if (x && (rc == VSHE_OK || rc == VSHE_E_NOT_CONVERGED)) {
    int rc2 = vshe_system_get_x(ctx, h, x);
    if (rc2) return rc2;
  }
  return rc;
}

int vshe_system_get_x(vshe_ctx *ctx, int64_t h, double *x) {
  if (!ctx || !x) return VSHE_E_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lk(ctx->mu);
  auto it = ctx->systems.find(h);
  if (it == ctx->systems.end()) return ctx->fail(VSHE_E_NOT_FOUND, "");
  System *S = it->second.get();
  cudaError_t e = cudaMemcpyAsync(x, S->d_x64, sizeof(double) * size_t(S->n), cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) return ctx->cuda_fail(e, "download x");
  return VSHE_OK;
}

int vshe_system_free(vshe_ctx *ctx, int64_t h) {
  if (!ctx) return VSHE_E_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lk(ctx->mu);
  cudaSetDevice(ctx->device);
  cudaStreamSynchronize(ctx->stream);
  drop_batches_with(ctx, h);
  auto it = ctx->systems.find(h);
  if (it == ctx->systems.end()) return ctx->fail(VSHE_E_NOT_FOUND, "");
  ctx->systems.erase(it);
  return VSHE_OK;
}

int vshe_solve_csr(vshe_ctx *ctx, int64_t n, int64_t nnz, const int64_t *rp, const int32_t *ci, const double *v,
                   const double *rhs, const vshe_solve_opts *opts, double *x, vshe_solve_stats *stats) {
  if (!ctx || !x || !rhs) return VSHE_E_INVALID_ARGUMENT;
  int64_t h = 0;
  int rc = vshe_system_create(ctx, n, nnz, rp, ci, v, rhs, opts, &h);
  if (rc) return rc;
  rc = vshe_system_solve(ctx, h, x, stats);
  vshe_system_free(ctx, h);
  return rc;
}

int vshe_system_spmv(vshe_ctx *ctx, int64_t h, int32_t precision, const double *x, double *y) {
  if (!ctx || !x || !y) return VSHE_E_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lk(ctx->mu);
  cudaSetDevice(ctx->device);
  auto it = ctx->systems.find(h);
  if (it == ctx->systems.end()) return ctx->fail(VSHE_E_NOT_FOUND, "");
  System *S = it->second.get();
  cudaStream_t s = ctx->stream;
  cudaError_t e;
  const int grid = std::max(1, int(std::min<int64_t>((S->n * S->spmv_group + 255) / 256, 65535 * 8)));
  if (precision == 1) {
    if (!S->mixed) return ctx->fail(VSHE_E_UNSUPPORTED, "FP32 values exist only for mixed-precision systems");
    std::vector<float> xf((size_t)S->n), yf((size_t)S->n);
    for (int64_t i = 0; i < S->n; ++i) xf[size_t(i)] = float(x[i]);
    float *dx = (float *)S->kv[0], *dy = (float *)S->kv[1];
    if ((e = cudaMemcpyAsync(dx, xf.data(), sizeof(float) * xf.size(), cudaMemcpyHostToDevice, s)) != cudaSuccess) return ctx->cuda_fail(e, "x");
    vk_spmv_plain_f32(S->spmv_group, grid, S->n, S->d_rp, S->d_ci, S->d_av32, dx, dy, s);
    if ((e = cudaMemcpyAsync(yf.data(), dy, sizeof(float) * yf.size(), cudaMemcpyDeviceToHost, s)) != cudaSuccess) return ctx->cuda_fail(e, "y");
    if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return ctx->cuda_fail(e, "spmv");
    for (int64_t i = 0; i < S->n; ++i) y[i] = double(yf[size_t(i)]);
    return VSHE_OK;
  }
  double *dx = S->d_x64, *dy = S->d_r64;
  if ((e = cudaMemcpyAsync(dx, x, sizeof(double) * size_t(S->n), cudaMemcpyHostToDevice, s)) != cudaSuccess) return ctx->cuda_fail(e, "x");
  vk_spmv_plain_f64(S->spmv_group, grid, S->n, S->d_rp, S->d_ci, S->d_av64, dx, dy, s);
  if ((e = cudaMemcpyAsync(y, dy, sizeof(double) * size_t(S->n), cudaMemcpyDeviceToHost, s)) != cudaSuccess) return ctx->cuda_fail(e, "y");
  if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return ctx->cuda_fail(e, "spmv");
  return VSHE_OK;
}

int vshe_system_time_spmv(vshe_ctx *ctx, int64_t h, int32_t precision, int32_t reps, double *ms) {
  if (!ctx || !ms || reps <= 0) return VSHE_E_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lk(ctx->mu);
  cudaSetDevice(ctx->device);
  auto it = ctx->systems.find(h);
  if (it == ctx->systems.end()) return ctx->fail(VSHE_E_NOT_FOUND, "");
  System *S = it->second.get();
  cudaStream_t s = ctx->stream;
  const int grid = std::max(1, int(std::min<int64_t>((S->n * S->spmv_group + 255) / 256, 65535 * 8)));
  cudaEvent_t a, b;
  cudaEventCreate(&a); cudaEventCreate(&b);
  if (precision == 1 && !S->mixed) return ctx->fail(VSHE_E_UNSUPPORTED, "");
  for (int w = 0; w < 3; ++w) {
    if (precision == 1) vk_spmv_plain_f32(S->spmv_group, grid, S->n, S->d_rp, S->d_ci, S->d_av32, (float *)S->kv[0], (float *)S->kv[1], s);
    else vk_spmv_plain_f64(S->spmv_group, grid, S->n, S->d_rp, S->d_ci, S->d_av64, S->d_x64, S->d_r64, s);
  }
  cudaEventRecord(a, s);
  for (int r = 0; r < reps; ++r) {
    if (precision == 1) vk_spmv_plain_f32(S->spmv_group, grid, S->n, S->d_rp, S->d_ci, S->d_av32, (float *)S->kv[0], (float *)S->kv[1], s);
    else vk_spmv_plain_f64(S->spmv_group, grid, S->n, S->d_rp, S->d_ci, S->d_av64, S->d_x64, S->d_r64, s);
  }
  cudaEventRecord(b, s);
  cudaError_t e = cudaEventSynchronize(b);
  float t = 0;
  cudaEventElapsedTime(&t, a, b);
  cudaEventDestroy(a); cudaEventDestroy(b);
  if (e != cudaSuccess) return ctx->cuda_fail(e, "time spmv");
  *ms = double(t) / reps;
  return VSHE_OK;
}

int vshe_system_factor_values(vshe_ctx *ctx, int64_t h, double *lu) {
  if (!ctx || !lu) return VSHE_E_INVALID_ARGUMENT;
  int rc;
  {
    std::lock_guard<std::mutex> lk(ctx->mu);
    cudaSetDevice(ctx->device);
    std::vector<int64_t> hs{h};
    Batch *B = get_batch(ctx, hs, rc);
    if (!B) return rc;
    if (!B->has_pc) return ctx->fail(VSHE_E_UNSUPPORTED, "no preconditioner");
    rc = B->factor(*ctx);
    if (rc) return rc;
    System *S = B->sys[0];
    cudaError_t e = cudaMemcpyAsync(lu, S->d_lu64, sizeof(double) * size_t(S->nnz), cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) return ctx->cuda_fail(e, "download factor");
    // entries coupling two blocks are not part of the factor
    for (int64_t i = 0; i < S->n; ++i)
      for (int64_t k = S->rp[i]; k < S->rp[i + 1]; ++k)
        if (S->blk[size_t(S->ci[k])] != S->blk[size_t(i)]) lu[k] = 0.0;
  }
  return VSHE_OK;
}

}  // extern "C"

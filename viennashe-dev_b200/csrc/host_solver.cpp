// host_solver.cpp -- C++ host side of the SHE linear-solve backend.
//
// Owns resident systems (CSR on the device, incomplete factors, Krylov
// vectors), builds their orderings, level schedules and tiles, merges several
// systems into one batch, and drives the batched BiCGStab (FP64, or FP32 with
// FP64 reliable updates) through the thin kernel launchers of kernels.h.
// Exposes the public C ABI of include/vshe_gpu.h.
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
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <cstdio>
#include <cstring>
#include <functional>
#include <thread>
#include <map>
#include <memory>
#include <mutex>
#include <numeric>
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
    case VSHE_E_CAPACITY: return "size exceeds the fixed scratch capacity of the no-allocation entry point";
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

// ----------------------------------------------------------------- System
int System::create(Ctx &ctx, int64_t n_, int64_t nnz_, const int64_t *rp_, const int32_t *ci_, const double *v,
                   const double *rhs, const vshe_solve_opts &o) {
  n = n_; nnz = nnz_; opts = o;
  if (n <= 0 || nnz <= 0 || !rp_ || !ci_ || !v || !rhs) return ctx.fail(VSHE_E_INVALID_ARGUMENT, "empty system or null pointer");
  if (n >= (int64_t(1) << 31) - 64) return ctx.fail(VSHE_E_INVALID_ARGUMENT, "more than 2^31 - 64 rows");
  if (rp_[0] != 0 || rp_[n] != nnz) return ctx.fail(VSHE_E_INVALID_ARGUMENT, "row_ptr does not span nnz");
  rp.assign(rp_, rp_ + n + 1);
  ci.assign(ci_, ci_ + nnz);
  // src/solvers/solve.hpp:54-58: empty rows are an error
  for (int64_t i = 0; i < n; ++i) {
    if (rp[i + 1] < rp[i]) return ctx.fail(VSHE_E_INVALID_ARGUMENT, "row_ptr not monotone");
    if (rp[i + 1] == rp[i]) return ctx.fail(VSHE_E_EMPTY_ROW, "row " + std::to_string(i));
  }
  for (int64_t i = 0; i < n; ++i) {
    int32_t prev = -1;
    for (int64_t k = rp[i]; k < rp[i + 1]; ++k) {
      int32_t j = ci[k];
      if (j < 0 || j >= n) return ctx.fail(VSHE_E_INVALID_ARGUMENT, "column index out of range");
      if (j <= prev) return ctx.fail(VSHE_E_INVALID_ARGUMENT, "columns not strictly ascending in row " + std::to_string(i));
      prev = j;
    }
  }
  for (int64_t k = 0; k < nnz; ++k)
    if (!std::isfinite(v[k])) return ctx.fail(VSHE_E_NAN, "matrix entry " + std::to_string(k));
  for (int64_t i = 0; i < n; ++i)
    if (!std::isfinite(rhs[i])) return ctx.fail(VSHE_E_NAN, "rhs entry " + std::to_string(i));
  cudaError_t e;
  d_rp = (int64_t *)arena.alloc(sizeof(int64_t) * size_t(n + 1), e);
  if (!d_rp) return ctx.cuda_fail(e, "cudaMalloc rp");
  d_ci = (int32_t *)arena.alloc(sizeof(int32_t) * size_t(nnz), e);
  if (!d_ci) return ctx.cuda_fail(e, "cudaMalloc ci");
  d_av64 = (double *)arena.alloc(sizeof(double) * size_t(nnz), e);
  if (!d_av64) return ctx.cuda_fail(e, "cudaMalloc values");
  d_b64 = (double *)arena.alloc(sizeof(double) * size_t(n), e);
  if (!d_b64) return ctx.cuda_fail(e, "cudaMalloc rhs");
  if ((e = cudaMemcpyAsync(d_rp, rp.data(), sizeof(int64_t) * rp.size(), cudaMemcpyHostToDevice, ctx.stream)) != cudaSuccess) return ctx.cuda_fail(e, "upload rp");
  if ((e = cudaMemcpyAsync(d_ci, ci.data(), sizeof(int32_t) * ci.size(), cudaMemcpyHostToDevice, ctx.stream)) != cudaSuccess) return ctx.cuda_fail(e, "upload ci");
  int rc = setup_pattern(ctx, v);
  if (rc) return rc;
  rc = set_values(ctx, v, rhs);
  if (rc) return rc;
  if ((e = cudaStreamSynchronize(ctx.stream)) != cudaSuccess) return ctx.cuda_fail(e, "upload");
  return VSHE_OK;
}

int System::create_borrowed(Ctx &ctx, int64_t n_, int64_t nnz_, const int64_t *rp_, const int32_t *ci_, int64_t *d_rp_,
                            int32_t *d_ci_, double *d_val, double *d_rhs, const vshe_solve_opts &o, const double *host_val) {
  int rc = init_borrowed(ctx, n_, nnz_, rp_, ci_, d_rp_, d_ci_, d_val, d_rhs, o);
  if (rc) return rc;
  return setup_pattern(ctx, host_val);
}

int System::init_borrowed(Ctx &ctx, int64_t n_, int64_t nnz_, const int64_t *rp_, const int32_t *ci_, int64_t *d_rp_,
                          int32_t *d_ci_, double *d_val, double *d_rhs, const vshe_solve_opts &o) {
  n = n_; nnz = nnz_; opts = o; borrowed = true;
  if (n <= 0 || nnz <= 0) return ctx.fail(VSHE_E_INVALID_ARGUMENT, "empty system");
  if (n >= (int64_t(1) << 31) - 64) return ctx.fail(VSHE_E_INVALID_ARGUMENT, "more than 2^31 - 64 rows");
  rp.assign(rp_, rp_ + n + 1);
  ci.assign(ci_, ci_ + nnz);
  for (int64_t i = 0; i < n; ++i)
    if (rp[i + 1] == rp[i]) return ctx.fail(VSHE_E_EMPTY_ROW, "row " + std::to_string(i));
  d_rp = d_rp_; d_ci = d_ci_; d_av64 = d_val; d_b64 = d_rhs;
  bnorm_host = 1.0;  // the trivial-rhs test uses the device-side norm
  return VSHE_OK;
}

// Host threads of the library's host work (vshe_set_host_threads; 0: up to 16).
static std::atomic<int> g_host_threads{0};

// Host threads for n items in chunks of at least `grain`: up to 16 (or the vshe_set_host_threads cap).
static int64_t host_threads(int64_t n, int64_t grain) {
  const int64_t hw = std::max<int64_t>(1, int64_t(std::thread::hardware_concurrency()));
  const int cap = g_host_threads.load();
  const int64_t tmax = cap > 0 ? int64_t(cap) : std::min<int64_t>(hw, 16);
  return std::min<int64_t>(tmax, std::max<int64_t>(1, n / std::max<int64_t>(grain, 1)));
}

// Runs fn(begin, end) over [0, n) in contiguous chunks of at least `grain` on up to 16 host
// threads (the host-side checks of the drop-in call on arrays of hundreds of MB, the layout).
static void host_parallel(int64_t n, int64_t grain, const std::function<void(int64_t, int64_t)> &fn) {
  const int64_t T = host_threads(n, grain);
  if (T <= 1) { fn(0, n); return; }
  std::vector<std::thread> th;
  for (int64_t t = 0; t < T; ++t) th.emplace_back(fn, n * t / T, n * (t + 1) / T);
  for (auto &x : th) x.join();
}

// Runs fn(r0, r1) over the runs of a row partition (run r = rows [runs[r], runs[r + 1])) on the
// host threads, in contiguous chunks of whole runs that hold about the same number of rows.
static void host_parallel_runs(const std::vector<int64_t> &runs, const std::function<void(int64_t, int64_t)> &fn) {
  const int64_t nruns = int64_t(runs.size()) - 1;
  if (nruns <= 0) return;
  const int64_t T = host_threads(nruns, 1);
  if (T <= 1) { fn(0, nruns); return; }
  const int64_t first = runs.front(), rows = runs.back() - runs.front();
  std::vector<int64_t> cut(1, 0);
  for (int64_t t = 1; t < T; ++t) {
    const int64_t r = int64_t(std::lower_bound(runs.begin(), runs.end() - 1, first + rows * t / T) - runs.begin());
    if (r > cut.back() && r < nruns) cut.push_back(r);
  }
  cut.push_back(nruns);
  std::vector<std::thread> th;
  for (size_t c = 0; c + 1 < cut.size(); ++c) th.emplace_back(fn, cut[c], cut[c + 1]);
  for (auto &x : th) x.join();
}

// Transpose of the pattern (rp, ci) of n rows over n columns: tp (n + 1 offsets) and tr, the rows
// holding each column, ascending.  Each host thread owns a range of columns and scans all rows
// for them: no atomics, and every column's rows come out in row order.
static void transpose_pattern(int64_t n, const int64_t *rp, const int32_t *ci, std::vector<int64_t> &tp, std::vector<int32_t> &tr) {
  const int64_t T = host_threads(n, int64_t(1) << 16);
  tp.assign(size_t(n) + 1, 0);
  auto own = [&](int64_t t, auto &&fn) {
    const uint32_t c0 = uint32_t(n * t / T), w = uint32_t(n * (t + 1) / T) - c0;
    for (int64_t i = 0; i < n; ++i)
      for (int64_t k = rp[i]; k < rp[i + 1]; ++k)
        if (uint32_t(ci[k]) - c0 < w) fn(i, ci[k]);
  };
  host_parallel(T, 1, [&](int64_t t0, int64_t t1) {
    for (int64_t t = t0; t < t1; ++t) own(t, [&](int64_t, int32_t c) { tp[size_t(c) + 1]++; });
  });
  for (int64_t i = 0; i < n; ++i) tp[size_t(i) + 1] += tp[size_t(i)];
  tr.resize(size_t(tp[size_t(n)]));
  std::vector<int64_t> cur(tp.begin(), tp.end() - 1);
  host_parallel(T, 1, [&](int64_t t0, int64_t t1) {
    for (int64_t t = t0; t < t1; ++t) own(t, [&](int64_t i, int32_t c) { tr[size_t(cur[size_t(c)]++)] = int32_t(i); });
  });
}

// Stable counting sort of seq by key(x) in [0, range): equal keys keep their order.
template <class Key>
static void counting_sort_by(std::vector<int32_t> &seq, int64_t range, Key key) {
  if (range <= 1) return;
  std::vector<int64_t> pos(size_t(range) + 1, 0);
  for (int32_t x : seq) pos[size_t(key(x)) + 1]++;
  for (int64_t k = 0; k < range; ++k) pos[size_t(k) + 1] += pos[size_t(k)];
  std::vector<int32_t> out(seq.size());
  for (int32_t x : seq) out[size_t(pos[size_t(key(x))]++)] = x;
  seq.swap(out);
}

// First index in [0, n) whose value is not finite, or n.
static int64_t first_nonfinite(const double *v, int64_t n) {
  std::atomic<int64_t> first{n};
  host_parallel(n, int64_t(1) << 20, [&](int64_t a, int64_t b) {
    for (int64_t k = a; k < b && k < first.load(std::memory_order_relaxed); ++k)
      if (!std::isfinite(v[k])) {
        int64_t cur = first.load();
        while (k < cur && !first.compare_exchange_weak(cur, k)) {}
        return;
      }
  });
  return first.load();
}

// memcmp(a, b, bytes) == 0, on several host threads for large arrays.
static bool host_equal(const void *a, const void *b, size_t bytes) {
  std::atomic<bool> eq{true};
  host_parallel(int64_t(bytes), int64_t(1) << 24, [&](int64_t x, int64_t y) {
    if (eq.load(std::memory_order_relaxed) && std::memcmp((const char *)a + x, (const char *)b + x, size_t(y - x)) != 0) eq = false;
  });
  return eq.load();
}

int System::set_values(Ctx &ctx, const double *v, const double *rhs) {
  cudaStream_t s = ctx.stream;
  cudaError_t e;
  const int64_t bad = first_nonfinite(v, nnz);
  if (bad < nnz) return ctx.fail(VSHE_E_NAN, "matrix entry " + std::to_string(bad));
  bnorm_host = 0.0;
  for (int64_t i = 0; i < n; ++i) {
    if (!std::isfinite(rhs[i])) return ctx.fail(VSHE_E_NAN, "rhs entry " + std::to_string(i));
    bnorm_host += rhs[i] * rhs[i];
  }
  bnorm_host = std::sqrt(bnorm_host);
  if ((e = cudaMemcpyAsync(d_av64, v, sizeof(double) * size_t(nnz), cudaMemcpyHostToDevice, s)) != cudaSuccess) return ctx.cuda_fail(e, "upload values");
  if ((e = cudaMemcpyAsync(d_b64, rhs, sizeof(double) * size_t(n), cudaMemcpyHostToDevice, s)) != cudaSuccess) return ctx.cuda_fail(e, "upload rhs");
  return VSHE_OK;
}

void System::prepare(Ctx &ctx) {
  cudaStream_t s = ctx.stream;
  vk_gather_values(padA, d_amapS, d_av64, d_aval, s);
  if (has_pc) vk_gather_values(nnzF, d_amap, d_av64, d_lu64, s);
  vk_permute(n, d_perm, d_b64, d_bp, 1, s);
}


// Contiguous runs of equal block id: run r = rows [runs[r], runs[r + 1]).
static std::vector<int64_t> block_runs(const std::vector<int32_t> &blk) {
  std::vector<int64_t> runs(1, 0);
  for (size_t i = 1; i < blk.size(); ++i)
    if (blk[i] != blk[i - 1]) runs.push_back(int64_t(i));
  runs.push_back(int64_t(blk.size()));
  return runs;
}

// Greedy colouring of the symmetrised pattern within blocks: distance 1 (coupled rows differ)
// or distance 2 (rows with a common neighbour differ as well).  Rows are coloured in index
// order; a row's colour depends only on rows of its own block, so runs of rows of one block are
// coloured on several host threads with the same result.
static void greedy_colours(int64_t n, const std::vector<int64_t> &rp, const std::vector<int32_t> &ci, const std::vector<int32_t> &blk,
                           std::vector<int32_t> &col, int distance) {
  // neighbours of every row in the symmetrised pattern, each once and without the row itself (a
  // row's colour depends only on the set of colours around it): the union of its row and its
  // column, on the host threads
  std::vector<int64_t> sp(size_t(n) + 1, 0);
  std::vector<int32_t> sj;
  {
    std::vector<int64_t> tcnt;
    std::vector<int32_t> tci;
    transpose_pattern(n, rp.data(), ci.data(), tcnt, tci);
    auto gather = [&](int64_t i, std::vector<int32_t> &v) {
      v.clear();
      for (int64_t k = rp[i]; k < rp[i + 1]; ++k) if (ci[k] != i) v.push_back(ci[k]);
      for (int64_t k = tcnt[size_t(i)]; k < tcnt[size_t(i) + 1]; ++k) if (tci[size_t(k)] != i) v.push_back(tci[size_t(k)]);
      std::sort(v.begin(), v.end());
      v.erase(std::unique(v.begin(), v.end()), v.end());
    };
    host_parallel(n, int64_t(1) << 16, [&](int64_t a, int64_t b) {
      std::vector<int32_t> v;
      for (int64_t i = a; i < b; ++i) { gather(i, v); sp[size_t(i) + 1] = int64_t(v.size()); }
    });
    for (int64_t i = 0; i < n; ++i) sp[size_t(i) + 1] += sp[size_t(i)];
    sj.resize(size_t(sp[size_t(n)]));
    host_parallel(n, int64_t(1) << 16, [&](int64_t a, int64_t b) {
      std::vector<int32_t> v;
      for (int64_t i = a; i < b; ++i) { gather(i, v); std::copy(v.begin(), v.end(), sj.begin() + sp[size_t(i)]); }
    });
  }
  col.assign(size_t(n), -1);
  auto neighbours = [&](int64_t i, auto &&fn) {
    for (int64_t k = sp[size_t(i)]; k < sp[size_t(i) + 1]; ++k) fn(sj[size_t(k)]);
  };
  const std::vector<int64_t> runs = block_runs(blk);
  host_parallel_runs(runs, [&](int64_t r0, int64_t r1) {
    std::vector<int64_t> mark(64, -1);
    for (int64_t i = runs[size_t(r0)]; i < runs[size_t(r1)]; ++i) {
      auto visit = [&](int32_t j) {
        if (j == i || blk[size_t(j)] != blk[size_t(i)] || col[size_t(j)] < 0) return;
        int32_t c = col[size_t(j)];
        if (c >= int32_t(mark.size())) mark.resize(size_t(c) + 1, -1);
        mark[size_t(c)] = i;
      };
      neighbours(i, [&](int32_t j) {
        visit(j);
        if (distance > 1 && blk[size_t(j)] == blk[size_t(i)]) neighbours(j, visit);
      });
      int32_t c = 0;
      while (c < int32_t(mark.size()) && mark[size_t(c)] == i) ++c;
      col[size_t(i)] = c;
    }
  });
}

// SELL-32 layout of a row sequence rows[t] (t = 0..m-1) made of groups: group g is the run
// [gstart[g], gstart[g+1]) of level glev[g] (non-decreasing) and one preconditioner block.
// Slices of 32 rows never straddle a group; width of a slice = its longest row.  Returns the slot
// offsets (one per slice + 1), the slice starts in t, the first slice of every level
// (lvl_slices, nlev + 1 entries) and of every group (grp_slices, groups + 1 entries).
static void sell_layout(const std::vector<int64_t> &len_of_t, const std::vector<int64_t> &gstart, const std::vector<int32_t> &glev,
                        int32_t nlev, std::vector<int64_t> &off, std::vector<int64_t> &start, std::vector<int64_t> &lvl_slices,
                        std::vector<int64_t> &grp_slices) {
  off.assign(1, 0);
  start.clear();
  lvl_slices.assign(size_t(nlev) + 1, 0);
  grp_slices.clear();
  int32_t lv = 0;
  for (size_t g = 0; g + 1 < gstart.size(); ++g) {
    while (lv < glev[g]) lvl_slices[size_t(++lv)] = int64_t(start.size());
    grp_slices.push_back(int64_t(start.size()));
    for (int64_t t = gstart[g]; t < gstart[g + 1]; t += 32) {
      const int64_t e = std::min<int64_t>(t + 32, gstart[g + 1]);
      int64_t w = 0;
      for (int64_t u = t; u < e; ++u) w = std::max(w, len_of_t[size_t(u)]);
      start.push_back(t);
      off.push_back(off.back() + 32 * w);
    }
  }
  grp_slices.push_back(int64_t(start.size()));
  while (lv < nlev) lvl_slices[size_t(++lv)] = int64_t(start.size());
  start.push_back(gstart.empty() ? 0 : gstart.back());
}

// Groups of a row sequence: maximal runs of equal (level, block); the sequence is sorted by
// level, then block.
static void row_groups(int64_t m, const std::function<int32_t(int64_t)> &lev_of, const std::function<int32_t(int64_t)> &blk_of,
                       std::vector<int64_t> &gstart, std::vector<int32_t> &glev, std::vector<int32_t> &gblk) {
  gstart.clear(); glev.clear(); gblk.clear();
  for (int64_t t = 0; t < m; ++t) {
    const int32_t l = lev_of(t), b = blk_of(t);
    if (t == 0 || l != glev.back() || b != gblk.back()) { gstart.push_back(t); glev.push_back(l); gblk.push_back(b); }
  }
  gstart.push_back(m);
}

int Layout::build(int64_t n, int64_t nnz, const std::vector<int64_t> &rp, const std::vector<int32_t> &ci,
                  const vshe_solve_opts &opts, const double *values, std::string &err) {
  const bool has_pc = opts.precond != VSHE_PRECOND_NONE;
  const bool ilut = opts.precond == VSHE_PRECOND_ILUT;
  if (ilut && !values) { err = "the ILUT pattern needs the matrix values at creation"; return VSHE_E_INVALID_ARGUMENT; }
  // block ids in the caller's order
  std::vector<int32_t> blk0((size_t)(n), 0);
  // (block-ILU, and ILUT restricted to the blocks when the caller gives them)
  if ((opts.precond == VSHE_PRECOND_BLOCK_ILU0 || opts.precond == VSHE_PRECOND_ILUT) && opts.n_blocks > 0 && opts.block_ptr) {
    const int64_t *bp = opts.block_ptr;
    if (bp[0] != 0 || bp[opts.n_blocks] != n) { err = "block_ptr must span [0, n]"; return VSHE_E_INVALID_ARGUMENT; }
    for (int64_t b = 0; b < opts.n_blocks; ++b) {
      if (bp[b + 1] < bp[b]) { err = "block_ptr not monotone"; return VSHE_E_INVALID_ARGUMENT; }
      for (int64_t i = bp[b]; i < bp[b + 1]; ++i) blk0[size_t(i)] = int32_t(b);
    }
  }
  const int64_t nblk = int64_t(*std::max_element(blk0.begin(), blk0.end())) + 1;
  // base ordering of the preconditioner: base[i] = caller row at base position i
  std::vector<int32_t> base((size_t)n);
  if (opts.perm) {
    std::vector<char> seen((size_t)(n), 0);
    for (int64_t i = 0; i < n; ++i) {
      int32_t o = opts.perm[i];
      if (o < 0 || o >= n || seen[size_t(o)]) { err = "perm is not a permutation"; return VSHE_E_INVALID_ARGUMENT; }
      seen[size_t(o)] = 1;
      base[size_t(i)] = o;
    }
  } else if (has_pc && opts.ordering == VSHE_ORDER_MULTICOLOR) {
    std::vector<int32_t> col;
    // ILU(k > 0): rows two steps apart get different colours too, so that the fill (which
    // couples such rows) does not chain rows of one colour into extra levels
    greedy_colours(n, rp, ci, blk0, col, opts.fill_level > 0 ? 2 : 1);
    // by block, then colour, then row (two stable counting passes)
    std::iota(base.begin(), base.end(), 0);
    counting_sort_by(base, int64_t(*std::max_element(col.begin(), col.end())) + 1, [&](int32_t a) { return col[size_t(a)]; });
    counting_sort_by(base, nblk, [&](int32_t a) { return blk0[size_t(a)]; });
  } else {
    std::iota(base.begin(), base.end(), 0);
  }
  std::vector<int32_t> binv((size_t)n);
  for (int64_t i = 0; i < n; ++i) binv[size_t(base[size_t(i)])] = int32_t(i);

  // Blocks in base order, as runs of base positions; when every block is one run, the phases in
  // which a row reads only earlier rows of its own block run on several host threads.
  std::vector<int32_t> bblk((size_t)n);
  for (int64_t i = 0; i < n; ++i) bblk[size_t(i)] = blk0[size_t(base[size_t(i)])];
  const std::vector<int64_t> runs = block_runs(bblk);
  const int64_t nruns = int64_t(runs.size()) - 1;
  bool contiguous = true;
  {
    std::vector<char> seen;
    for (int64_t r = 0; r < nruns && contiguous; ++r) {
      const int32_t b = bblk[size_t(runs[size_t(r)])];
      if (b >= int32_t(seen.size())) seen.resize(size_t(b) + 1, 0);
      if (seen[size_t(b)]) contiguous = false;
      seen[size_t(b)] = 1;
    }
  }

  // Pattern of the incomplete factor F in base order (row i is caller row base[i]; columns are
  // base positions, ascending; fsrc = entry of A, -1 for fill): A's entries and, for ILU(k) with
  // k = fill_level > 0, the fill of levels <= k from the symbolic phase of Saad's Alg. 10.5 run
  // in base order, fill kept inside the row's block; for ILUT, the positions that pass its drop
  // test (below).
  std::vector<int64_t> frp;
  std::vector<int32_t> fci;
  std::vector<int64_t> fsrc;
  const int kfill = has_pc && !ilut ? std::max(0, int(opts.fill_level)) : 0;
  {
    // base-order rows of A: (base column, entry)
    std::vector<int64_t> brp((size_t)n + 1, 0);
    for (int64_t i = 0; i < n; ++i) brp[size_t(i) + 1] = brp[size_t(i)] + (rp[size_t(base[size_t(i)]) + 1] - rp[size_t(base[size_t(i)])]);
    std::vector<std::pair<int32_t, int64_t>> bent((size_t)nnz);
    host_parallel(n, int64_t(1) << 16, [&](int64_t i0, int64_t i1) {
      for (int64_t i = i0; i < i1; ++i) {
        const int32_t o = base[size_t(i)];
        int64_t p = brp[size_t(i)];
        for (int64_t k = rp[size_t(o)]; k < rp[size_t(o) + 1]; ++k) bent[size_t(p++)] = {binv[size_t(ci[size_t(k)])], k};
        std::sort(bent.begin() + brp[size_t(i)], bent.begin() + p);
      }
    });
    if (kfill == 0 && !ilut) {
      frp.swap(brp);
      fci.resize((size_t)nnz);
      fsrc.resize((size_t)nnz);
      host_parallel(nnz, int64_t(1) << 20, [&](int64_t k0, int64_t k1) {
        for (int64_t k = k0; k < k1; ++k) { fci[size_t(k)] = bent[size_t(k)].first; fsrc[size_t(k)] = bent[size_t(k)].second; }
      });
    } else {
    // rows of F in base order, (base column, entry or -1), in one store per host thread: a store
    // holds the consecutive rows from row0 on, one after the other; rcnt[i] = entries of row i
    struct RowStore {
      int64_t row0 = 0;
      std::vector<int32_t> col;
      std::vector<int64_t> src;
    };
    std::vector<std::unique_ptr<RowStore>> rstore;
    std::mutex rmu;
    std::vector<int64_t> rcnt((size_t)n, 0);
    // a new store for the rows from row0 on (taken under the lock: another thread may grow
    // rstore meanwhile)
    auto new_store = [&](int64_t row0) {
      std::lock_guard<std::mutex> lk(rmu);
      rstore.emplace_back(new RowStore);
      rstore.back()->row0 = row0;
      return rstore.back().get();
    };
    if (ilut) {
      // ILUT(p, tau), Saad Alg. 10.6, in base order: the row is eliminated with the kept rows
      // above it in increasing column order; a multiplier or entry below tau * ||a_i|| is
      // dropped, then the p largest of L and of U are kept (the diagonal always).  Only the
      // pattern is kept here: every position that survives the tau test, joined with A's.  The
      // device repeats the same elimination with the same two dropping rules inside that
      // pattern (k_ilut), which reproduces ILUT for the values seen here.  With blocks the
      // elimination stays inside the row's block (no elimination with, and no fill from, rows of
      // other blocks), as the device's does; tau * ||a_i|| uses the whole row.
      const int pkeep = opts.ilut_entries > 0 ? opts.ilut_entries : 60;
      const double tau = opts.ilut_drop > 0 ? opts.ilut_drop : 1e-4;
      //
      // With blocks that are runs of base positions, each host thread eliminates whole blocks.
      // Otherwise rows are eliminated on the host threads in claims of consecutive rows, in
      // increasing order.
      // A row reads only rows above it: before it reads row k's pivot and kept upper part it waits
      // until row k is final (done[k], set with release after they are written).  The row holding
      // the first unfinished position never waits, so the elimination always progresses, and every
      // row computes exactly what the serial elimination computes.
      std::vector<std::vector<int32_t>> ucol((size_t)n);   // kept upper part of each row
      std::vector<std::vector<double>> uval((size_t)n);
      std::vector<double> udiag((size_t)n, 0.0);
      std::unique_ptr<std::atomic<uint8_t>[]> done(new std::atomic<uint8_t>[size_t(n)]);
      for (int64_t i = 0; i < n; ++i) done[size_t(i)].store(0, std::memory_order_relaxed);
      std::atomic<int64_t> next_claim{0};
      constexpr int64_t kClaimRows = 64;
      // eliminates the row ranges that next() hands out, one after the other
      auto eliminate = [&](const std::function<bool(int64_t &, int64_t &)> &next) {
        // dense scratch over all columns, calloc'd: a thread touches only the pages its rows reach
        std::unique_ptr<double, void (*)(void *)> wbuf((double *)std::calloc(size_t(n), sizeof(double)), std::free);
        std::unique_ptr<char, void (*)(void *)> nzbuf((char *)std::calloc(size_t(n), 1), std::free);
        if (!wbuf || !nzbuf) throw std::bad_alloc();
        double *w = wbuf.get();
        char *nz = nzbuf.get();
        std::vector<int32_t> cols, heap;
        std::vector<std::pair<double, int32_t>> lo, up;
        int64_t c0 = 0, c1 = 0;
        while (next(c0, c1)) {
          RowStore &st = *new_store(c0);
          for (int64_t i = c0; i < c1; ++i) {
            cols.clear(); heap.clear();
            double rn = 0.0;
            for (int64_t k = brp[size_t(i)]; k < brp[size_t(i) + 1]; ++k) {
              const int32_t j = bent[size_t(k)].first;
              const double a = values[bent[size_t(k)].second];
              w[size_t(j)] = a; nz[size_t(j)] = 1; cols.push_back(j);
              rn += a * a;
              if (j < i) heap.push_back(j);
            }
            const double ti = tau * std::sqrt(rn);
            if (!nz[size_t(i)]) { nz[size_t(i)] = 1; w[size_t(i)] = 0.0; cols.push_back(int32_t(i)); }
            std::make_heap(heap.begin(), heap.end(), std::greater<int32_t>());
            int32_t last = -1;
            while (!heap.empty()) {
              std::pop_heap(heap.begin(), heap.end(), std::greater<int32_t>());
              const int32_t k = heap.back(); heap.pop_back();
              if (k == last) continue;
              last = k;
              if (bblk[size_t(k)] != bblk[size_t(i)]) continue;  // another block: no elimination
              while (!done[size_t(k)].load(std::memory_order_acquire)) std::this_thread::yield();
              if (udiag[size_t(k)] == 0.0) { w[size_t(k)] = 0.0; continue; }
              const double wk = w[size_t(k)] / udiag[size_t(k)];
              if (std::fabs(wk) < ti) { w[size_t(k)] = 0.0; continue; }
              w[size_t(k)] = wk;
              const std::vector<int32_t> &uck = ucol[size_t(k)];
              const std::vector<double> &uvk = uval[size_t(k)];
              for (size_t kk = 0; kk < uck.size(); ++kk) {
                const int32_t j = uck[kk];
                if (bblk[size_t(j)] != bblk[size_t(i)]) continue;
                if (!nz[size_t(j)]) {
                  nz[size_t(j)] = 1; w[size_t(j)] = 0.0; cols.push_back(j);
                  if (j < i) { heap.push_back(j); std::push_heap(heap.begin(), heap.end(), std::greater<int32_t>()); }
                }
                w[size_t(j)] -= wk * uvk[kk];
              }
            }
            lo.clear(); up.clear();
            for (int32_t j : cols) {
              if (j == i || w[size_t(j)] == 0.0 || std::fabs(w[size_t(j)]) < ti) continue;
              (j < i ? lo : up).push_back({std::fabs(w[size_t(j)]), j});
            }
            auto keep = [&](std::vector<std::pair<double, int32_t>> &v) {
              if (int(v.size()) > pkeep) {
                std::nth_element(v.begin(), v.begin() + pkeep, v.end(),
                [](const std::pair<double, int32_t> &a, const std::pair<double, int32_t> &b) { return a.first > b.first; });
                v.resize(size_t(pkeep));
              }
            };
            // the factor pattern of row i: every entry that survived the tau test (the device applies
            // the p-largest rule itself, and multipliers beyond the p largest still take part in the
            // elimination), the diagonal and A's own entries
            std::vector<int32_t> pat;
            for (auto &e : lo) pat.push_back(e.second);
            pat.push_back(int32_t(i));
            for (auto &e : up) pat.push_back(e.second);
            keep(lo); keep(up);
            double d = w[size_t(i)];
            if (d == 0.0) d = ti > 0.0 ? ti : 1.0;
            udiag[size_t(i)] = d;
            std::sort(up.begin(), up.end(), [](const std::pair<double, int32_t> &a, const std::pair<double, int32_t> &b) { return a.second < b.second; });
            for (auto &e : up) { ucol[size_t(i)].push_back(e.second); uval[size_t(i)].push_back(w[size_t(e.second)]); }
            done[size_t(i)].store(1, std::memory_order_release);
            for (int64_t k = brp[size_t(i)]; k < brp[size_t(i) + 1]; ++k) pat.push_back(bent[size_t(k)].first);
            std::sort(pat.begin(), pat.end());
            pat.erase(std::unique(pat.begin(), pat.end()), pat.end());
            const size_t before = st.col.size();
            int64_t ka = brp[size_t(i)];
            for (int32_t j : pat) {
              while (ka < brp[size_t(i) + 1] && bent[size_t(ka)].first < j) ++ka;
              const bool in_a = ka < brp[size_t(i) + 1] && bent[size_t(ka)].first == j;
              st.col.push_back(j);
              st.src.push_back(in_a ? bent[size_t(ka)].second : int64_t(-1));
            }
            rcnt[size_t(i)] = int64_t(st.col.size() - before);
            for (int32_t j : cols) { nz[size_t(j)] = 0; w[size_t(j)] = 0.0; }
          }
        }
      };
      if (contiguous && nruns > 1) {
        // every block is one run of base positions and a row reads only rows of its block: whole
        // blocks per thread, so no row waits
        host_parallel_runs(runs, [&](int64_t r0, int64_t r1) {
          bool given = false;
          eliminate([&](int64_t &a, int64_t &b) {
            if (given) return false;
            given = true;
            a = runs[size_t(r0)];
            b = runs[size_t(r1)];
            return true;
          });
        });
      } else {
        host_parallel(host_threads(n, kClaimRows * 16), 1, [&](int64_t, int64_t) {
          eliminate([&](int64_t &a, int64_t &b) {
            a = next_claim.fetch_add(kClaimRows);
            if (a >= n) return false;
            b = std::min<int64_t>(n, a + kClaimRows);
            return true;
          });
        });
      }
    } else {
      // symbolic ILU(k): the final rows' upper parts (column, level) feed later rows.  A row
      // reads only earlier rows of its own block, so when every block is one run of base
      // positions the runs are processed on several host threads (each with its own scratch
      // and its own store of upper parts), with the same result.
      std::vector<int64_t> ub((size_t)n, 0), ue((size_t)n, 0);  // upper part of row k: [ub[k], ue[k]) in its thread's store
      auto symbolic = [&](int64_t r0, int64_t r1) {
        std::vector<int32_t> ucolv, ulevv;
        // scratch over all columns: lvl1[j] = level of fill of column j + 1 (0: not in the row),
        // src[j] its entry of A; calloc'd and left uninitialised, so that a thread touches only the
        // pages of the columns its rows reach
        std::unique_ptr<int32_t, void (*)(void *)> lvl1((int32_t *)std::calloc(size_t(n), sizeof(int32_t)), std::free);
        std::unique_ptr<int64_t[]> src(new int64_t[size_t(n)]);
        if (!lvl1) throw std::bad_alloc();
        int32_t *lvl = lvl1.get();
        RowStore &st = *new_store(runs[size_t(r0)]);
        std::vector<int32_t> cols, heap;
        for (int64_t i = runs[size_t(r0)]; i < runs[size_t(r1)]; ++i) {
          const int32_t bi = bblk[size_t(i)];
          cols.clear(); heap.clear();
          for (int64_t k = brp[size_t(i)]; k < brp[size_t(i) + 1]; ++k) {
            const int32_t j = bent[size_t(k)].first;
            lvl[size_t(j)] = 1; src[size_t(j)] = bent[size_t(k)].second; cols.push_back(j);
            if (j < i) heap.push_back(j);
          }
          std::make_heap(heap.begin(), heap.end(), std::greater<int32_t>());
          int32_t last = -1;
          while (!heap.empty()) {
            std::pop_heap(heap.begin(), heap.end(), std::greater<int32_t>());
            const int32_t k = heap.back(); heap.pop_back();
            if (k == last) continue;
            last = k;
            if (bblk[size_t(k)] != bi) continue;
            const int32_t lik = lvl[size_t(k)] - 1;
            for (int64_t kk = ub[size_t(k)]; kk < ue[size_t(k)]; ++kk) {
              const int32_t j = ucolv[size_t(kk)];
              if (bblk[size_t(j)] != bi) continue;
              const int32_t l = lik + ulevv[size_t(kk)] + 1;
              if (l > kfill) continue;
              if (lvl[size_t(j)] == 0) {
                lvl[size_t(j)] = l + 1; src[size_t(j)] = -1; cols.push_back(j);
                if (j < i) { heap.push_back(j); std::push_heap(heap.begin(), heap.end(), std::greater<int32_t>()); }
              } else if (l < lvl[size_t(j)] - 1) {
                lvl[size_t(j)] = l + 1;
              }
            }
          }
          std::sort(cols.begin(), cols.end());
          ub[size_t(i)] = int64_t(ucolv.size());
          for (int32_t j : cols) {
            st.col.push_back(j);
            st.src.push_back(src[size_t(j)]);
            if (j > i) { ucolv.push_back(j); ulevv.push_back(lvl[size_t(j)] - 1); }
            lvl[size_t(j)] = 0;
          }
          rcnt[size_t(i)] = int64_t(cols.size());
          ue[size_t(i)] = int64_t(ucolv.size());
        }
      };
      if (contiguous) host_parallel_runs(runs, symbolic);
      else symbolic(0, nruns);
    }
    // one CSR in base order: the stores' rows are consecutive and in ascending base column, so
    // each store is one contiguous piece of it
    frp.assign((size_t)n + 1, 0);
    for (int64_t i = 0; i < n; ++i) frp[size_t(i) + 1] = frp[size_t(i)] + rcnt[size_t(i)];
    {
      size_t stored = 0;
      for (const auto &st : rstore) stored += st->col.size();
      if (stored != size_t(frp[size_t(n)])) { err = "factor pattern stores do not tile the rows"; return VSHE_E_INVALID_ARGUMENT; }
    }
    fci.resize(size_t(frp[size_t(n)]));
    fsrc.resize(size_t(frp[size_t(n)]));
    host_parallel(int64_t(rstore.size()), 1, [&](int64_t s0, int64_t s1) {
      for (int64_t q = s0; q < s1; ++q) {
        const RowStore &st = *rstore[size_t(q)];
        std::copy(st.col.begin(), st.col.end(), fci.begin() + frp[size_t(st.row0)]);
        std::copy(st.src.begin(), st.src.end(), fsrc.begin() + frp[size_t(st.row0)]);
      }
    });
    }
  }
  const int64_t fnnz = frp[size_t(n)];
  nnzF = fnnz;

  // Forward levels over the symmetrised, block-restricted graph of F in base order: a row's
  // level is one more than the highest level of any coupled (F_ij or F_ji != 0) earlier row of
  // its block.  Sorting by these levels keeps the relative order of every coupled pair, so the
  // incomplete factorisation in the sorted order is the one in the base order, relabelled.
  std::vector<int32_t> lev((size_t)n, 0);   // by caller row
  nlevL = 1;
  if (has_pc) {
    std::vector<int64_t> tp;
    std::vector<int32_t> tr;
    transpose_pattern(n, frp.data(), fci.data(), tp, tr);
    std::vector<int32_t> levb((size_t)n, 0);  // by base position
    std::mutex mu;
    auto level = [&](int64_t r0, int64_t r1) {
      int32_t nl = 1;
      for (int64_t i = runs[size_t(r0)]; i < runs[size_t(r1)]; ++i) {
        int32_t m = -1;
        for (int64_t k = frp[size_t(i)]; k < frp[size_t(i) + 1]; ++k) {
          const int32_t j = fci[size_t(k)];
          if (j < i && bblk[size_t(j)] == bblk[size_t(i)]) m = std::max(m, levb[size_t(j)]);
        }
        for (int64_t k = tp[size_t(i)]; k < tp[size_t(i) + 1]; ++k) {
          const int32_t j = tr[size_t(k)];
          if (j < i && bblk[size_t(j)] == bblk[size_t(i)]) m = std::max(m, levb[size_t(j)]);
        }
        levb[size_t(i)] = m + 1;
        nl = std::max(nl, m + 2);
      }
      std::lock_guard<std::mutex> lk(mu);
      nlevL = std::max(nlevL, nl);
    };
    if (contiguous) host_parallel_runs(runs, level);
    else level(0, nruns);
    for (int64_t i = 0; i < n; ++i) lev[size_t(base[size_t(i)])] = levb[size_t(i)];
  }
  // solver order: by level, then block (each block's rows of a level are one run, which the
  // per-block sweeps walk), then longest rows first (less SELL padding), then by the base
  // position of the row's first neighbour (the lanes of a slice then gather nearby entries:
  // 4 % faster sweeps on the 2D bar than base position), then base position
  // (two stable counting passes give (level, block) groups in base order; each group is then
  // sorted by the last three keys on the host threads)
  perm = base;
  std::vector<int32_t> nbk((size_t)n, 0);
  host_parallel(n, int64_t(1) << 16, [&](int64_t i0, int64_t i1) {
    for (int64_t i = i0; i < i1; ++i) {
      int32_t m = INT32_MAX;
      for (int64_t k = frp[size_t(i)]; k < frp[size_t(i) + 1]; ++k)
        if (fci[size_t(k)] != i) m = std::min(m, fci[size_t(k)]);
      nbk[size_t(base[size_t(i)])] = m;
    }
  });
  counting_sort_by(perm, nblk, [&](int32_t a) { return blk0[size_t(a)]; });
  counting_sort_by(perm, int64_t(nlevL), [&](int32_t a) { return lev[size_t(a)]; });
  {
    std::vector<int64_t> grp(1, 0);
    for (int64_t i = 1; i < n; ++i)
      if (lev[size_t(perm[size_t(i)])] != lev[size_t(perm[size_t(i) - 1])] || blk0[size_t(perm[size_t(i)])] != blk0[size_t(perm[size_t(i) - 1])])
        grp.push_back(i);
    grp.push_back(n);
    host_parallel_runs(grp, [&](int64_t g0, int64_t g1) {
      for (int64_t g = g0; g < g1; ++g)
        std::sort(perm.begin() + grp[size_t(g)], perm.begin() + grp[size_t(g) + 1], [&](int32_t a, int32_t b) {
          const int64_t la = rp[size_t(a) + 1] - rp[size_t(a)], lb = rp[size_t(b) + 1] - rp[size_t(b)];
          if (la != lb) return la > lb;
          if (nbk[size_t(a)] != nbk[size_t(b)]) return nbk[size_t(a)] < nbk[size_t(b)];
          return binv[size_t(a)] < binv[size_t(b)];
        });
    });
  }
  std::vector<int32_t> inv((size_t)(n));
  for (int64_t i = 0; i < n; ++i) inv[size_t(perm[size_t(i)])] = int32_t(i);
  blk.resize(size_t(n));
  for (int64_t i = 0; i < n; ++i) blk[size_t(i)] = blk0[size_t(perm[size_t(i)])];
  lvr.assign(size_t(nlevL) + 1, 0);
  for (int64_t i = 0; i < n; ++i) lvr[size_t(lev[size_t(i)]) + 1]++;
  for (size_t k = 1; k < lvr.size(); ++k) lvr[k] += lvr[k - 1];

  // solver-order CSR with the map back to A's entries
  prp.assign((size_t)n + 1, 0); pdiag.assign((size_t)n, -1); amap.assign((size_t)fnnz, 0);
  pci.assign((size_t)fnnz, 0);
  {
    // solver position of every base position
    std::vector<int32_t> sinv((size_t)n);
    for (int64_t i = 0; i < n; ++i) sinv[size_t(i)] = inv[size_t(base[size_t(i)])];
    for (int64_t i = 0; i < n; ++i) {
      const int32_t b = binv[size_t(perm[size_t(i)])];
      prp[size_t(i) + 1] = prp[size_t(i)] + (frp[size_t(b) + 1] - frp[size_t(b)]);
    }
    host_parallel(n, int64_t(1) << 16, [&](int64_t i0, int64_t i1) {
      // a row's columns are distinct: sort (solver column, position in the row) keys
      std::vector<uint64_t> key;
      for (int64_t i = i0; i < i1; ++i) {
        const int32_t b = binv[size_t(perm[size_t(i)])];
        const int64_t k0 = frp[size_t(b)];
        key.clear();
        for (int64_t k = k0; k < frp[size_t(b) + 1]; ++k) key.push_back((uint64_t(uint32_t(sinv[size_t(fci[size_t(k)])])) << 32) | uint64_t(k - k0));
        std::sort(key.begin(), key.end());
        int64_t p = prp[size_t(i)];
        for (uint64_t x : key) {
          const int32_t c = int32_t(x >> 32);
          if (c == i) pdiag[size_t(i)] = p;
          pci[size_t(p)] = c;
          amap[size_t(p)] = fsrc[size_t(k0 + int64_t(x & 0xffffffffu))];
          ++p;
        }
      }
    });
    if (has_pc)
      for (int64_t i = 0; i < n; ++i)
        if (pdiag[size_t(i)] < 0) { err = "no diagonal entry in row " + std::to_string(perm[size_t(i)]); return VSHE_E_ZERO_PIVOT; }
  }
  const int32_t PAD = int32_t(n);  // padding column: entry n of every vector stays 0

  // SELL-32 A in solver order: slices of 32 consecutive rows, A's own entries only (the fill of
  // an ILU(k) factor is not part of A)
  std::vector<int64_t> alvs;
  {
    std::vector<int64_t> len((size_t)n, 0);
    host_parallel(n, int64_t(1) << 16, [&](int64_t i0, int64_t i1) {
      for (int64_t i = i0; i < i1; ++i)
        for (int64_t p = prp[size_t(i)]; p < prp[size_t(i) + 1]; ++p) len[size_t(i)] += amap[size_t(p)] >= 0 ? 1 : 0;
    });
    std::vector<int64_t> one{0, n}, agrp;
    sell_layout(len, one, std::vector<int32_t>{0}, 1, aoff, astart, alvs, agrp);
  }
  nslA = int64_t(astart.size()) - 1;
  padA = aoff.back();
  amapS.assign((size_t)padA, -1);
  acol.assign((size_t)padA, PAD);
  host_parallel(nslA, int64_t(1) << 12, [&](int64_t j0, int64_t j1) {
    for (int64_t j = j0; j < j1; ++j) {
      for (int64_t i = astart[size_t(j)]; i < astart[size_t(j) + 1]; ++i) {
        const int lane = int(i - astart[size_t(j)]);
        int64_t kk = 0;
        for (int64_t p = prp[size_t(i)]; p < prp[size_t(i) + 1]; ++p) {
          if (amap[size_t(p)] < 0) continue;
          const int64_t slot = aoff[size_t(j)] + 32 * kk + lane;
          acol[size_t(slot)] = pci[size_t(p)];
          amapS[size_t(slot)] = amap[size_t(p)];
          ++kk;
        }
      }
    }
  });

  // factor layouts
  if (has_pc) {
    // forward sweep: rows of a level are contiguous; L entries = in-block columns left of the diagonal
    std::vector<int64_t> llen((size_t)n), ulen((size_t)n);
    host_parallel(n, int64_t(1) << 16, [&](int64_t i0, int64_t i1) {
      for (int64_t i = i0; i < i1; ++i) {
        int64_t cl = 0, cu = 0;
        for (int64_t k = prp[size_t(i)]; k < prp[size_t(i) + 1]; ++k) {
          if (blk[size_t(pci[size_t(k)])] != blk[size_t(i)]) continue;
          if (k < pdiag[size_t(i)]) ++cl; else if (k > pdiag[size_t(i)]) ++cu;
        }
        llen[size_t(i)] = cl; ulen[size_t(i)] = cu;
      }
    });
    {
      std::vector<int64_t> gs;
      std::vector<int32_t> qlev((size_t)n);
      for (int32_t k = 0; k < nlevL; ++k)
        for (int64_t q = lvr[size_t(k)]; q < lvr[size_t(k) + 1]; ++q) qlev[size_t(q)] = k;
      row_groups(n, [&](int64_t q) { return qlev[size_t(q)]; }, [&](int64_t q) { return blk[size_t(q)]; }, gs, lgrp_lev, lgrp_blk);
      sell_layout(llen, gs, lgrp_lev, nlevL, loff, lstart, lvsL, lgrp_s0);
    }
    nslL = int64_t(lstart.size()) - 1;
    padL = loff.back();
    // backward levels in solver order (real U dependencies, block-restricted): a row reads only
    // later rows of its own block, so the blocks are levelled on the host threads, each from its
    // last solver row backwards
    std::vector<int32_t> levU((size_t)n, 0);
    nlevU = 1;
    {
      std::vector<int32_t> byblk((size_t)n);
      std::iota(byblk.begin(), byblk.end(), 0);
      counting_sort_by(byblk, nblk, [&](int32_t a) { return blk[size_t(a)]; });
      std::vector<int64_t> bruns(1, 0);
      for (int64_t t = 1; t < n; ++t)
        if (blk[size_t(byblk[size_t(t)])] != blk[size_t(byblk[size_t(t) - 1])]) bruns.push_back(t);
      bruns.push_back(n);
      std::mutex mu;
      host_parallel_runs(bruns, [&](int64_t r0, int64_t r1) {
        int32_t nl = 1;
        for (int64_t r = r0; r < r1; ++r)
          for (int64_t t = bruns[size_t(r) + 1] - 1; t >= bruns[size_t(r)]; --t) {
            const int32_t i = byblk[size_t(t)];
            int32_t m = -1;
            for (int64_t k = pdiag[size_t(i)] + 1; k < prp[size_t(i) + 1]; ++k) {
              const int32_t j = pci[size_t(k)];
              if (blk[size_t(j)] == blk[size_t(i)]) m = std::max(m, levU[size_t(j)]);
            }
            levU[size_t(i)] = m + 1;
            nl = std::max(nl, m + 2);
          }
        std::lock_guard<std::mutex> lk(mu);
        nlevU = std::max(nlevU, nl);
      });
    }
    // backward-sweep slots: by backward level, then block, then solver row (two stable counting passes)
    urow.resize((size_t)n);
    std::iota(urow.begin(), urow.end(), 0);
    counting_sort_by(urow, nblk, [&](int32_t a) { return blk[size_t(a)]; });
    counting_sort_by(urow, int64_t(nlevU), [&](int32_t a) { return levU[size_t(a)]; });
    std::vector<int64_t> ulen_t((size_t)n);
    dpos.resize((size_t)n);
    for (int64_t t = 0; t < n; ++t) { ulen_t[size_t(t)] = ulen[size_t(urow[size_t(t)])]; dpos[size_t(urow[size_t(t)])] = t; }
    {
      std::vector<int64_t> gs;
      row_groups(n, [&](int64_t t) { return levU[size_t(urow[size_t(t)])]; }, [&](int64_t t) { return blk[size_t(urow[size_t(t)])]; },
                 gs, ugrp_lev, ugrp_blk);
      sell_layout(ulen_t, gs, ugrp_lev, nlevU, uoff, ustart, lvsU, ugrp_s0);
    }
    nslU = int64_t(ustart.size()) - 1;
    padU = uoff.back();
    fmap.assign((size_t)fnnz, -1);
    lcol.assign((size_t)padL, PAD);
    ucol.assign((size_t)padU, PAD);
    nnzL = std::accumulate(llen.begin(), llen.end(), int64_t(0));
    nnzU = std::accumulate(ulen.begin(), ulen.end(), int64_t(0));
    // every slice writes its own slots, and every row's entries of fmap belong to one slice
    host_parallel(nslL, int64_t(1) << 12, [&](int64_t j0, int64_t j1) {
      for (int64_t j = j0; j < j1; ++j)
        for (int64_t i = lstart[size_t(j)]; i < lstart[size_t(j) + 1]; ++i) {
          const int lane = int(i - lstart[size_t(j)]);
          int64_t kk = 0;
          for (int64_t k = prp[size_t(i)]; k < pdiag[size_t(i)]; ++k) {
            if (blk[size_t(pci[size_t(k)])] != blk[size_t(i)]) continue;
            const int64_t slot = loff[size_t(j)] + 32 * kk + lane;
            lcol[size_t(slot)] = pci[size_t(k)];
            fmap[size_t(k)] = slot;
            ++kk;
          }
        }
    });
    host_parallel(nslU, int64_t(1) << 12, [&](int64_t j0, int64_t j1) {
      for (int64_t j = j0; j < j1; ++j)
        for (int64_t t = ustart[size_t(j)]; t < ustart[size_t(j) + 1]; ++t) {
          const int lane = int(t - ustart[size_t(j)]);
          const int32_t i = urow[size_t(t)];
          int64_t kk = 0;
          for (int64_t k = pdiag[size_t(i)] + 1; k < prp[size_t(i) + 1]; ++k) {
            if (blk[size_t(pci[size_t(k)])] != blk[size_t(i)]) continue;
            const int64_t slot = uoff[size_t(j)] + 32 * kk + lane;
            ucol[size_t(slot)] = pci[size_t(k)];
            fmap[size_t(k)] = -(slot + 2);
            ++kk;
          }
        }
    });
  } else {
    nlevU = 1;
  }

  return VSHE_OK;
}

int System::setup_pattern(Ctx &ctx, const double *host_val) {
  Layout Lt;
  std::string err;
  int rc = Lt.build(n, nnz, rp, ci, opts, host_val, err);
  if (rc) return ctx.fail(rc, err);
  return setup_from_layout(ctx, Lt);
}

// The host copies of a layout's schedules and sizes (no device work).
void System::adopt_layout(const Layout &Lt) {
  has_pc = opts.precond != VSHE_PRECOND_NONE;
  mixed = opts.precision == VSHE_PRECISION_MIXED;
  perm = Lt.perm; blk = Lt.blk; lvr = Lt.lvr; lvsL = Lt.lvsL; lvsU = Lt.lvsU;
  lgrp_s0 = Lt.lgrp_s0; lgrp_lev = Lt.lgrp_lev; lgrp_blk = Lt.lgrp_blk;
  ugrp_s0 = Lt.ugrp_s0; ugrp_lev = Lt.ugrp_lev; ugrp_blk = Lt.ugrp_blk;
  loff_h = Lt.loff; uoff_h = Lt.uoff;
  lrow0_h.assign(Lt.lstart.begin(), Lt.lstart.end()); uslot0_h.assign(Lt.ustart.begin(), Lt.ustart.end());
  nlevL = Lt.nlevL; nlevU = Lt.nlevU; nslA = Lt.nslA; nslL = Lt.nslL; nslU = Lt.nslU;
  padA = Lt.padA; padL = Lt.padL; padU = Lt.padU; nnzL = Lt.nnzL; nnzU = Lt.nnzU; nnzF = Lt.nnzF;
}

int System::setup_from_layout(Ctx &ctx, const Layout &Lt) {
  adopt_layout(Lt);
  cudaError_t e;
  const auto &prp = Lt.prp; const auto &pci = Lt.pci; const auto &pdiag = Lt.pdiag; const auto &amap = Lt.amap;
  const auto &aoff = Lt.aoff; const auto &amapS = Lt.amapS; const auto &acol = Lt.acol;
  const auto &fmap = Lt.fmap; const auto &dpos = Lt.dpos; const auto &loff = Lt.loff; const auto &uoff = Lt.uoff;
  const auto &lstart = Lt.lstart; const auto &ustart = Lt.ustart; const auto &lcol = Lt.lcol; const auto &ucol = Lt.ucol;
  const auto &urow = Lt.urow;
  // ---- device buffers ----
  const size_t tsz = mixed ? sizeof(float) : sizeof(double);
#define ALLOC(ptr, type, count)                                              \
  ptr = (type *)arena.alloc(sizeof(type) * size_t(count), e);               \
  if (!ptr) return ctx.cuda_fail(e, "cudaMalloc " #ptr);
#define ALLOCT(ptr, count)                                                   \
  ptr = arena.alloc(tsz * size_t(count), e);                                 \
  if (!ptr) return ctx.cuda_fail(e, "cudaMalloc " #ptr);
  // Krylov vectors x r rh p v s t ph sh (FP64, solver order) with the zero entry n
  for (int k = 0; k < 9; ++k) { ALLOC(kv[k], double, n + kVecPad); }
  ALLOC(d_x64, double, n);
  ALLOC(d_bp, double, n + 1);
  ALLOC(d_perm, int32_t, n);
  ALLOC(d_aoff, int64_t, nslA + 1);
  ALLOC(d_amapS, int64_t, padA);
  ALLOC(d_acol, int32_t, padA);
  ALLOC(d_aval, double, padA);
  if (has_pc) {
    ALLOC(d_blk, int32_t, n);
    ALLOC(d_prp, int64_t, n + 1);
    ALLOC(d_pci, int32_t, nnzF);
    ALLOC(d_pdiag, int64_t, n);
    ALLOC(d_amap, int64_t, nnzF);
    ALLOC(d_fmap, int64_t, nnzF);
    ALLOC(d_dpos, int64_t, n);
    ALLOC(d_lvr, int64_t, nlevL + 1);
    ALLOC(d_lu64, double, nnzF);
    ALLOC(d_lrow0, int32_t, nslL + 1);
    ALLOC(d_loff, int64_t, nslL + 1);
    ALLOC(d_uslot0, int32_t, nslU + 1);
    ALLOC(d_uoff, int64_t, nslU + 1);
    ALLOC(d_urow, int32_t, n + kVecPad);
    ALLOC(d_lvsL, int64_t, lvsL.size());
    ALLOC(d_lvsU, int64_t, lvsU.size());
    ALLOC(d_lcol, int32_t, std::max<int64_t>(padL, 1));
    ALLOC(d_ucol, int32_t, std::max<int64_t>(padU, 1));
    ALLOCT(d_lval, std::max<int64_t>(padL, 1));
    ALLOCT(d_uval, std::max<int64_t>(padU, 1));
    ALLOCT(d_udinv, n + kVecPad);
    ALLOC(d_ytmp, double, n + 1);
  }
#undef ALLOC
#undef ALLOCT
  cudaStream_t s = ctx.stream;
  // every vector starts at 0 (entry n is the SELL padding target and is never written)
  for (int k = 0; k < 9; ++k)
    if ((e = cudaMemsetAsync(kv[k], 0, sizeof(double) * size_t(n + kVecPad), s)) != cudaSuccess) return ctx.cuda_fail(e, "memset");
  if ((e = cudaMemsetAsync(d_bp, 0, sizeof(double) * size_t(n + 1), s)) != cudaSuccess) return ctx.cuda_fail(e, "memset");
  if ((e = cudaMemsetAsync(d_x64, 0, sizeof(double) * size_t(n), s)) != cudaSuccess) return ctx.cuda_fail(e, "memset");
#define H2D(dst, vec)                                                                                        \
  if (!vec.empty() && (e = cudaMemcpyAsync(dst, vec.data(), sizeof(vec[0]) * vec.size(), cudaMemcpyHostToDevice, s)) != cudaSuccess) \
    return ctx.cuda_fail(e, "upload " #dst);
  H2D(d_perm, perm);
  H2D(d_aoff, aoff);
  H2D(d_amapS, amapS);
  H2D(d_acol, acol);
  if (has_pc) {
    std::vector<int32_t> lrow0(lstart.begin(), lstart.end()), uslot0(ustart.begin(), ustart.end());
    H2D(d_blk, blk);
    H2D(d_prp, prp);
    H2D(d_pci, pci);
    H2D(d_pdiag, pdiag);
    H2D(d_amap, amap);
    H2D(d_fmap, fmap);
    H2D(d_dpos, dpos);
    H2D(d_lvr, lvr);
    H2D(d_lrow0, lrow0);
    H2D(d_loff, loff);
    H2D(d_uslot0, uslot0);
    H2D(d_uoff, uoff);
    H2D(d_urow, urow);
    H2D(d_lvsL, lvsL);
    H2D(d_lvsU, lvsU);
    H2D(d_lcol, lcol);
    H2D(d_ucol, ucol);
    if ((e = cudaMemsetAsync(d_lval, 0, tsz * size_t(std::max<int64_t>(padL, 1)), s)) != cudaSuccess) return ctx.cuda_fail(e, "memset");
    if ((e = cudaMemsetAsync(d_uval, 0, tsz * size_t(std::max<int64_t>(padU, 1)), s)) != cudaSuccess) return ctx.cuda_fail(e, "memset");
    if ((e = cudaMemsetAsync(d_ytmp, 0, sizeof(double) * size_t(n + 1), s)) != cudaSuccess) return ctx.cuda_fail(e, "memset");
    if ((e = cudaMemsetAsync(d_urow + n, 0, sizeof(int32_t) * size_t(kVecPad), s)) != cudaSuccess) return ctx.cuda_fail(e, "memset");
    if ((e = cudaMemsetAsync((char *)d_udinv + tsz * size_t(n), 0, tsz * size_t(kVecPad), s)) != cudaSuccess) return ctx.cuda_fail(e, "memset");
  }
#undef H2D
  if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return ctx.cuda_fail(e, "upload pattern");
  return VSHE_OK;
}

void System::fill_sysdev(void *out) const {
  // SysDev<P> has the same layout for both factor types (pointers only); fill through the
  // float view, whose factor pointers the FP64 solver reads as double
  SysDev<float> d;
  std::memset(&d, 0, sizeof(d));
  d.n = n;
  d.aoff = d_aoff; d.acol = d_acol; d.aval = d_aval; d.b = d_bp;
  d.lrow0 = d_lrow0; d.loff = d_loff; d.lcol = d_lcol; d.lval = (const float *)d_lval;
  d.uslot0 = d_uslot0; d.uoff = d_uoff; d.ucol = d_ucol; d.uval = (const float *)d_uval; d.udinv = (const float *)d_udinv;
  d.urow = d_urow;
  d.ytmp = d_ytmp;
  d.lvsL = d_lvsL; d.lvsU = d_lvsU; d.nlevL = nlevL; d.nlevU = nlevU;
  d.x = (double *)kv[0]; d.r = (double *)kv[1]; d.rh = (double *)kv[2]; d.p = (double *)kv[3];
  d.v = (double *)kv[4]; d.s = (double *)kv[5]; d.t = (double *)kv[6]; d.ph = (double *)kv[7]; d.sh = (double *)kv[8];
  std::memcpy(out, &d, sizeof(d));
}

// ------------------------------------------------------------------ Batch
// Writes the context's poll limit into the batch's barrier words (bar[2..3]) when it changed;
// every bounded device-side wait of the batch's kernels reads it there (outside any capture).
int Batch::sync_spin_limit(Ctx &ctx) {
  if (bar_limit == ctx.spin_limit) return VSHE_OK;
  const unsigned long long v = ctx.spin_limit;
  cudaError_t e = cudaMemcpyAsync(d_bar + 2, &v, sizeof(v), cudaMemcpyHostToDevice, ctx.stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx.stream);
  if (e != cudaSuccess) return ctx.cuda_fail(e, "spin limit");
  bar_limit = v;
  return VSHE_OK;
}

// Sweep plan of a batch (host only): which members sweep as tasks (k_trsv_task, k_trsv_cluster)
// and which in the grid-wide schedule, the tasks, the chunks of their levels with the chunks'
// slice descriptors, and the level slice ranges of the cluster sweeps.
//
// Triangular sweeps.  A member sweeps either as tasks, one CTA each walking its levels with
// a CTA barrier per level (k_trsv_task), or in the merged level schedule of the grid-wide sweep
// (k_trsv_persistent).  Tasks are whole systems for members with many short levels (fewer than
// kCtaRowsPerLevel rows per forward level on average and more than kCtaMinLevels levels: 1D
// devices) whose apply one SM finishes sooner than the grid-wide sweep, and preconditioner
// blocks for block-ILU members with at least two blocks of at most kTaskMaxRows rows (energy
// slabs: the factor has no entry between blocks, so they sweep independently).
// VSHE_TRSV_PER_SYSTEM / VSHE_TRSV_PER_BLOCK force the former / latter for every member; the
// grid-wide modes force the merged schedule.  The time estimates use rates measured on the 2D
// bar: one CTA streams a task's factor and vectors at about kTaskBytesPerUs, and a level of the
// grid-wide sweep costs about kGridLevelUs (its grid barrier and the latency of the level's
// rows) on top of the apply's bytes at kGridBytesPerUs.
void plan_sweep_tasks(const std::vector<System *> &sys, bool mixed, bool has_pc, int64_t num_sms_hint, SweepPlan &P) {
  constexpr int64_t kCtaRowsPerLevel = 4096;
  constexpr int32_t kCtaMinLevels = 32;
  constexpr int64_t kTaskMaxRows = int64_t(1) << 18;
  constexpr double kTaskBytesPerUs = 3.0e4, kGridBytesPerUs = 3.0e6, kGridLevelUs = 4.0;
  const int nsys = int(sys.size());
  std::vector<char> &on_task = P.on_task;  // 0 grid, 1 whole system, 2 per block
  on_task.assign((size_t)nsys, 0);
  if (has_pc) {
    for (int k = 0; k < nsys; ++k) {
      const System *S = sys[size_t(k)];
      const int mode = S->opts.trsv_mode;
      int32_t nb = 0;
      for (int32_t b : S->blk) nb = std::max(nb, b + 1);
      std::vector<int64_t> bsz((size_t)nb, 0);
      for (int32_t b : S->blk) bsz[size_t(b)]++;
      const int64_t bmax = nb ? *std::max_element(bsz.begin(), bsz.end()) : 0;
      const double apply_bytes = double(4 + (mixed ? 4 : 8)) * double(S->padL + S->padU) + 40.0 * double(S->n);
      const bool one_sm_sooner = apply_bytes / kTaskBytesPerUs < kGridLevelUs * double(S->nlevL + S->nlevU) + apply_bytes / kGridBytesPerUs;
      const bool per_sys = S->nlevL > kCtaMinLevels && S->n / std::max(S->nlevL, 1) < kCtaRowsPerLevel && one_sm_sooner;
      const bool per_blk = (S->opts.precond == VSHE_PRECOND_BLOCK_ILU0 || S->opts.precond == VSHE_PRECOND_ILUT) && nb >= 2 &&
                           bmax <= kTaskMaxRows;
      if (mode == VSHE_TRSV_PER_SYSTEM) on_task[size_t(k)] = 1;
      else if (mode == VSHE_TRSV_PER_BLOCK) on_task[size_t(k)] = 2;
      else if (mode == VSHE_TRSV_AUTO) on_task[size_t(k)] = per_blk ? 2 : per_sys ? 1 : 0;
    }
  }
  std::vector<TaskDev> &tasks = P.tasks;
  std::vector<ChunkDev> &chunks = P.chunks;
  std::vector<SliceDesc> &sdesc = P.sdesc;
  std::vector<ClusterTask> &ctasks = P.ctasks;
  std::vector<int64_t> &clv = P.clv;
  {
    const int vbytes = mixed ? int(sizeof(float)) : int(sizeof(double));
    // chunks of the slices [a, b) of one level of one system's L (lower) or U sweep: runs of
    // whole slices whose descriptors, factor slots and row operands fit one stage, with their
    // slice descriptors; a slice too wide for a stage is its own chunk, read from global memory
    auto add_level = [&](const System *S, bool lower, int64_t a, int64_t b) {
      if (a >= b) return;
      const std::vector<int64_t> &off = lower ? S->loff_h : S->uoff_h;
      const std::vector<int64_t> &rs = lower ? S->lrow0_h : S->uslot0_h;
      auto bytes = [&](int64_t j0, int64_t e) {
        return task_chunk_bytes(e - j0, off[size_t(e)] - off[size_t(j0)], rs[size_t(j0)] & ~int64_t(3),
                                (rs[size_t(e)] + 3) & ~int64_t(3), lower, vbytes);
      };
      for (int64_t j = a; j < b;) {
        ChunkDev c{};
        c.s0 = int32_t(j);
        c.o0 = off[size_t(j)];
        c.d0 = int64_t(sdesc.size());
        c.rot = int32_t((j - a) % kTaskConsumers);
        if (bytes(j, j + 1) > kTaskStageBytes) {
          c.s1 = int32_t(j + 1);
          c.flags = kChunkDirect;
          chunks.push_back(c);
          ++j;
          continue;
        }
        int64_t e = j + 1;
        while (e < b && bytes(j, e + 1) <= kTaskStageBytes) ++e;
        c.s1 = int32_t(e);
        c.nslot = int32_t(off[size_t(e)] - off[size_t(j)]);
        c.r0 = int32_t(rs[size_t(j)] & ~int64_t(3));
        c.r1 = int32_t((rs[size_t(e)] + 3) & ~int64_t(3));
        for (int64_t i = j; i < e; ++i)
          sdesc.push_back({int32_t(off[size_t(i)] - off[size_t(j)]), int32_t((off[size_t(i) + 1] - off[size_t(i)]) >> 5),
                           int32_t(rs[size_t(i)]), int32_t(rs[size_t(i) + 1] - rs[size_t(i)])});
        chunks.push_back(c);
        j = e;
      }
      chunks.back().flags |= kChunkLevelEnd;
    };
    std::vector<std::pair<int64_t, TaskDev>> tw;  // (work in slots, task)
    std::vector<std::vector<int64_t>> twl, twu;    // per task: level slice ranges (pairs) of L and U
    for (int k = 0; k < nsys; ++k) {
      if (!on_task[size_t(k)]) continue;
      const System *S = sys[size_t(k)];
      auto make = [&](const std::vector<std::pair<int64_t, int64_t>> &lv_l, const std::vector<std::pair<int64_t, int64_t>> &lv_u) {
        TaskDev t{k, int32_t(chunks.size()), 0, 0, 0, 0};
        int64_t work = 0;
        for (auto &r : lv_l) {
          add_level(S, true, r.first, r.second);
          work += S->loff_h[size_t(r.second)] - S->loff_h[size_t(r.first)] + 32 * (r.second - r.first);
        }
        t.cL1 = int32_t(chunks.size());
        t.cU0 = int32_t(chunks.size());
        for (auto &r : lv_u) {
          add_level(S, false, r.first, r.second);
          work += S->uoff_h[size_t(r.second)] - S->uoff_h[size_t(r.first)] + 32 * (r.second - r.first);
        }
        t.cU1 = int32_t(chunks.size());
        if (t.cL1 > t.cL0 || t.cU1 > t.cU0) {
          t.pad = int32_t(tw.size());  // index into twl / twu until the tasks are sorted
          tw.push_back({work, t});
          twl.emplace_back();
          twu.emplace_back();
          for (auto &r : lv_l) { twl.back().push_back(r.first); twl.back().push_back(r.second); }
          for (auto &r : lv_u) { twu.back().push_back(r.first); twu.back().push_back(r.second); }
        }
      };
      if (on_task[size_t(k)] == 1) {
        std::vector<std::pair<int64_t, int64_t>> l, u;
        for (int32_t v = 0; v < S->nlevL; ++v) l.push_back({S->lvsL[size_t(v)], S->lvsL[size_t(v) + 1]});
        for (int32_t v = 0; v < S->nlevU; ++v) u.push_back({S->lvsU[size_t(v)], S->lvsU[size_t(v) + 1]});
        make(l, u);
      } else {
        // runs of consecutive blocks: a block of more than the target work is a task of its own,
        // smaller neighbours share one (the level slices of consecutive blocks are contiguous,
        // blocks being ordered inside every level), so that the tasks of the batch fit one wave
        // of one CTA per SM
        int32_t nb = 0;
        for (int32_t b : S->blk) nb = std::max(nb, b + 1);
        std::vector<int64_t> wb((size_t)nb, 0);
        for (size_t g = 0; g + 1 < S->lgrp_s0.size(); ++g)
          wb[size_t(S->lgrp_blk[g])] += S->loff_h[size_t(S->lgrp_s0[g + 1])] - S->loff_h[size_t(S->lgrp_s0[g])];
        for (size_t g = 0; g + 1 < S->ugrp_s0.size(); ++g)
          wb[size_t(S->ugrp_blk[g])] += S->uoff_h[size_t(S->ugrp_s0[g + 1])] - S->uoff_h[size_t(S->ugrp_s0[g])];
        int64_t total = 0, wmax = 0;
        for (int64_t w : wb) { total += w; wmax = std::max(wmax, w); }
        const int64_t slots = std::max<int64_t>(1, num_sms_hint - int64_t(nsys) + 1);
        std::vector<int32_t> gstart;  // first block of each task
        for (int64_t target = std::max<int64_t>(wmax, (total + slots - 1) / slots);; target += std::max<int64_t>(1, target / 20)) {
          gstart.clear();
          int64_t acc = 0;
          for (int32_t b = 0; b < nb; ++b) {
            if (wb[size_t(b)] == 0) continue;
            if (gstart.empty() || acc + wb[size_t(b)] > target) { gstart.push_back(b); acc = 0; }
            acc += wb[size_t(b)];
          }
          if (int64_t(gstart.size()) <= slots) break;
        }
        std::vector<int32_t> task_of((size_t)nb, -1);
        for (size_t t = 0; t < gstart.size(); ++t) {
          const int32_t e = t + 1 < gstart.size() ? gstart[t + 1] : nb;
          for (int32_t b = gstart[t]; b < e; ++b) task_of[size_t(b)] = int32_t(t);
        }
        // merged level ranges of each task: the task's groups of one level are adjacent slices
        std::vector<std::vector<std::pair<int64_t, int64_t>>> l(gstart.size()), u(gstart.size());
        auto add = [&](std::vector<std::pair<int64_t, int64_t>> &v, int32_t lev, std::vector<int32_t> &lastlev, size_t t, int64_t a, int64_t b) {
          if (!v.empty() && lastlev[t] == lev && v.back().second == a) v.back().second = b;
          else v.push_back({a, b});
          lastlev[t] = lev;
        };
        std::vector<int32_t> lastL(gstart.size(), -1), lastU(gstart.size(), -1);
        for (size_t g = 0; g + 1 < S->lgrp_s0.size(); ++g) {
          const int32_t t = task_of[size_t(S->lgrp_blk[g])];
          if (t >= 0) add(l[size_t(t)], S->lgrp_lev[g], lastL, size_t(t), S->lgrp_s0[g], S->lgrp_s0[g + 1]);
        }
        for (size_t g = 0; g + 1 < S->ugrp_s0.size(); ++g) {
          const int32_t t = task_of[size_t(S->ugrp_blk[g])];
          if (t >= 0) add(u[size_t(t)], S->ugrp_lev[g], lastU, size_t(t), S->ugrp_s0[g], S->ugrp_s0[g + 1]);
        }
        for (size_t t = 0; t < gstart.size(); ++t) make(l[t], u[t]);
      }
    }
    std::stable_sort(tw.begin(), tw.end(), [](const std::pair<int64_t, TaskDev> &a, const std::pair<int64_t, TaskDev> &b) { return a.first > b.first; });
    for (auto &t : tw) {
      const std::vector<int64_t> &l = twl[size_t(t.second.pad)], &u = twu[size_t(t.second.pad)];
      ClusterTask c{t.second.sys, int32_t(l.size() / 2), int32_t(u.size() / 2), 0, int64_t(clv.size()), 0};
      clv.insert(clv.end(), l.begin(), l.end());
      c.offU = int64_t(clv.size());
      clv.insert(clv.end(), u.begin(), u.end());
      ctasks.push_back(c);
      t.second.pad = 0;
      tasks.push_back(t.second);
    }
    const int ntasks = int(tasks.size());
    // shape class of the task sweep: precision, the largest task's work and the task count (the
    // apply's time is the largest task's walk, in waves of one CTA per SM)
    auto log2c = [](int64_t v) { int c = 0; while (v > 1) { v >>= 1; ++c; } return c; };
    if (!tw.empty()) {
      P.tune_key_tasks = (int64_t(mixed ? 1 : 0) << 40) | (int64_t(log2c(tw.front().first)) << 20) | int64_t(log2c(ntasks));
      P.has_tune_key = true;
    }
  }
}

int Batch::build(Ctx &ctx, const std::vector<System *> &members) {
  int rc0 = 0;
  sys = members;
  nsys = int(sys.size());
  mixed = sys[0]->mixed;
  has_pc = sys[0]->has_pc;
  for (System *S : sys)
    if (S->mixed != mixed || S->has_pc != has_pc)
      return ctx.fail(VSHE_E_INVALID_ARGUMENT, "systems in one batch need the same precision and preconditioner kind");
  // triangular sweeps: tasks or the grid-wide schedule per member (plan_sweep_tasks)
  SweepPlan plan;
  {
    int64_t num_sms = 148;
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) == cudaSuccess && cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) == cudaSuccess && sms > 0)
      num_sms = sms;
    plan_sweep_tasks(sys, mixed, has_pc, num_sms, plan);
  }
  const std::vector<char> &on_task = plan.on_task;
  const std::vector<TaskDev> &tasks = plan.tasks;
  const std::vector<ChunkDev> &chunks = plan.chunks;
  const std::vector<SliceDesc> &sdesc = plan.sdesc;
  const std::vector<ClusterTask> &ctasks = plan.ctasks;
  const std::vector<int64_t> &clv = plan.clv;
  ntasks = int(tasks.size());
  if (plan.has_tune_key) tune_key_tasks = plan.tune_key_tasks;
  grid_group = false;
  {
    int64_t grid_rows = 0;
    for (int k = 0; k < nsys; ++k)
      if (!on_task[size_t(k)]) { grid_group = true; grid_rows += sys[size_t(k)]->n; }
    int c = 0;
    for (int64_t v = grid_rows; v > 1; v >>= 1) ++c;
    tune_key_grid = (int64_t(mixed ? 1 : 0) << 40) | (int64_t(sys[0]->opts.trsv_mode) << 32) | int64_t(c);
  }
  task_kind.assign(on_task.begin(), on_task.end());
  std::vector<int64_t> cptrL, cptrU, fptr;
  std::vector<int32_t> csL, cqL, csU, cqU, fsys, frow;
  auto slices = [&](bool lower, std::vector<int64_t> &cptr, std::vector<int32_t> &cs, std::vector<int32_t> &cq, int32_t &nl) {
    nl = 0;
    for (int k = 0; k < nsys; ++k)
      if (!on_task[size_t(k)]) nl = std::max(nl, lower ? sys[size_t(k)]->nlevL : sys[size_t(k)]->nlevU);
    cptr.assign(1, 0);
    for (int32_t l = 0; l < nl; ++l) {
      for (int k = 0; k < nsys; ++k) {
        if (on_task[size_t(k)]) continue;
        const auto &vp = lower ? sys[size_t(k)]->lvsL : sys[size_t(k)]->lvsU;
        if (l + 1 >= int32_t(vp.size())) continue;
        for (int64_t j = vp[size_t(l)]; j < vp[size_t(l) + 1]; ++j) {
          cs.push_back(k);
          cq.push_back(int32_t(j));
        }
      }
      cptr.push_back(int64_t(cs.size()));
    }
  };
  if (has_pc) {
    slices(true, cptrL, csL, cqL, nlevL);
    slices(false, cptrU, csU, cqU, nlevU);
    // factorisation: merged level l = the forward-level-l rows of every member (all members,
    // whichever sweep they use)
    nlevF = 0;
    for (System *S : sys) nlevF = std::max(nlevF, S->nlevL);
    if (nsys > 1) {
      fptr.assign(1, 0);
      for (int32_t l = 0; l < nlevF; ++l) {
        for (int k = 0; k < nsys; ++k) {
          const System *S = sys[size_t(k)];
          if (l + 1 >= int32_t(S->lvr.size())) continue;
          for (int64_t q = S->lvr[size_t(l)]; q < S->lvr[size_t(l) + 1]; ++q) {
            fsys.push_back(k);
            frow.push_back(int32_t(q));
          }
        }
        fptr.push_back(int64_t(fsys.size()));
      }
    }
  }
  cudaError_t e;
#define ALLOC(ptr, type, count)                                              \
  ptr = (type *)arena.alloc(sizeof(type) * size_t(count), e);               \
  if (!ptr) return ctx.cuda_fail(e, "cudaMalloc batch " #ptr);
  ALLOC(d_active, int32_t, nsys);
  ALLOC(d_counters, int32_t, nsys);
  ALLOC(d_bar, unsigned, 4);
  ALLOC(d_err, int32_t, 1);
  ALLOC(d_rnorm2, double, nsys);
  ALLOC(d_bnorm2, double, nsys);
  d_tasks = arena.alloc(sizeof(TaskDev) * std::max<size_t>(tasks.size(), 1), e);
  if (!d_tasks) return ctx.cuda_fail(e, "cudaMalloc tasks");
  d_chunks = arena.alloc(sizeof(ChunkDev) * std::max<size_t>(chunks.size(), 1), e);
  if (!d_chunks) return ctx.cuda_fail(e, "cudaMalloc chunks");
  d_sdesc = arena.alloc(sizeof(SliceDesc) * std::max<size_t>(sdesc.size(), 1), e);
  if (!d_sdesc) return ctx.cuda_fail(e, "cudaMalloc slice descriptors");
  d_ctasks = arena.alloc(sizeof(ClusterTask) * std::max<size_t>(ctasks.size(), 1), e);
  if (!d_ctasks) return ctx.cuda_fail(e, "cudaMalloc cluster tasks");
  ALLOC(d_clv, int64_t, std::max<size_t>(clv.size(), 1));
  d_sysdev = arena.alloc(vk_sysdev_size() * size_t(nsys), e);
  if (!d_sysdev) return ctx.cuda_fail(e, "cudaMalloc sysdev");
  d_state = arena.alloc(vk_bistate_size() * size_t(nsys), e);
  if (!d_state) return ctx.cuda_fail(e, "cudaMalloc state");
  d_refdev = arena.alloc(vk_refdev_size() * size_t(nsys), e);
  if (!d_refdev) return ctx.cuda_fail(e, "cudaMalloc refdev");
  d_factdev = arena.alloc(vk_factdev_size() * size_t(nsys), e);
  if (!d_factdev) return ctx.cuda_fail(e, "cudaMalloc factdev");
  if (has_pc) {
    ALLOC(d_cptrL, int64_t, cptrL.size());
    ALLOC(d_cptrU, int64_t, cptrU.size());
    ALLOC(d_csL, int32_t, std::max<size_t>(csL.size(), 1));
    ALLOC(d_cqL, int32_t, std::max<size_t>(cqL.size(), 1));
    ALLOC(d_csU, int32_t, std::max<size_t>(csU.size(), 1));
    ALLOC(d_cqU, int32_t, std::max<size_t>(cqU.size(), 1));
    if (nsys > 1) {
      ALLOC(d_fptr, int64_t, fptr.size());
      ALLOC(d_fsys, int32_t, std::max<size_t>(fsys.size(), 1));
      ALLOC(d_frow, int32_t, std::max<size_t>(frow.size(), 1));
    }
  }
#undef ALLOC
  cudaStream_t s = ctx.stream;
  std::vector<char> sd(vk_sysdev_size() * size_t(nsys));
  std::vector<char> rd(vk_refdev_size() * size_t(nsys));
  std::vector<char> fd(vk_factdev_size() * size_t(nsys));
  for (int k = 0; k < nsys; ++k) {
    System *S = sys[size_t(k)];
    S->fill_sysdev(sd.data() + vk_sysdev_size() * size_t(k));
    // the final / replacement residual is written into the Krylov r
    RefDev r{S->n, S->d_aoff, S->d_acol, S->d_aval, S->d_bp, (const double *)S->kv[0], (double *)S->kv[1]};
    std::memcpy(rd.data() + vk_refdev_size() * size_t(k), &r, sizeof(r));
    FactDev f{S->n, S->d_prp, S->d_pci, S->d_lu64, S->d_pdiag, S->d_blk, 0, 0, 0.0};
    if (S->opts.precond == VSHE_PRECOND_ILUT) {
      f.ilut = 1;
      f.pkeep = S->opts.ilut_entries > 0 ? S->opts.ilut_entries : 60;
      f.tau = S->opts.ilut_drop > 0 ? S->opts.ilut_drop : 1e-4;
    }
    std::memcpy(fd.data() + vk_factdev_size() * size_t(k), &f, sizeof(f));
  }
  std::vector<int32_t> ones((size_t)(nsys), 1), zeros(size_t(nsys), 0);
#define H2D(dst, src, bytes)                                                             \
  if ((e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s)) != cudaSuccess) \
    return ctx.cuda_fail(e, "upload batch " #dst);
  H2D(d_active, ones.data(), sizeof(int32_t) * size_t(nsys));
  H2D(d_counters, zeros.data(), sizeof(int32_t) * size_t(nsys));
  H2D(d_sysdev, sd.data(), sd.size());
  H2D(d_refdev, rd.data(), rd.size());
  H2D(d_factdev, fd.data(), fd.size());
  if (!tasks.empty()) { H2D(d_tasks, tasks.data(), sizeof(TaskDev) * tasks.size()); }
  if (!chunks.empty()) { H2D(d_chunks, chunks.data(), sizeof(ChunkDev) * chunks.size()); }
  if (!sdesc.empty()) { H2D(d_sdesc, sdesc.data(), sizeof(SliceDesc) * sdesc.size()); }
  if (!ctasks.empty()) { H2D(d_ctasks, ctasks.data(), sizeof(ClusterTask) * ctasks.size()); }
  if (!clv.empty()) { H2D(d_clv, clv.data(), sizeof(int64_t) * clv.size()); }
  if (has_pc) {
    H2D(d_cptrL, cptrL.data(), sizeof(int64_t) * cptrL.size());
    H2D(d_cptrU, cptrU.data(), sizeof(int64_t) * cptrU.size());
    if (!csL.empty()) {
      H2D(d_csL, csL.data(), sizeof(int32_t) * csL.size());
      H2D(d_cqL, cqL.data(), sizeof(int32_t) * cqL.size());
    }
    if (!csU.empty()) {
      H2D(d_csU, csU.data(), sizeof(int32_t) * csU.size());
      H2D(d_cqU, cqU.data(), sizeof(int32_t) * cqU.size());
    }
    if (nsys > 1) {
      H2D(d_fptr, fptr.data(), sizeof(int64_t) * fptr.size());
      if (!fsys.empty()) {
        H2D(d_fsys, fsys.data(), sizeof(int32_t) * fsys.size());
        H2D(d_frow, frow.data(), sizeof(int32_t) * frow.size());
      }
    }
  }
#undef H2D
  if ((e = cudaMemsetAsync(d_bar, 0, 2 * sizeof(unsigned), s)) != cudaSuccess) return ctx.cuda_fail(e, "memset");
  bar_limit = 0;
  if ((rc0 = sync_spin_limit(ctx))) return rc0;
  if ((e = cudaMemsetAsync(d_err, 0, sizeof(int32_t), s)) != cudaSuccess) return ctx.cuda_fail(e, "memset");
  if ((e = cudaMemsetAsync(d_state, 0, vk_bistate_size() * size_t(nsys), s)) != cudaSuccess) return ctx.cuda_fail(e, "memset");
  if (has_pc) {
    levL = VkLevels{nlevL, d_cptrL, d_csL, d_cqL, nullptr};
    levU = VkLevels{nlevU, d_cptrU, d_csU, d_cqU, nullptr};
    if (nsys > 1) levF = VkLevels{nlevF, d_fptr, d_fsys, d_frow, nullptr};
    else levF = VkLevels{nlevF, sys[0]->d_lvr, nullptr, nullptr, nullptr};
  }
  int dev = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&num_sms, cudaDevAttrMultiProcessorCount, dev);
  int bps = 0;
  if (mixed) vk_trsv_occupancy_f32(&bps); else vk_trsv_occupancy_f64(&bps);
  trsv_grid = std::max(1, std::min(bps, 4)) * num_sms;
  trsv_bps_max = std::max(1, std::min(bps, 8));
  int bpf = 0;
  vk_ilu0_occupancy(&bpf);
  ilu_grid = std::max(1, std::min(bpf, 4)) * num_sms;
  cudaError_t es = cudaStreamSynchronize(s);
  if (es != cudaSuccess) return ctx.cuda_fail(es, "batch upload");
  return set_tiles(ctx);
}

// Row tiles (whole SELL slices: multiples of 32 rows) that never straddle two systems; the tile
// kernels run one CTA per tile and reduce per tile.  Member k uses its own tile_rows (2048 until
// tuned); only_member >= 0 builds tiles of `rows` rows for that member alone (autotuner trials).
int Batch::set_tiles(Ctx &ctx, int only_member, int64_t rows) {
  std::vector<int32_t> tsys, st0;
  std::vector<int64_t> tr0, tr1;
  for (int k = 0; k < nsys; ++k) {
    st0.push_back(int32_t(tsys.size()));
    if (only_member >= 0 && k != only_member) continue;
    const int64_t tr = only_member >= 0 ? rows : (sys[size_t(k)]->tile_rows > 0 ? sys[size_t(k)]->tile_rows : 2048);
    for (int64_t a = 0; a < sys[size_t(k)]->n; a += tr) {
      tsys.push_back(k);
      tr0.push_back(a);
      tr1.push_back(std::min(a + tr, sys[size_t(k)]->n));
    }
  }
  st0.push_back(int32_t(tsys.size()));
  cudaError_t e;
  cudaStream_t s = ctx.stream;
  if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return ctx.cuda_fail(e, "tiles");  // old tiles no longer in use
  tile_arena.release();
  ntiles = int(tsys.size());
#define ALLOC(ptr, type, count)                                              \
  ptr = (type *)tile_arena.alloc(sizeof(type) * size_t(count), e);          \
  if (!ptr) return ctx.cuda_fail(e, "cudaMalloc tiles " #ptr);
  ALLOC(d_tile_sys, int32_t, ntiles);
  ALLOC(d_tile_r0, int64_t, ntiles);
  ALLOC(d_tile_r1, int64_t, ntiles);
  ALLOC(d_sys_tile0, int32_t, nsys + 1);
  ALLOC(d_partials, double, size_t(ntiles) * 3);
#undef ALLOC
#define H2D(dst, src, bytes)                                                             \
  if ((e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s)) != cudaSuccess) \
    return ctx.cuda_fail(e, "upload tiles " #dst);
  H2D(d_tile_sys, tsys.data(), sizeof(int32_t) * tsys.size());
  H2D(d_tile_r0, tr0.data(), sizeof(int64_t) * tr0.size());
  H2D(d_tile_r1, tr1.data(), sizeof(int64_t) * tr1.size());
  H2D(d_sys_tile0, st0.data(), sizeof(int32_t) * st0.size());
#undef H2D
  tiles = VkTiles{ntiles, d_tile_sys, d_tile_r0, d_tile_r1, d_sys_tile0};
  if (chunk_exec) { cudaGraphExecDestroy(chunk_exec); chunk_exec = nullptr; }  // the graph holds the old tiles
  if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return ctx.cuda_fail(e, "tiles");
  return VSHE_OK;
}

// Autotuner of the row-tile size.  For a member whose size class (floor(log2 n)) has no choice
// in the context yet, it times the FP64 SELL SpMV with its fused tile reduction (the residual
// kernel, the same structure as the SpMV of every BiCGStab step) on that member alone for each
// candidate, with CUDA events, and records the fastest for the class.  Runs before a solve (the
// residual it writes is overwritten by the solve).
int Batch::autotune_tiles(Ctx &ctx) {
  static const int64_t cand[] = {512, 1024, 2048, 4096};
  bool changed = false;
  for (int k = 0; k < nsys; ++k) {
    System *S = sys[size_t(k)];
    if (S->tile_rows > 0) continue;
    int cls = 0;
    while ((int64_t(1) << (cls + 1)) <= S->n) ++cls;
    auto it = ctx.tile_choice.find(cls);
    if (it == ctx.tile_choice.end()) {
      cudaStream_t s = ctx.stream;
      cudaEvent_t a, b;
      cudaEventCreate(&a); cudaEventCreate(&b);
      double best = 1e30;
      int64_t best_rows = 2048;
      std::vector<double> t;
      for (int64_t rows : cand) {
        int rc = set_tiles(ctx, k, rows);
        if (rc) { cudaEventDestroy(a); cudaEventDestroy(b); return rc; }
        vk_residual64(ntiles, d_refdev, &tiles, d_partials, d_counters, d_active, d_rnorm2, d_bnorm2, s);  // warm-up
        cudaEventRecord(a, s);
        for (int r = 0; r < 5; ++r) vk_residual64(ntiles, d_refdev, &tiles, d_partials, d_counters, d_active, d_rnorm2, d_bnorm2, s);
        cudaEventRecord(b, s);
        cudaError_t e = cudaEventSynchronize(b);
        float ms = 0;
        cudaEventElapsedTime(&ms, a, b);
        if (e != cudaSuccess) { cudaEventDestroy(a); cudaEventDestroy(b); return ctx.cuda_fail(e, "autotune"); }
        t.push_back(ms / 5.0);
        if (ms < best) { best = ms; best_rows = rows; }
      }
      cudaEventDestroy(a); cudaEventDestroy(b);
      it = ctx.tile_choice.emplace(cls, best_rows).first;
      ctx.tile_timings[cls] = t;
    }
    S->tile_rows = it->second;
    changed = true;
  }
  return changed ? set_tiles(ctx) : VSHE_OK;
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
  int rs = sync_spin_limit(ctx);
  if (rs) return rs;
  cudaStream_t s = ctx.stream;
  const int mode = (sys[0]->opts.trsv_mode == VSHE_TRSV_PER_LEVEL) ? 2 : 1;
  int rc = vk_ilu0(mode, mode == 1 ? ilu_grid : std::max(1, num_sms * 8), d_factdev, &levF, d_bar, d_err, s);
  if (rc) return ctx.cuda_fail(cudaError_t(rc), "ilu0 launch");
  for (System *S : sys) {
    if (mixed)
      vk_split_factor_f32(S->nnzF, S->n, S->d_lu64, S->d_fmap, S->d_pdiag, S->d_dpos, (float *)S->d_lval, (float *)S->d_uval, (float *)S->d_udinv, s);
    else
      vk_split_factor_f64(S->nnzF, S->n, S->d_lu64, S->d_fmap, S->d_pdiag, S->d_dpos, (double *)S->d_lval, (double *)S->d_uval, (double *)S->d_udinv, s);
  }
  return check_err(ctx, "ilu0 factorisation");
}

// Autotuner of the grid-wide sweep's CTA count (1 .. 6 CTAs per SM: fewer CTAs make each grid
// barrier cheaper, more put more slices in flight), for the sweep kind the options name (a grid
// barrier per level unless VSHE_TRSV_FLOW asks for the barrier-free sweep, which measured 2-3x
// slower on the 2D bar with 21 and with 779 levels, so AUTO does not try it).  Timed once per
// batch on its own factors (one forward + backward apply, CUDA events), before the first
// iteration; the choice does not change any result (each slice is computed the same way by
// whichever warp, in either kind).
// The task sweep launched: task_kernel 0 = one CTA per task with the factor slices staged
// through shared memory (k_trsv_task), K > 0 = one thread-block cluster of K CTAs per task
// (k_trsv_cluster).
int Batch::launch_tasks(Ctx &ctx, int which) {
  cudaStream_t s = ctx.stream;
  if (task_kernel == 0)
    return mixed ? vk_trsv_task_f32(ntasks, d_sysdev, d_state, d_active, d_tasks, d_chunks, d_sdesc, which, d_bar, d_err, s)
                 : vk_trsv_task_f64(ntasks, d_sysdev, d_state, d_active, d_tasks, d_chunks, d_sdesc, which, d_bar, d_err, s);
  return mixed ? vk_trsv_cluster_f32(ntasks, task_kernel, d_sysdev, d_state, d_active, d_ctasks, d_clv, which, s)
               : vk_trsv_cluster_f64(ntasks, task_kernel, d_sysdev, d_state, d_active, d_ctasks, d_clv, which, s);
}

// Autotuner of the task sweep: one apply of each candidate (staged single CTA; clusters of 2, 4
// and 8 CTAs) timed on the batch's own factors with CUDA events, once per batch before its first
// iteration; the fastest is kept.  Every candidate computes every row the same way, so the
// choice changes no result.
int Batch::autotune_tasks(Ctx &ctx) {
  if (ctx.task_sweep >= 0 && task_kernel != ctx.task_sweep) {
    task_kernel = ctx.task_sweep;
    if (chunk_exec) { cudaGraphExecDestroy(chunk_exec); chunk_exec = nullptr; }
  }
  if (ctx.task_sweep >= 0 || tasks_tuned || !has_pc || ntasks == 0) return VSHE_OK;
  tasks_tuned = true;
  {
    auto it = ctx.task_choice.find(tune_key_tasks);
    if (it != ctx.task_choice.end()) {
      if (task_kernel != it->second) {
        task_kernel = it->second;
        if (chunk_exec) { cudaGraphExecDestroy(chunk_exec); chunk_exec = nullptr; }
      }
      return VSHE_OK;
    }
  }
  cudaStream_t s = ctx.stream;
  cudaEvent_t a, b;
  cudaEventCreate(&a); cudaEventCreate(&b);
  double best = 1e30;
  int best_k = task_kernel;
  task_tune_ms.clear();
  for (int k : {0, 2, 4, 8}) {
    task_kernel = k;
    int rc = launch_tasks(ctx, 0);  // warm-up
    cudaEventRecord(a, s);
    for (int r = 0; r < 3; ++r) rc |= launch_tasks(ctx, 0);
    cudaEventRecord(b, s);
    cudaError_t e = cudaEventSynchronize(b);
    if (rc || e != cudaSuccess) { cudaEventDestroy(a); cudaEventDestroy(b); return ctx.cuda_fail(e != cudaSuccess ? e : cudaError_t(rc), "autotune task sweeps"); }
    float ms = 0;
    cudaEventElapsedTime(&ms, a, b);
    task_tune_ms.push_back(ms / 3.0);
    if (ms < best) { best = ms; best_k = k; }
  }
  cudaEventDestroy(a); cudaEventDestroy(b);
  task_kernel = best_k;
  ctx.task_choice[tune_key_tasks] = best_k;
  if (chunk_exec) { cudaGraphExecDestroy(chunk_exec); chunk_exec = nullptr; }
  return check_err(ctx, "autotune task sweeps");
}

int Batch::autotune_trsv(Ctx &ctx) {
  const int mode = sys[0]->opts.trsv_mode;
  if (mode == VSHE_TRSV_FLOW) trsv_kernel = 3;
  if (trsv_tuned || !has_pc || !grid_group || mode == VSHE_TRSV_PER_LEVEL) return VSHE_OK;
  trsv_tuned = true;
  {
    auto it = ctx.trsv_choice.find(tune_key_grid);
    if (it != ctx.trsv_choice.end()) {
      if (trsv_grid != it->second.first || trsv_kernel != it->second.second) {
        trsv_grid = it->second.first;
        trsv_kernel = it->second.second;
        if (chunk_exec) { cudaGraphExecDestroy(chunk_exec); chunk_exec = nullptr; }
      }
      return VSHE_OK;
    }
  }
  cudaStream_t s = ctx.stream;
  cudaEvent_t a, b;
  cudaEventCreate(&a); cudaEventCreate(&b);
  double best = 1e30;
  int best_grid = trsv_grid, best_kernel = trsv_kernel;
  for (int kernel : {1, 3}) {
    if ((kernel == 3) != (mode == VSHE_TRSV_FLOW)) continue;
    for (int per_sm = 1; per_sm <= trsv_bps_max; ++per_sm) {
      const int grid = per_sm * num_sms;
      int rc = 0;
      auto apply = [&]() {
        return mixed ? vk_trsv_f32(kernel, grid, d_sysdev, d_state, d_active, &levL, &levU, 0, d_bar, d_err, s)
                     : vk_trsv_f64(kernel, grid, d_sysdev, d_state, d_active, &levL, &levU, 0, d_bar, d_err, s);
      };
      rc |= apply();  // warm-up
      cudaEventRecord(a, s);
      for (int r = 0; r < 3; ++r) rc |= apply();
      cudaEventRecord(b, s);
      cudaError_t e = cudaEventSynchronize(b);
      if (rc || e != cudaSuccess) { cudaEventDestroy(a); cudaEventDestroy(b); return ctx.cuda_fail(e != cudaSuccess ? e : cudaError_t(rc), "autotune sweeps"); }
      float ms = 0;
      cudaEventElapsedTime(&ms, a, b);
      trsv_tune_ms.push_back(ms / 3.0);
      if (ms < best) { best = ms; best_grid = grid; best_kernel = kernel; }
    }
  }
  cudaEventDestroy(a); cudaEventDestroy(b);
  trsv_grid = best_grid;
  trsv_kernel = best_kernel;
  ctx.trsv_choice[tune_key_grid] = {best_grid, best_kernel};
  if (chunk_exec) { cudaGraphExecDestroy(chunk_exec); chunk_exec = nullptr; }  // the graph holds the old grid
  return check_err(ctx, "autotune sweeps");
}

// A small pool of CUDA events for the per-kernel-class timing of a profiled solve.
struct EventProf {
  bool on = false;
  cudaStream_t s = nullptr;
  std::vector<cudaEvent_t> pool;
  std::vector<std::pair<int, std::pair<cudaEvent_t, cudaEvent_t>>> recs;
  size_t used = 0;
  cudaEvent_t get() {
    if (used == pool.size()) { cudaEvent_t e; cudaEventCreate(&e); pool.push_back(e); }
    return pool[used++];
  }
  cudaEvent_t begin() {
    if (!on) return nullptr;
    cudaEvent_t a = get();
    cudaEventRecord(a, s);
    return a;
  }
  void end(int cls, cudaEvent_t a) {
    if (!on) return;
    cudaEvent_t b = get();
    cudaEventRecord(b, s);
    recs.push_back({cls, {a, b}});
  }
  void collect(double *out, int64_t *counts) {
    for (auto &r : recs) {
      float ms = 0;
      cudaEventElapsedTime(&ms, r.second.first, r.second.second);
      out[r.first] += ms;
      if (r.first < 2) counts[r.first] += 1;
    }
    recs.clear();
    used = 0;
  }
  ~EventProf() { for (auto e : pool) cudaEventDestroy(e); }
};
static thread_local EventProf g_prof;

// BiCGStab (FP64) on every active system to relative tolerance `tol`; the ILU(0) apply runs
// in the factor precision.  resume = true continues after a residual replacement (r holds
// b - A x).  Iteration chunks of `check_every` run without host synchronisation.
// Sets the iteration parameters of the active members and (re)starts their recurrences:
// resume = false: x = 0, r = b (k_bicg_init); true: r already holds b - A x (k_bicg_resume).
int Batch::start(Ctx &ctx, double tol, int max_iter, bool resume) {
  cudaStream_t s = ctx.stream;
  if (sys[0]->opts.trsv_mode < VSHE_TRSV_AUTO || sys[0]->opts.trsv_mode > VSHE_TRSV_PER_BLOCK)
    return ctx.fail(VSHE_E_INVALID_ARGUMENT, "trsv_mode");
  const size_t bsz = vk_bistate_size();
  std::vector<char> stbuf;
  int rc = read_states(ctx, stbuf);
  if (rc) return rc;
  for (int k = 0; k < nsys; ++k) {
    if (!act_host.empty() && !act_host[size_t(k)]) continue;
    BiState *b = (BiState *)(stbuf.data() + bsz * size_t(k));
    b->tol = tol; b->max_iter = max_iter;
    b->shadow_r0 = sys[size_t(k)]->opts.shadow == VSHE_SHADOW_R0 ? 1 : 0;
    if (!resume) { b->done = 0; b->iter = 0; }
  }
  cudaError_t e;
  if ((e = cudaMemcpyAsync(d_state, stbuf.data(), stbuf.size(), cudaMemcpyHostToDevice, s)) != cudaSuccess) return ctx.cuda_fail(e, "write state");
  if (resume) vk_bicg_resume(ntiles, d_sysdev, d_state, &tiles, d_partials, d_counters, d_active, s);
  else vk_bicg_init(ntiles, d_sysdev, d_state, &tiles, d_partials, d_counters, d_active, s);
  return VSHE_OK;
}

int Batch::read_states(Ctx &ctx, std::vector<char> &out) {
  out.assign(vk_bistate_size() * size_t(nsys), 0);
  cudaError_t e = cudaMemcpyAsync(out.data(), d_state, out.size(), cudaMemcpyDeviceToHost, ctx.stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx.stream);
  if (e != cudaSuccess) return ctx.cuda_fail(e, "read state");
  return VSHE_OK;
}

int Batch::write_states(Ctx &ctx, const std::vector<char> &in) {
  cudaError_t e = cudaMemcpyAsync(d_state, in.data(), std::min(in.size(), vk_bistate_size() * size_t(nsys)), cudaMemcpyHostToDevice, ctx.stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx.stream);
  if (e != cudaSuccess) return ctx.cuda_fail(e, "write state");
  return VSHE_OK;
}

// One chunk of `every` BiCGStab iterations of every active, unfinished member: 7 launches per
// iteration (update_p, forward/backward sweeps, SpMV + dots, update_s, sweeps, SpMV + dots,
// update_xr), no host synchronisation.  The chunk is captured once into a CUDA graph (every
// kernel reads its scalars from the device-resident state, so one graph serves every chunk) and
// replayed; under profiling, or if the driver refuses the capture, it is launched directly.
int Batch::run_chunk(Ctx &ctx, int every) {
  int rs = sync_spin_limit(ctx);
  if (rs) return rs;
  cudaStream_t s = ctx.stream;
  const int mode = (sys[0]->opts.trsv_mode == VSHE_TRSV_PER_LEVEL) ? 2 : trsv_kernel;
  const int lvl_grid = mode != 2 ? trsv_grid : std::max(1, num_sms * 8);
  EventProf &P = g_prof;
  P.on = profile; P.s = s;
  auto trsv = [&](int which) -> int {
    if (!has_pc) { vk_precond_copy(ntiles, d_sysdev, d_state, &tiles, d_active, which, s); return 0; }
    int rc = 0;
    if (ntasks) {
      rc = launch_tasks(ctx, which);
      if (rc) return rc;
    }
    if (!grid_group) return 0;
    if (mixed) return vk_trsv_f32(mode, lvl_grid, d_sysdev, d_state, d_active, &levL, &levU, which, d_bar, d_err, s);
    return vk_trsv_f64(mode, lvl_grid, d_sysdev, d_state, d_active, &levL, &levU, which, d_bar, d_err, s);
  };
  auto chunk = [&]() -> int {
    int rc = 0;
    for (int it = 0; it < every; ++it) {
      cudaEvent_t a;
      a = P.begin(); vk_update_p(ntiles, d_sysdev, d_state, &tiles, d_active, s); P.end(2, a);
      a = P.begin(); rc |= trsv(0); P.end(1, a);
      a = P.begin(); vk_spmv_dot(ntiles, d_sysdev, d_state, &tiles, d_partials, d_counters, d_active, 0, s); P.end(0, a);
      a = P.begin(); vk_update_s(ntiles, d_sysdev, d_state, &tiles, d_partials, d_counters, d_active, s); P.end(2, a);
      a = P.begin(); rc |= trsv(1); P.end(1, a);
      a = P.begin(); vk_spmv_dot(ntiles, d_sysdev, d_state, &tiles, d_partials, d_counters, d_active, 1, s); P.end(0, a);
      a = P.begin(); vk_update_xr(ntiles, d_sysdev, d_state, &tiles, d_partials, d_counters, d_active, s); P.end(2, a);
    }
    return rc;
  };
  const bool use_graph = !profile && !graph_failed && std::getenv("VSHE_NO_GRAPHS") == nullptr;
  if (use_graph && (!chunk_exec || chunk_every != every)) {
    if (chunk_exec) { cudaGraphExecDestroy(chunk_exec); chunk_exec = nullptr; }
    const long long l0 = vk_launches_total();
    cudaGraph_t g = nullptr;
    cudaError_t eb = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal);
    int rcap = eb == cudaSuccess ? chunk() : 1;
    cudaError_t ee = eb == cudaSuccess ? cudaStreamEndCapture(s, &g) : eb;
    chunk_launches = vk_launches_total() - l0;
    vk_count_launches(-chunk_launches);  // captured, not executed
    if (eb != cudaSuccess || rcap || ee != cudaSuccess || !g || cudaGraphInstantiate(&chunk_exec, g, 0) != cudaSuccess) {
      chunk_exec = nullptr;
      graph_failed = true;
      (void)cudaGetLastError();
    }
    if (g) cudaGraphDestroy(g);
    chunk_every = every;
  }
  cudaError_t e;
  if (use_graph && chunk_exec) {
    if ((e = cudaGraphLaunch(chunk_exec, s)) != cudaSuccess) return ctx.cuda_fail(e, "graph launch");
    vk_count_launches(chunk_launches);
    return VSHE_OK;
  }
  int rc = chunk();
  if (rc) return ctx.cuda_fail(cudaError_t(rc), "trsv launch");
  return VSHE_OK;
}

// BiCGStab on every active member to relative tolerance `tol`, chunk by chunk, until all are
// done (converged, broken down or out of iterations).
int Batch::bicgstab(Ctx &ctx, double tol, int max_iter, bool resume, int &iters_out) {
  cudaStream_t s = ctx.stream;
  const int every = sys[0]->opts.check_every > 0 ? sys[0]->opts.check_every : 8;
  const size_t bsz = vk_bistate_size();
  int rc = start(ctx, tol, max_iter, resume);
  if (rc) return rc;
  EventProf &P = g_prof;
  std::vector<char> stbuf;
  int done_iters = 0;
  while (true) {
    if ((rc = run_chunk(ctx, every))) return rc;
    done_iters += every;
    if ((rc = read_states(ctx, stbuf))) return rc;
    if ((rc = check_err(ctx, "bicgstab"))) return rc;
    bool all_done = true;
    int maxit = 0;
    for (int k = 0; k < nsys; ++k) {
      const BiState *b = (const BiState *)(stbuf.data() + bsz * size_t(k));
      if (!b->done) all_done = false;
      maxit = std::max(maxit, int(b->iter));
    }
    iters_out = maxit;
    if (all_done || done_iters >= max_iter + 2 * every) break;
  }
  if (profile) {
    cudaError_t e;
    if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return ctx.cuda_fail(e, "profile");
    double t[5] = {0, 0, 0, 0, 0};
    int64_t c[2] = {0, 0};
    P.collect(t, c);
    t_spmv += t[0]; t_trsv += t[1]; t_vec += t[2];
    n_spmv += c[0]; n_trsv += c[1];
  }
  last_state.assign(stbuf.begin(), stbuf.end());
  return VSHE_OK;
}

int Batch::state_of(int k, int32_t &status, int32_t &iter) const {
  if (last_state.empty()) { status = 0; iter = 0; return 0; }
  const BiState *b = (const BiState *)(last_state.data() + vk_bistate_size() * size_t(k));
  status = b->status; iter = b->iter;
  return 0;
}

// FP64 residual r = b - A x for all active members (written into the Krylov r);
// returns per-system ||r|| / ||b||.
int Batch::residual(Ctx &ctx, std::vector<double> &rel) {
  cudaStream_t s = ctx.stream;
  vk_residual64(ntiles, d_refdev, &tiles, d_partials, d_counters, d_active, d_rnorm2, d_bnorm2, s);
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
  act_host = act;
  cudaError_t e = cudaMemcpyAsync(d_active, act.data(), sizeof(int32_t) * act.size(), cudaMemcpyHostToDevice, ctx.stream);
  if (e != cudaSuccess) return ctx.cuda_fail(e, "active flags");
  return VSHE_OK;
}

// Factor, iterate, then check every system's true FP64 residual; a system whose recursive
// residual met the tolerance but whose true residual does not is resumed from r = b - A x
// (at most kMaxReplacements times, within its iteration budget).
int Batch::solve(Ctx &ctx, std::vector<vshe_solve_stats> &stats) {
  constexpr int kMaxReplacements = 3;
  cudaStream_t s = ctx.stream;
  cudaError_t e;
  stats.assign(size_t(nsys), vshe_solve_stats{});
  profile = ctx.profile;
  t_spmv = t_trsv = t_vec = t_reliable = t_factor = 0;
  n_spmv = n_trsv = 0;
  cudaEvent_t e0, e1, e2;
  cudaEventCreate(&e0); cudaEventCreate(&e1); cudaEventCreate(&e2);
  struct EvGuard { cudaEvent_t a, b, c; ~EvGuard() { cudaEventDestroy(a); cudaEventDestroy(b); cudaEventDestroy(c); } } guard{e0, e1, e2};
  std::vector<int32_t> act((size_t)(nsys), 1);
  int rc = set_active(ctx, act);
  if (rc) return rc;
  cudaEventRecord(e0, s);
  for (System *S : sys) S->prepare(ctx);
  if ((rc = autotune_tiles(ctx))) return rc;
  rc = factor(ctx);
  if (rc) return rc;
  if ((rc = autotune_trsv(ctx))) return rc;
  if ((rc = autotune_tasks(ctx))) return rc;
  cudaEventRecord(e1, s);
  const vshe_solve_opts &o = sys[0]->opts;
  int it = 0;
  rc = bicgstab(ctx, o.tol, o.max_iters, false, it);
  if (rc) return rc;
  std::vector<double> rel;
  if ((rc = residual(ctx, rel))) return rc;  // true FP64 residual of the final x
  std::vector<int32_t> nrep((size_t)nsys, 0);
  for (int round = 0; round < kMaxReplacements; ++round) {
    bool any = false;
    for (int k = 0; k < nsys; ++k) {
      int32_t status, iters;
      state_of(k, status, iters);
      act[size_t(k)] = (status == 0 && rel[size_t(k)] >= o.tol && iters < o.max_iters) ? 1 : 0;
      if (act[size_t(k)]) { any = true; nrep[size_t(k)]++; }
    }
    if (!any) break;
    if ((rc = set_active(ctx, act))) return rc;
    if ((rc = bicgstab(ctx, o.tol, o.max_iters, true, it))) return rc;
    std::vector<double> rel2;
    if ((rc = residual(ctx, rel2))) return rc;
    for (int k = 0; k < nsys; ++k)
      if (act[size_t(k)]) rel[size_t(k)] = rel2[size_t(k)];
  }
  std::fill(act.begin(), act.end(), 1);
  if ((rc = set_active(ctx, act))) return rc;
  for (System *S : sys) vk_permute(S->n, S->d_perm, (const double *)S->kv[0], S->d_x64, 0, s);  // x back to caller order
  cudaEventRecord(e2, s);
  if ((e = cudaEventSynchronize(e2)) != cudaSuccess) return ctx.cuda_fail(e, "solve");
  float ms_setup = 0, ms_solve = 0;
  cudaEventElapsedTime(&ms_setup, e0, e1);
  cudaEventElapsedTime(&ms_solve, e1, e2);
  if (profile) {
    ctx.prof[0] = t_spmv; ctx.prof[1] = t_trsv; ctx.prof[2] = t_vec; ctx.prof[3] = 0.0; ctx.prof[4] = ms_setup;
    ctx.prof_counts[0] = n_spmv; ctx.prof_counts[1] = n_trsv;
  }
  for (int k = 0; k < nsys; ++k) {
    vshe_solve_stats &st = stats[size_t(k)];
    System *S = sys[size_t(k)];
    int32_t status, iters;
    state_of(k, status, iters);
    st.iterations = iters;
    st.refinements = nrep[size_t(k)];
    st.rel_residual = rel[size_t(k)];
    st.setup_ms = ms_setup;
    st.solve_ms = ms_solve;
    st.levels_L = S->nlevL;
    st.levels_U = S->nlevU;
    st.bytes_device = int64_t(S->arena.total);
    const int tk = task_kind.empty() ? 0 : task_kind[size_t(k)];
    st.sweep_ctas = !has_pc ? 0 : tk ? (task_kernel > 0 ? task_kernel : 1) : trsv_grid;
    st.sweep_mode = !has_pc ? 0
                    : tk == 1 ? VSHE_TRSV_PER_SYSTEM
                    : tk == 2 ? VSHE_TRSV_PER_BLOCK
                    : S->opts.trsv_mode == VSHE_TRSV_PER_LEVEL ? VSHE_TRSV_PER_LEVEL
                    : trsv_kernel == 3 ? VSHE_TRSV_FLOW : VSHE_TRSV_PERSISTENT;
    st.tile_rows = int32_t(S->tile_rows);
    int32_t code = status;
    if (code == 0 && rel[size_t(k)] >= o.tol) code = VSHE_E_NOT_CONVERGED;
    if (code != 0 && rel[size_t(k)] < o.tol) code = 0;
    st.status = code;
  }
  return VSHE_OK;
}

}  // namespace vshe

// =======================================================================
// public C ABI
// =======================================================================
using namespace vshe;

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
  vshe::she_release_all(ctx);
  vshe::poisson_release_all(ctx);
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
  for (auto &kv : ctx->batches) t += kv.second->arena.total + kv.second->tile_arena.total;
  return t + vshe::she_bytes(ctx) + vshe::poisson_bytes(ctx);
}

int vshe_set_task_sweep(vshe_ctx *ctx, int32_t kernel) {
  if (!ctx || kernel < -1 || kernel > 8 || kernel == 1 || (kernel > 2 && kernel != 4 && kernel != 8)) return VSHE_E_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lk(ctx->mu);
  ctx->task_sweep = kernel;
  return VSHE_OK;
}

int vshe_set_host_threads(int32_t threads) {
  if (threads < 0) return VSHE_E_INVALID_ARGUMENT;
  g_host_threads.store(threads);
  return VSHE_OK;
}

int vshe_set_spin_limit(vshe_ctx *ctx, uint64_t polls) {
  if (!ctx) return VSHE_E_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lk(ctx->mu);
  ctx->spin_limit = polls ? polls : kDefaultSpinLimit;
  return VSHE_OK;
}

int vshe_set_profiling(vshe_ctx *ctx, int32_t on) {
  if (!ctx) return VSHE_E_INVALID_ARGUMENT;
  ctx->profile = on != 0;
  return VSHE_OK;
}

int64_t vshe_kernel_launches(void) { return (int64_t)vk_launches_total(); }

int vshe_autotune_info(vshe_ctx *ctx, int64_t n, int64_t *tile_rows, double *ms) {
  if (!ctx || n <= 0 || !tile_rows) return VSHE_E_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lk(ctx->mu);
  int cls = 0;
  while ((int64_t(1) << (cls + 1)) <= n) ++cls;
  auto it = ctx->tile_choice.find(cls);
  if (it == ctx->tile_choice.end()) return ctx->fail(VSHE_E_NOT_FOUND, "no system of this size class solved yet");
  *tile_rows = it->second;
  if (ms) {
    const auto &t = ctx->tile_timings[cls];
    for (size_t k = 0; k < 4; ++k) ms[k] = k < t.size() ? t[k] : 0.0;
  }
  return VSHE_OK;
}

int vshe_get_profile(vshe_ctx *ctx, double *ms, int64_t *counts) {
  if (!ctx || !ms) return VSHE_E_INVALID_ARGUMENT;
  for (int k = 0; k < 5; ++k) ms[k] = ctx->prof[k];
  if (counts) { counts[0] = ctx->prof_counts[0]; counts[1] = ctx->prof_counts[1]; }
  return VSHE_OK;
}

int vshe_system_create(vshe_ctx *ctx, int64_t n, int64_t nnz, const int64_t *rp, const int32_t *ci, const double *v,
                       const double *rhs, const vshe_solve_opts *opts, int64_t *handle) {
  if (!ctx || !handle) return VSHE_E_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lk(ctx->mu);
  cudaSetDevice(ctx->device);
  vshe_solve_opts o;
  if (opts) o = *opts; else vshe_default_opts(&o);
  // admission against the HBM budget (upper estimate of the system's footprint)
  const size_t est = size_t(nnz) * (4 + 8 + 8 + 4 + 8 + 8 + 8 + 8) + size_t(n) * (8 * 8 + 9 * 8 + 32);
  if (vshe_bytes_in_use(ctx) + est > ctx->budget) return ctx->fail(VSHE_E_BUDGET, std::to_string(est) + " bytes requested");
  std::unique_ptr<System> S(new System);
  int rc = S->create(*ctx, n, nnz, rp, ci, v, rhs, o);
  if (rc) return rc;
  S->opts.block_ptr = nullptr;  // read during creation only
  S->opts.perm = nullptr;
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

// Pattern cache of vshe_solve_csr: the system of the last call stays resident with its solver
// order, schedules and tuned launch shapes; a call whose pattern (row offsets and columns,
// compared entry by entry) and options equal it uploads only values and rhs.  ILUT systems are
// not kept (their factor pattern comes from the values at creation).
static bool same_solve_opts(const vshe_solve_opts &a, const vshe_solve_opts &b) {
  return a.precision == b.precision && a.precond == b.precond && a.ordering == b.ordering && a.tol == b.tol &&
         a.max_iters == b.max_iters && a.n_blocks == b.n_blocks && a.trsv_mode == b.trsv_mode && a.check_every == b.check_every &&
         a.shadow == b.shadow && a.fill_level == b.fill_level && a.ilut_entries == b.ilut_entries && a.ilut_drop == b.ilut_drop;
}

int vshe_solve_csr(vshe_ctx *ctx, int64_t n, int64_t nnz, const int64_t *rp, const int32_t *ci, const double *v,
                   const double *rhs, const vshe_solve_opts *opts, double *x, vshe_solve_stats *stats) {
  if (!ctx || !x || !rhs || !rp || !ci || !v || n <= 0 || nnz <= 0) return VSHE_E_INVALID_ARGUMENT;
  vshe_solve_opts o;
  if (opts) o = *opts; else vshe_default_opts(&o);
  const bool keep = o.precond != VSHE_PRECOND_ILUT;
  const bool has_blocks = o.n_blocks > 0 && o.block_ptr;
  bool hit = false;
  {
    std::lock_guard<std::mutex> lk(ctx->mu);
    auto it = ctx->systems.find(ctx->csr_cache);
    if (keep && it != ctx->systems.end()) {
      const System *S = it->second.get();
      const bool blocks_same = has_blocks ? (ctx->csr_cache_blocks.size() == size_t(o.n_blocks) + 1 &&
                                             std::equal(ctx->csr_cache_blocks.begin(), ctx->csr_cache_blocks.end(), o.block_ptr))
                                          : ctx->csr_cache_blocks.empty();
      const bool perm_same = o.perm ? (ctx->csr_cache_perm.size() == size_t(n) && std::equal(ctx->csr_cache_perm.begin(), ctx->csr_cache_perm.end(), o.perm))
                                    : ctx->csr_cache_perm.empty();
      hit = S->n == n && S->nnz == nnz && same_solve_opts(ctx->csr_cache_opts, o) && blocks_same && perm_same &&
            host_equal(S->rp.data(), rp, sizeof(int64_t) * size_t(n + 1)) &&
            host_equal(S->ci.data(), ci, sizeof(int32_t) * size_t(nnz));
    }
  }
  int rc;
  if (hit) {
    rc = vshe_system_set_values(ctx, ctx->csr_cache, v, rhs);
    if (rc) return rc;
    return vshe_system_solve(ctx, ctx->csr_cache, x, stats);
  }
  if (ctx->csr_cache) {
    vshe_system_free(ctx, ctx->csr_cache);
    ctx->csr_cache = 0;
  }
  int64_t h = 0;
  rc = vshe_system_create(ctx, n, nnz, rp, ci, v, rhs, &o, &h);
  if (rc) return rc;
  rc = vshe_system_solve(ctx, h, x, stats);
  if (!keep) {
    vshe_system_free(ctx, h);
    return rc;
  }
  std::lock_guard<std::mutex> lk(ctx->mu);
  ctx->csr_cache = h;
  ctx->csr_cache_opts = o;
  ctx->csr_cache_opts.block_ptr = nullptr;
  ctx->csr_cache_opts.perm = nullptr;
  if (has_blocks) ctx->csr_cache_blocks.assign(o.block_ptr, o.block_ptr + o.n_blocks + 1);
  else ctx->csr_cache_blocks.clear();
  if (o.perm) ctx->csr_cache_perm.assign(o.perm, o.perm + n);
  else ctx->csr_cache_perm.clear();
  return rc;
}

int vshe_solve_csr_release(vshe_ctx *ctx) {
  if (!ctx) return VSHE_E_INVALID_ARGUMENT;
  if (ctx->csr_cache) vshe_system_free(ctx, ctx->csr_cache);
  ctx->csr_cache = 0;
  return VSHE_OK;
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
  if (precision != VSHE_PRECISION_FP64) return ctx->fail(VSHE_E_UNSUPPORTED, "the SpMV runs in FP64 in every solver mode");
  const int grid = std::max(1, int(std::min<int64_t>(S->nslA / 8 + 1, 148 * 32)));
  // the solver-order SELL copy of A, then y = A x through it; scratch: the search-direction
  // vectors (the solution x stays untouched)
  S->prepare(*ctx);
  double *dxo = (double *)S->kv[5], *dx = (double *)S->kv[3], *dy = (double *)S->kv[4];
  if ((e = cudaMemcpyAsync(dxo, x, sizeof(double) * size_t(S->n), cudaMemcpyHostToDevice, s)) != cudaSuccess) return ctx->cuda_fail(e, "x");
  vk_permute(S->n, S->d_perm, dxo, dx, 1, s);
  vk_spmv_plain(grid, S->n, S->d_aoff, S->d_acol, S->d_aval, dx, dy, s);
  vk_permute(S->n, S->d_perm, dy, dxo, 0, s);
  if ((e = cudaMemcpyAsync(y, dxo, sizeof(double) * size_t(S->n), cudaMemcpyDeviceToHost, s)) != cudaSuccess) return ctx->cuda_fail(e, "y");
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
  if (precision != VSHE_PRECISION_FP64) return ctx->fail(VSHE_E_UNSUPPORTED, "the SpMV runs in FP64 in every solver mode");
  cudaStream_t s = ctx->stream;
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int grid = std::max(1, int(std::min<int64_t>(S->nslA / 8 + 1, int64_t(sms) * 4)));
  S->prepare(*ctx);
  cudaEvent_t a, b;
  cudaEventCreate(&a); cudaEventCreate(&b);
  for (int w = 0; w < 3; ++w)
    vk_spmv_plain(grid, S->n, S->d_aoff, S->d_acol, S->d_aval, (const double *)S->kv[3], (double *)S->kv[4], s);
  cudaEventRecord(a, s);
  for (int r = 0; r < reps; ++r)
    vk_spmv_plain(grid, S->n, S->d_aoff, S->d_acol, S->d_aval, (const double *)S->kv[3], (double *)S->kv[4], s);
  cudaEventRecord(b, s);
  cudaError_t e = cudaEventSynchronize(b);
  float t = 0;
  cudaEventElapsedTime(&t, a, b);
  cudaEventDestroy(a); cudaEventDestroy(b);
  if (e != cudaSuccess) return ctx->cuda_fail(e, "time spmv");
  *ms = double(t) / reps;
  return VSHE_OK;
}

// Factor values of P A P^T (solver order) in A's entry order (FP64, host array of length nnz);
// entries coupling two blocks are not part of the factor and read 0.
int vshe_system_factor_values(vshe_ctx *ctx, int64_t h, double *lu) {
  if (!ctx || !lu) return VSHE_E_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lk(ctx->mu);
  cudaSetDevice(ctx->device);
  std::vector<int64_t> hs{h};
  int rc;
  Batch *B = get_batch(ctx, hs, rc);
  if (!B) return rc;
  if (!B->has_pc) return ctx->fail(VSHE_E_UNSUPPORTED, "no preconditioner");
  B->sys[0]->prepare(*ctx);
  rc = B->factor(*ctx);
  if (rc) return rc;
  System *S = B->sys[0];
  std::vector<double> lp((size_t)S->nnzF);
  std::vector<int64_t> amap((size_t)S->nnzF);
  std::vector<int32_t> pci((size_t)S->nnzF);
  std::vector<int64_t> prp((size_t)S->n + 1);
  cudaError_t e = cudaMemcpyAsync(lp.data(), S->d_lu64, sizeof(double) * lp.size(), cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(amap.data(), S->d_amap, sizeof(int64_t) * amap.size(), cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(pci.data(), S->d_pci, sizeof(int32_t) * pci.size(), cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(prp.data(), S->d_prp, sizeof(int64_t) * prp.size(), cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) return ctx->cuda_fail(e, "download factor");
  for (int64_t i = 0; i < S->n; ++i)
    for (int64_t k = prp[size_t(i)]; k < prp[size_t(i) + 1]; ++k) {
      if (amap[size_t(k)] < 0) continue;  // ILU(k) fill: not an entry of A
      const bool in_factor = S->blk[size_t(pci[size_t(k)])] == S->blk[size_t(i)];
      lu[amap[size_t(k)]] = in_factor ? lp[size_t(k)] : 0.0;
    }
  return VSHE_OK;
}

// Host-only view of the solver layout (no GPU): validates the inputs like vshe_system_create
// and builds the same Layout a resident system would use.
static int layout_for(int64_t n, int64_t nnz, const int64_t *rp, const int32_t *ci, const double *val, const vshe_solve_opts *opts, Layout &L) {
  if (n <= 0 || nnz <= 0 || !rp || !ci) return VSHE_E_INVALID_ARGUMENT;
  if (rp[0] != 0 || rp[n] != nnz) return VSHE_E_INVALID_ARGUMENT;
  std::vector<int64_t> vrp(rp, rp + n + 1);
  std::vector<int32_t> vci(ci, ci + nnz);
  for (int64_t i = 0; i < n; ++i) {
    if (vrp[size_t(i) + 1] < vrp[size_t(i)]) return VSHE_E_INVALID_ARGUMENT;
    if (vrp[size_t(i) + 1] == vrp[size_t(i)]) return VSHE_E_EMPTY_ROW;
    for (int64_t k = vrp[size_t(i)]; k < vrp[size_t(i) + 1]; ++k)
      if (vci[size_t(k)] < 0 || vci[size_t(k)] >= n || (k > vrp[size_t(i)] && vci[size_t(k)] <= vci[size_t(k) - 1])) return VSHE_E_INVALID_ARGUMENT;
  }
  vshe_solve_opts o;
  if (opts) o = *opts; else vshe_default_opts(&o);
  std::string err;
  return L.build(n, nnz, vrp, vci, o, val, err);
}

int vshe_layout_sweep_plan(int64_t n, int64_t nnz, const int64_t *rp, const int32_t *ci, const double *val, const vshe_solve_opts *opts,
                           int32_t num_sms, int64_t *counts, int32_t *tasks, int64_t *chunks, int32_t *sdesc) {
  if (!counts) return VSHE_E_INVALID_ARGUMENT;
  Layout L;
  int rc = layout_for(n, nnz, rp, ci, val, opts, L);
  if (rc) return rc;
  System S;
  S.n = n;
  S.nnz = nnz;
  if (opts) S.opts = *opts; else vshe_default_opts(&S.opts);
  S.adopt_layout(L);
  SweepPlan P;
  plan_sweep_tasks(std::vector<System *>{&S}, S.mixed, S.has_pc, num_sms > 0 ? num_sms : 148, P);
  counts[0] = int64_t(P.tasks.size());
  counts[1] = int64_t(P.chunks.size());
  counts[2] = int64_t(P.sdesc.size());
  counts[3] = P.on_task.empty() ? 0 : int64_t(P.on_task[0]);
  if (tasks)
    for (size_t t = 0; t < P.tasks.size(); ++t) {
      const TaskDev &d = P.tasks[t];
      const int32_t v[6] = {d.sys, d.cL0, d.cL1, d.cU0, d.cU1, d.pad};
      std::copy(v, v + 6, tasks + 6 * t);
    }
  if (chunks) {
    const int vbytes = S.mixed ? int(sizeof(float)) : int(sizeof(double));
    for (const TaskDev &d : P.tasks)
      for (int32_t c = d.cL0; c < d.cU1; ++c) {
        const ChunkDev &h = P.chunks[size_t(c)];
        const bool lower = c < d.cL1;
        const int64_t v[10] = {h.s0, h.s1, h.flags, h.nslot, h.o0, h.d0, h.r0, h.r1, h.rot,
                               task_chunk_bytes(h.s1 - h.s0, h.nslot, h.r0, h.r1, lower, vbytes)};
        std::copy(v, v + 10, chunks + 10 * size_t(c));
      }
  }
  if (sdesc)
    for (size_t k = 0; k < P.sdesc.size(); ++k) {
      const SliceDesc &d = P.sdesc[k];
      const int32_t v[4] = {d.soff, d.width, d.r0, d.nr};
      std::copy(v, v + 4, sdesc + 4 * k);
    }
  return VSHE_OK;
}

int vshe_layout_sizes(int64_t n, int64_t nnz, const int64_t *rp, const int32_t *ci, const double *val, const vshe_solve_opts *opts,
                      int64_t *sizes) {
  if (!sizes) return VSHE_E_INVALID_ARGUMENT;
  Layout L;
  int rc = layout_for(n, nnz, rp, ci, val, opts, L);
  if (rc) return rc;
  const int64_t v[10] = {L.nslA, L.padA, L.nslL, L.padL, L.nslU, L.padU, L.nlevL, L.nlevU, L.nnzL, L.nnzU};
  for (int k = 0; k < 10; ++k) sizes[k] = v[k];
  return VSHE_OK;
}

int vshe_layout_export(int64_t n, int64_t nnz, const int64_t *rp, const int32_t *ci, const double *val, const vshe_solve_opts *opts,
                       int32_t *perm, int64_t *lvr, int64_t *aoff, int32_t *acol, int64_t *amap_a,
                       int32_t *lrow0, int64_t *loff, int32_t *lcol, int64_t *lmap,
                       int32_t *uslot0, int64_t *uoff, int32_t *ucol, int64_t *umap, int32_t *urow) {
  Layout L;
  int rc = layout_for(n, nnz, rp, ci, val, opts, L);
  if (rc) return rc;
  auto put = [](auto *dst, const auto &src) { if (dst) for (size_t k = 0; k < src.size(); ++k) dst[k] = src[k]; };
  put(perm, L.perm);
  put(lvr, L.lvr);
  put(aoff, L.aoff);
  put(acol, L.acol);
  put(amap_a, L.amapS);
  put(lrow0, L.lstart);
  put(loff, L.loff);
  put(lcol, L.lcol);
  put(uslot0, L.ustart);
  put(uoff, L.uoff);
  put(ucol, L.ucol);
  put(urow, L.urow);
  // caller entry of every factor slot (-1: padding)
  if (lmap || umap) {
    std::vector<int64_t> lm((size_t)L.padL, -1), um((size_t)L.padU, -1);
    for (int64_t k = 0; k < nnz; ++k) {
      const int64_t m = L.fmap.empty() ? -1 : L.fmap[size_t(k)];
      if (m >= 0) lm[size_t(m)] = L.amap[size_t(k)];
      else if (m <= -2) um[size_t(-(m + 2))] = L.amap[size_t(k)];
    }
    put(lmap, lm);
    put(umap, um);
  }
  return VSHE_OK;
}

}  // extern "C"

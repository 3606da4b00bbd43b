// solver_kernels.cu -- sm_100a kernels of the Krylov solver (thin launchers at the end).
//
// Everything here is memory-bound sparse work: CSR SpMV with sub-warp row
// groups and fused dot products, BiCGStab vector updates fused with their
// reductions, level-scheduled ILU(0) factorisation and triangular solves run
// as persistent cooperative kernels with a bounded grid barrier per level,
// and the FP64 side of the mixed-precision solve (reliable updates).  No
// tensor cores: nothing on this path is a dense contraction.
//
// Batches: each kernel works on a batch of independent systems described by
// per-system pointer tables (SysDev) and row tiles that never straddle two
// systems; reductions are per tile and are finished by the last tile of each
// system, in a fixed order, so a system's iterates do not depend on what else
// is in the batch.
//
// BiCGStab follows van der Vorst (1992), right-preconditioned.  The shadow
// residual r^ is a fixed dense pseudo-random vector rather than r_0: the SHE
// right-hand side lives on the few contact rows only, and with r^ = r_0 the
// inner products (r^, r_k) collapse to rounding noise after a few iterations.
// Mixed precision runs the recurrences in FP32 and keeps x and the true
// residual in FP64 (reliable updates, Sleijpen & van der Vorst 1996): whenever
// the FP32 residual has dropped by `delta` since the last update, x64 += x32
// and the FP32 residual is replaced by b - A x64 computed in FP64.

#include <cuda_runtime.h>
#include <atomic>
#include <cstdint>
#include <cstdio>

#include "solver_kernels.cuh"
#include "kernels.h"

namespace vshe {

#define VSHE_E_BREAKDOWN_DEV (-5)
#define VSHE_E_NOT_CONVERGED_DEV (-6)
#define VSHE_E_TIMEOUT_DEV (-10)
#define VSHE_E_ZERO_PIVOT_DEV (-11)

constexpr int kThreads = 256;
constexpr double kReliableDelta = 0.1;

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Block-wide sums; results valid in thread 0.
template <typename T, int NV>
__device__ __forceinline__ void block_sum(T (&v)[NV]) {
  __shared__ T sh[NV][kThreads / 32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int i = 0; i < NV; ++i) v[i] = warp_sum(v[i]);
  if (lane == 0) {
#pragma unroll
    for (int i = 0; i < NV; ++i) sh[i][w] = v[i];
  }
  __syncthreads();
  if (w == 0) {
#pragma unroll
    for (int i = 0; i < NV; ++i) {
      T x = lane < (kThreads / 32) ? sh[i][lane] : T(0);
      v[i] = warp_sum(x);
    }
  }
  __syncthreads();
}

// Writes this tile's partial sums; if this block is the last tile of its
// system to arrive, sums all partials of the system in tile order into tot[]
// and returns true (in thread 0 only).
template <typename T, int NV>
__device__ bool tile_finish(T (&v)[NV], int tile, int sys, const Tiles &tl, T *partials, int32_t *counters, T (&tot)[NV]) {
  block_sum<T, NV>(v);
  __shared__ int is_last;
  if (threadIdx.x == 0) {
#pragma unroll
    for (int i = 0; i < NV; ++i) partials[(size_t)tile * 3 + i] = v[i];
    __threadfence();
    const int t0 = tl.sys_tile0[sys], t1 = tl.sys_tile0[sys + 1];
    int ticket = atomicAdd(&counters[sys], 1);
    is_last = (ticket == t1 - t0 - 1);
  }
  __syncthreads();
  if (!is_last) return false;
  __threadfence();
  const int t0 = tl.sys_tile0[sys], t1 = tl.sys_tile0[sys + 1];
  T acc[NV];
#pragma unroll
  for (int i = 0; i < NV; ++i) acc[i] = T(0);
  for (int t = t0 + (int)threadIdx.x; t < t1; t += kThreads) {
#pragma unroll
    for (int i = 0; i < NV; ++i) acc[i] += ((volatile T *)partials)[(size_t)t * 3 + i];
  }
  block_sum<T, NV>(acc);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int i = 0; i < NV; ++i) tot[i] = acc[i];
    counters[sys] = 0;
  }
  return threadIdx.x == 0;
}

// ------------------------------------------------------------ CSR row chunks
// Row sums of a chunk of nr <= 32 consecutive CSR rows starting at row q0 of (ptr, col, val):
// lane l returns sum_k val[k] * x[col[k]] over row q0 + l (0 for l >= nr).  The chunk's entries
// are one contiguous range; it is streamed with coalesced loads, U entries per lane in flight
// (all column/value loads of a pass first, then all x gathers), the products are staged in the
// warp's shared-memory slice sm[32 * U] and every lane sums its own row in index order, so the
// result does not depend on the launch shape.  CG: read x through L2 only (x is written by
// other CTAs of the same launch).
template <typename T, int U, bool CG>
__device__ __forceinline__ T chunk_rowsums(const int64_t *__restrict__ ptr, const int32_t *__restrict__ col, const T *__restrict__ val,
                                           const T *x, int64_t q0, int nr, T *sm) {
  const int lane = threadIdx.x & 31;
  int64_t b = 0, e = 0;
  if (lane < nr) { b = ptr[q0 + lane]; e = ptr[q0 + lane + 1]; }
  const int64_t kb = __shfl_sync(0xffffffffu, b, 0);
  const int64_t ke = __shfl_sync(0xffffffffu, e, nr - 1);
  T sum = T(0);
  for (int64_t pb = kb; pb < ke; pb += 32 * U) {
    int32_t c[U];
    T a[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int64_t k = pb + u * 32 + lane;
      c[u] = 0; a[u] = T(0);
      if (k < ke) { c[u] = col[k]; a[u] = val[k]; }
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int64_t k = pb + u * 32 + lane;
      T xv = T(0);
      if (k < ke) xv = CG ? __ldcg(&x[c[u]]) : x[c[u]];
      sm[u * 32 + lane] = a[u] * xv;
    }
    __syncwarp();
    const int64_t lo = b > pb ? b : pb;
    const int64_t hi = e < pb + 32 * U ? e : pb + 32 * U;
    for (int64_t k = lo; k < hi; ++k) sum += sm[k - pb];
    __syncwarp();
  }
  return sum;
}

constexpr int kWarps = kThreads / 32;
constexpr int kSpmvU = 12;  // entries per lane in flight: ~12 nnz per row fit one pass
constexpr int kTrsvU = 8;   // triangular factors hold about half of A's entries per row

template <typename T>
__device__ __forceinline__ T dsqrt(T x);
template <>
__device__ __forceinline__ float dsqrt<float>(float x) { return sqrtf(x); }
template <>
__device__ __forceinline__ double dsqrt<double>(double x) { return sqrt(x); }

// deterministic dense shadow residual in [0.5, 1.5): a hash of the row index
__device__ __forceinline__ float shadow_value(int64_t i) {
  uint32_t h = (uint32_t)((uint64_t)i * 2654435761ull) ^ (uint32_t)((uint64_t)i >> 32);
  h ^= h >> 16; h *= 0x7feb352dU; h ^= h >> 15; h *= 0x846ca68bU; h ^= h >> 16;
  return 0.5f + (float)(h >> 8) * (1.0f / 16777216.0f);
}

// ------------------------------------------------------------------ BiCGStab
// init: r holds the right-hand side; rh = shadow; x = p = v = 0; ||b||, (rh, r) -> state
template <typename T>
__global__ void __launch_bounds__(kThreads) k_bicg_init(const SysDev<T> *sys, BiState<T> *st, Tiles tl, T *partials, int32_t *counters, const int32_t *active) {
  const int tile = blockIdx.x;
  const int s = tl.tile_sys[tile];
  if (!active[s]) return;
  const SysDev<T> S = sys[s];
  T acc[2] = {T(0), T(0)};
  for (int64_t i = tl.tile_row0[tile] + threadIdx.x; i < tl.tile_row1[tile]; i += kThreads) {
    const T r = S.r[i];
    const T h = (T)shadow_value(i);
    S.rh[i] = h;
    S.x[i] = T(0); S.p[i] = T(0); S.v[i] = T(0);
    acc[0] += r * r;
    acc[1] += h * r;
  }
  T tot[2];
  if (tile_finish<T, 2>(acc, tile, s, tl, partials, counters, tot)) {
    BiState<T> &b = st[s];
    b.bnorm = dsqrt(tot[0]);
    b.rho = tot[1]; b.rho_old = T(1); b.alpha = T(1); b.omega = T(1);
    b.res = T(1); b.iter = 0; b.s_conv = 0; b.status = 0; b.upd = 0; b.restart = 1; b.nupd = 0;
    b.done = (tot[0] == T(0)) ? 1 : 0;
    if (b.done) b.res = T(0);
  }
}

// p = r + beta (p - omega v), or p = r after a (re)start
template <typename T>
__global__ void __launch_bounds__(kThreads) k_update_p(const SysDev<T> *sys, BiState<T> *st, Tiles tl, const int32_t *active) {
  const int tile = blockIdx.x;
  const int s = tl.tile_sys[tile];
  if (!active[s] || st[s].done) return;
  const SysDev<T> S = sys[s];
  const BiState<T> b = st[s];
  if (b.restart) {
    for (int64_t i = tl.tile_row0[tile] + threadIdx.x; i < tl.tile_row1[tile]; i += kThreads) S.p[i] = S.r[i];
  } else {
    const T beta = (b.rho / b.rho_old) * (b.alpha / b.omega);
    for (int64_t i = tl.tile_row0[tile] + threadIdx.x; i < tl.tile_row1[tile]; i += kThreads)
      S.p[i] = S.r[i] + beta * (S.p[i] - b.omega * S.v[i]);
  }
}

// y = A x over one tile (32-row chunks per warp), fused dots.
// which = 0: v = A ph, (rh, v) -> alpha.   which = 1: t = A sh, (t, s), (t, t) -> omega.
template <typename T>
__global__ void __launch_bounds__(kThreads) k_spmv_dot(const SysDev<T> *sys, BiState<T> *st, Tiles tl, T *partials, int32_t *counters, const int32_t *active, int which) {
  __shared__ T sm[kWarps][32 * kSpmvU];
  const int tile = blockIdx.x;
  const int s = tl.tile_sys[tile];
  if (!active[s] || st[s].done) return;
  if (which == 1 && st[s].s_conv) return;
  const SysDev<T> S = sys[s];
  const T *xin = which == 0 ? S.ph : S.sh;
  T *yout = which == 0 ? S.v : S.t;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int64_t r0 = tl.tile_row0[tile], r1 = tl.tile_row1[tile];
  T acc[2] = {T(0), T(0)};
  for (int64_t q0 = r0 + 32 * w; q0 < r1; q0 += 32 * kWarps) {
    const int nr = (int)(r1 - q0 < 32 ? r1 - q0 : 32);
    const T y = chunk_rowsums<T, kSpmvU, false>(S.rp, S.ci, S.av, xin, q0, nr, sm[w]);
    if (lane < nr) {
      const int64_t row = q0 + lane;
      yout[row] = y;
      if (which == 0) acc[0] += S.rh[row] * y;
      else { acc[0] += y * S.s[row]; acc[1] += y * y; }
    }
  }
  T tot[2];
  if (tile_finish<T, 2>(acc, tile, s, tl, partials, counters, tot)) {
    BiState<T> &b = st[s];
    if (which == 0) {
      if (tot[0] == T(0)) { b.alpha = T(0); b.s_conv = 0; b.status = VSHE_E_BREAKDOWN_DEV; }
      else b.alpha = b.rho / tot[0];
    } else {
      b.omega = tot[1] == T(0) ? T(0) : tot[0] / tot[1];
    }
  }
}

// s = r - alpha v, ||s|| -> s_conv
template <typename T>
__global__ void __launch_bounds__(kThreads) k_update_s(const SysDev<T> *sys, BiState<T> *st, Tiles tl, T *partials, int32_t *counters, const int32_t *active) {
  const int tile = blockIdx.x;
  const int s = tl.tile_sys[tile];
  if (!active[s] || st[s].done) return;
  const SysDev<T> S = sys[s];
  const T alpha = st[s].alpha;
  T acc[1] = {T(0)};
  for (int64_t i = tl.tile_row0[tile] + threadIdx.x; i < tl.tile_row1[tile]; i += kThreads) {
    T v = S.r[i] - alpha * S.v[i];
    S.s[i] = v;
    acc[0] += v * v;
  }
  T tot[1];
  if (tile_finish<T, 1>(acc, tile, s, tl, partials, counters, tot)) {
    BiState<T> &b = st[s];
    T sres = dsqrt(tot[0]) / b.bnorm;
    b.s_conv = (sres < b.tol) ? 1 : 0;
    if (b.s_conv) b.res = sres;
  }
}

// x += alpha ph + omega sh; r = s - omega t; ||r||, (rh, r) -> next rho, convergence.
// reliable = 1 (mixed): stopping is decided on the FP64 residual by k_reliable_r;
// here only a reliable update is requested.
template <typename T>
__global__ void __launch_bounds__(kThreads) k_update_xr(const SysDev<T> *sys, BiState<T> *st, Tiles tl, T *partials, int32_t *counters, const int32_t *active, int reliable) {
  const int tile = blockIdx.x;
  const int s = tl.tile_sys[tile];
  if (!active[s] || st[s].done) return;
  const SysDev<T> S = sys[s];
  const BiState<T> b0 = st[s];
  T acc[2] = {T(0), T(0)};
  if (b0.s_conv) {
    for (int64_t i = tl.tile_row0[tile] + threadIdx.x; i < tl.tile_row1[tile]; i += kThreads) {
      S.x[i] += b0.alpha * S.ph[i];
      T r = S.s[i];
      S.r[i] = r;
      acc[0] += r * r;
      acc[1] += S.rh[i] * r;
    }
  } else {
    for (int64_t i = tl.tile_row0[tile] + threadIdx.x; i < tl.tile_row1[tile]; i += kThreads) {
      S.x[i] += b0.alpha * S.ph[i] + b0.omega * S.sh[i];
      T r = S.s[i] - b0.omega * S.t[i];
      S.r[i] = r;
      acc[0] += r * r;
      acc[1] += S.rh[i] * r;
    }
  }
  T tot[2];
  if (tile_finish<T, 2>(acc, tile, s, tl, partials, counters, tot)) {
    BiState<T> &b = st[s];
    b.iter += 1;
    b.restart = 0;
    b.res = dsqrt(tot[0]) / b.bnorm;
    b.rho_old = b.rho;
    b.rho = tot[1];
    const bool broke = (b.status == VSHE_E_BREAKDOWN_DEV) || b.rho == T(0) || (!b.s_conv && b.omega == T(0));
    if (!reliable) {
      if (b.s_conv || b.res < b.tol) { b.done = 1; b.status = 0; return; }
      if (broke) { b.done = 1; b.status = VSHE_E_BREAKDOWN_DEV; return; }
      if (b.iter >= b.max_iter) { b.done = 1; b.status = VSHE_E_NOT_CONVERGED_DEV; }
      return;
    }
    // mixed: ask for an FP64 reliable update when ||r32|| dropped below the threshold (delta, or
    // the level at which the true residual would meet the tolerance), on breakdown, on a
    // non-finite value, or when the iteration budget is spent
    const bool bad = !isfinite(b.res) || !isfinite(b.rho) || !isfinite(b.alpha) || !isfinite(b.omega);
    if (bad) { b.bad = 1; b.status = 0; b.restart = 1; b.upd = 1; }
    else if (broke) { b.status = 0; b.restart = 1; b.upd = 1; }
    if (b.res < b.thresh || b.iter >= b.max_iter) b.upd = 1;
    b.s_conv = 0;
  }
}

// FP64 reliable update, part 1: x64 += sigma * x32, x32 = 0 (systems with upd set).  A cycle
// that went non-finite contributes nothing.
__global__ void __launch_bounds__(kThreads) k_reliable_x(const SysDev<float> *sys, const BiState<float> *st, Tiles tl, const int32_t *active) {
  const int tile = blockIdx.x;
  const int s = tl.tile_sys[tile];
  if (!active[s] || st[s].done || !st[s].upd) return;
  const SysDev<float> S = sys[s];
  const double sigma = st[s].sigma;
  const bool keep = !st[s].bad;
  for (int64_t i = tl.tile_row0[tile] + threadIdx.x; i < tl.tile_row1[tile]; i += kThreads) {
    if (keep) S.x64[i] += sigma * (double)S.x[i];
    S.x[i] = 0.0f;
  }
}

// FP64 reliable update, part 2: r64 = b - A x64; ||r64|| -> sigma_new, ||b||, convergence test.
// With force = 1 this is the initial residual of every active system (x64 = 0).
__global__ void __launch_bounds__(kThreads) k_reliable_r(const SysDev<float> *sys, BiState<float> *st, Tiles tl, double *partials, int32_t *counters, const int32_t *active, double tol64, int force) {
  __shared__ double sm[kWarps][32 * kSpmvU];
  const int tile = blockIdx.x;
  const int s = tl.tile_sys[tile];
  if (!active[s] || st[s].done) return;
  if (!force && !st[s].upd) return;
  const SysDev<float> S = sys[s];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int64_t r0 = tl.tile_row0[tile], r1 = tl.tile_row1[tile];
  double acc[2] = {0.0, 0.0};
  for (int64_t q0 = r0 + 32 * w; q0 < r1; q0 += 32 * kWarps) {
    const int nr = (int)(r1 - q0 < 32 ? r1 - q0 : 32);
    const double ax = chunk_rowsums<double, kSpmvU, false>(S.rp, S.ci, S.av64, S.x64, q0, nr, sm[w]);
    if (lane < nr) {
      const int64_t row = q0 + lane;
      const double bb = S.b64[row];
      const double r = bb - ax;
      S.r64[row] = r;
      acc[0] += r * r;
      acc[1] += bb * bb;
    }
  }
  double tot[2];
  if (tile_finish<double, 2>(acc, tile, s, tl, partials, counters, tot)) {
    BiState<float> &b = st[s];
    b.bnorm64 = sqrt(tot[1]);
    const double rn = sqrt(tot[0]);
    b.res64 = b.bnorm64 > 0 ? rn / b.bnorm64 : 0.0;
    b.sigma_new = rn;
    if (!force) b.nupd += 1;
    if (b.bnorm64 == 0.0 || b.res64 < tol64) { b.done = 1; b.status = 0; b.upd = 0; return; }
    if (!isfinite(rn)) { b.done = 1; b.status = VSHE_E_BREAKDOWN_DEV; b.upd = 0; return; }
    if (b.iter >= b.max_iter) { b.done = 1; b.status = VSHE_E_NOT_CONVERGED_DEV; b.upd = 0; return; }
  }
}

// FP64 reliable update, part 3: r32 = r64 / sigma_new (unit norm); the search direction p and
// v = A M^-1 p are carried over to the new scale (times sigma / sigma_new), so the Krylov
// recurrence continues without a restart; rho = (rh, r32).  force = 1: start of the solve
// (shadow residual, x32 = p = v = 0).
__global__ void __launch_bounds__(kThreads) k_reliable_scale(const SysDev<float> *sys, BiState<float> *st, Tiles tl, double *partials, int32_t *counters, const int32_t *active, double tol64, int force) {
  const int tile = blockIdx.x;
  const int s = tl.tile_sys[tile];
  if (!active[s] || st[s].done) return;
  if (!force && !st[s].upd) return;
  const SysDev<float> S = sys[s];
  const double inv = 1.0 / st[s].sigma_new;
  const float ratio = force ? 0.0f : (float)(st[s].sigma * inv);
  double acc[2] = {0.0, 0.0};
  for (int64_t i = tl.tile_row0[tile] + threadIdx.x; i < tl.tile_row1[tile]; i += kThreads) {
    const float r = (float)(S.r64[i] * inv);
    S.r[i] = r;
    float h;
    if (force) {
      h = shadow_value(i);
      S.rh[i] = h;
      S.x[i] = 0.0f; S.p[i] = 0.0f; S.v[i] = 0.0f;
    } else {
      h = S.rh[i];
      S.p[i] *= ratio;
      S.v[i] *= ratio;
    }
    acc[0] += (double)h * (double)r;
    acc[1] += (double)r * (double)r;
  }
  double tot[2];
  if (tile_finish<double, 2>(acc, tile, s, tl, partials, counters, tot)) {
    BiState<float> &b = st[s];
    if (force) {
      b.iter = 0; b.s_conv = 0; b.status = 0; b.nupd = 0; b.restart = 1;
      b.rho_old = 1.0f; b.alpha = 1.0f; b.omega = 1.0f;
    } else {
      b.rho_old *= ratio;
    }
    b.rho = (float)tot[0];
    b.sigma = b.sigma_new;
    b.bnorm = 1.0f;
    b.res = (float)sqrt(tot[1]);
    // the true residual meets tol64 once ||r32|| < tol64 * ||b|| / sigma; take the update a little before
    b.thresh = (float)fmax(kReliableDelta, 0.5 * tol64 * b.bnorm64 / b.sigma);
    b.upd = 0;
    b.bad = 0;
  }
}

// copy (no preconditioner): which 0: ph = p, which 1: sh = s
template <typename T>
__global__ void __launch_bounds__(kThreads) k_precond_copy(const SysDev<T> *sys, const BiState<T> *st, Tiles tl, const int32_t *active, int which) {
  const int tile = blockIdx.x;
  const int s = tl.tile_sys[tile];
  if (!active[s] || st[s].done) return;
  if (which == 1 && st[s].s_conv) return;
  const SysDev<T> S = sys[s];
  const T *in = which == 0 ? S.p : S.s;
  T *out = which == 0 ? S.ph : S.sh;
  for (int64_t i = tl.tile_row0[tile] + threadIdx.x; i < tl.tile_row1[tile]; i += kThreads) out[i] = in[i];
}

// ------------------------------------------------------------ grid barrier
// Generation barrier for a cooperative launch (all CTAs resident).  The spin is
// bounded: after `limit` polls the kernel records a timeout and every CTA leaves.
__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned *p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release_u32(unsigned *p, unsigned v) {
  asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

__device__ bool grid_barrier(unsigned *bar, int32_t *err) {
  __shared__ int ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    ok = 1;
    if (*((volatile int32_t *)err) != 0) ok = 0;
  }
  __syncthreads();
  if (!ok) return false;
  if (threadIdx.x == 0) {
    const unsigned nb = gridDim.x * gridDim.y * gridDim.z;
    const unsigned gen = ld_acquire_u32(&bar[1]);
    __threadfence();
    const unsigned arrived = atomicAdd(&bar[0], 1u);
    if (arrived == nb - 1) {
      bar[0] = 0;
      __threadfence();
      st_release_u32(&bar[1], gen + 1u);
    } else {
      unsigned long long spins = 0;
      const unsigned long long limit = 20000000ull;  // ~ 1-2 s with the backoff below
      while (ld_acquire_u32(&bar[1]) == gen) {
        if (++spins > limit) { atomicExch(err, VSHE_E_TIMEOUT_DEV); ok = 0; break; }
        if ((spins & 255) == 0 && *((volatile int32_t *)err) != 0) { ok = 0; break; }  // another CTA gave up
        if (spins > 64) __nanosleep(32);
      }
    }
    if (ok && *((volatile int32_t *)err) != 0) ok = 0;
  }
  __syncthreads();
  return ok != 0;
}

// ------------------------------------------------- triangular solves (ILU apply)
// out = P^T U^{-1} L^{-1} P in over the level-ordered factors.  which 0: ph = M^{-1} p, 1: sh = M^{-1} s.
// A level is a list of chunks (system, first level-ordered position, row count <= 32); the
// warps of the grid take its chunks in turn.  ytmp (permuted order) is written by other CTAs
// of the same launch and read through L2 only.
template <typename T>
__device__ __forceinline__ void trsv_level_rows(const SysDev<T> *sys, const BiState<T> *st, const int32_t *active, const Levels lv, int k,
                                                bool lower, int which, T *sm) {
  const int lane = threadIdx.x & 31;
  const int64_t gw = ((int64_t)blockIdx.x * kThreads + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * kThreads) >> 5;
  const int64_t c1 = lv.lvl_ptr[k + 1];
  for (int64_t c = lv.lvl_ptr[k] + gw; c < c1; c += nw) {
    const int s = lv.ent_sys[c];
    if (!active[s] || st[s].done || (which == 1 && st[s].s_conv)) continue;
    const SysDev<T> &S = sys[s];
    const int64_t q0 = lv.ent_row[c];
    const int nr = lv.ent_cnt[c];
    if (lower) {
      const T sum = chunk_rowsums<T, kTrsvU, true>(S.lptr, S.lcol, S.lval, S.ytmp, q0, nr, sm);
      if (lane < nr) {
        const int64_t q = q0 + lane;
        const T *in = which == 0 ? S.p : S.s;
        S.ytmp[S.lrow[q]] = in[S.lgat[q]] - sum;
      }
    } else {
      const T sum = chunk_rowsums<T, kTrsvU, true>(S.uptr, S.ucol, S.uval, S.ytmp, q0, nr, sm);
      if (lane < nr) {
        const int64_t q = q0 + lane;
        const int32_t row = S.urow[q];
        const T y = (__ldcg(&S.ytmp[row]) - sum) * S.udinv[q];
        S.ytmp[row] = y;
        T *out = which == 0 ? S.ph : S.sh;
        out[S.ugat[q]] = y;
      }
    }
  }
}

template <typename T>
__global__ void __launch_bounds__(kThreads) k_trsv_persistent(const SysDev<T> *sys, const BiState<T> *st, const int32_t *active, Levels lL, Levels lU, int which, unsigned *bar, int32_t *err) {
  __shared__ T sm[kWarps][32 * kTrsvU];
  T *my = sm[threadIdx.x >> 5];
  for (int k = 0; k < lL.nlev; ++k) {
    trsv_level_rows<T>(sys, st, active, lL, k, true, which, my);
    if (!grid_barrier(bar, err)) return;
  }
  for (int k = 0; k < lU.nlev; ++k) {
    trsv_level_rows<T>(sys, st, active, lU, k, false, which, my);
    if (k + 1 < lU.nlev && !grid_barrier(bar, err)) return;
  }
}

template <typename T>
__global__ void __launch_bounds__(kThreads) k_trsv_level(const SysDev<T> *sys, const BiState<T> *st, const int32_t *active, Levels lv, int k, int lower, int which) {
  __shared__ T sm[kWarps][32 * kTrsvU];
  trsv_level_rows<T>(sys, st, active, lv, k, lower != 0, which, sm[threadIdx.x >> 5]);
}

// ------------------------------------------------------ ILU(0) factorisation
// Row-wise IKJ ILU(0) (Saad, Alg. 10.4) restricted to within-block entries,
// one warp per row, rows of a level in parallel.  Values in FP64.
__device__ __forceinline__ int64_t find_col(const int32_t *ci, int64_t a, int64_t b, int32_t j) {
  int64_t lo = a, hi = b - 1;
  while (lo <= hi) {
    int64_t mid = (lo + hi) >> 1;
    int32_t c = ci[mid];
    if (c == j) return mid;
    if (c < j) lo = mid + 1; else hi = mid - 1;
  }
  return -1;
}

// level entries here are permuted-space row ids (ent_row = row) of system ent_sys
__device__ void ilu0_level_rows(const FactDev *fs, Levels lv, int k, int32_t *err) {
  const int lane = threadIdx.x & 31;
  const int64_t gid = ((int64_t)blockIdx.x * kThreads + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * kThreads) >> 5;
  const int64_t e0 = lv.lvl_ptr[k], e1 = lv.lvl_ptr[k + 1];
  for (int64_t e = e0 + gid; e < e1; e += nw) {
    const int s = lv.ent_sys ? lv.ent_sys[e] : 0;
    const FactDev F = fs[s];
    const int64_t i = lv.ent_row[e];
    const int64_t a = F.rp[i], b = F.rp[i + 1], d = F.diag[i];
    const int32_t bi = F.blk[i];
    for (int64_t kp = a; kp < d; ++kp) {
      const int32_t c = F.ci[kp];
      if (F.blk[c] != bi) continue;
      const double piv = __ldcg(&F.lu[F.diag[c]]);
      if (piv == 0.0) {
        if (lane == 0) atomicExch(err, VSHE_E_ZERO_PIVOT_DEV);
        break;
      }
      const double l = __ldcg(&F.lu[kp]) / piv;
      __syncwarp();
      if (lane == 0) F.lu[kp] = l;
      for (int64_t kk = F.diag[c] + 1 + lane; kk < F.rp[c + 1]; kk += 32) {
        const int32_t j = F.ci[kk];
        if (F.blk[j] != bi) continue;
        const int64_t pos = find_col(F.ci, kp + 1, b, j);
        if (pos >= 0) F.lu[pos] = __ldcg(&F.lu[pos]) - l * __ldcg(&F.lu[kk]);
      }
      __syncwarp();
    }
  }
}

__global__ void __launch_bounds__(kThreads) k_ilu0_persistent(const FactDev *fs, Levels lv, unsigned *bar, int32_t *err) {
  for (int k = 0; k < lv.nlev; ++k) {
    ilu0_level_rows(fs, lv, k, err);
    if (k + 1 < lv.nlev && !grid_barrier(bar, err)) return;
  }
}

__global__ void __launch_bounds__(kThreads) k_ilu0_level(const FactDev *fs, Levels lv, int k, int32_t *err) {
  ilu0_level_rows(fs, lv, k, err);
}

// permuted factor values from A: lu[kp] = av[amap[kp]]
__global__ void k_gather_values(int64_t nnz, const int64_t *amap, const double *av, double *lu) {
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < nnz; k += (int64_t)gridDim.x * blockDim.x)
    lu[k] = av[amap[k]];
}

// Split the permuted factor (FP64, permuted CSR) into level-ordered L, U and the
// inverse diagonal in precision T: fmap[kp] >= 0 -> L slot, <= -2 -> U slot -(fmap+2),
// -1 -> not part of the factor; dpos[row] is the U-level position of the row.
template <typename T>
__global__ void k_split_factor(int64_t nnz, int64_t n, const double *lu, const int64_t *fmap, const int64_t *diag, const int64_t *dpos,
                               T *lval, T *uval, T *udinv) {
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < nnz; k += (int64_t)gridDim.x * blockDim.x) {
    const int64_t m = fmap[k];
    if (m >= 0) lval[m] = (T)lu[k];
    else if (m <= -2) uval[-(m + 2)] = (T)lu[k];
  }
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    udinv[dpos[i]] = (T)(1.0 / lu[diag[i]]);
}

// ------------------------------------------------------- FP64 residual
// r = b - A x (FP64), ||r||^2 and ||b||^2 per system -> rnorm2 / bnorm2.
__global__ void __launch_bounds__(kThreads) k_residual64(const RefDev *sys, Tiles tl, double *partials, int32_t *counters, const int32_t *active, double *rnorm2, double *bnorm2) {
  __shared__ double sm[kWarps][32 * kSpmvU];
  const int tile = blockIdx.x;
  const int s = tl.tile_sys[tile];
  if (!active[s]) return;
  const RefDev S = sys[s];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int64_t r0 = tl.tile_row0[tile], r1 = tl.tile_row1[tile];
  double acc[2] = {0.0, 0.0};
  for (int64_t q0 = r0 + 32 * w; q0 < r1; q0 += 32 * kWarps) {
    const int nr = (int)(r1 - q0 < 32 ? r1 - q0 : 32);
    const double ax = chunk_rowsums<double, kSpmvU, false>(S.rp, S.ci, S.av, S.x, q0, nr, sm[w]);
    if (lane < nr) {
      const int64_t row = q0 + lane;
      const double bb = S.b[row];
      const double r = bb - ax;
      S.r[row] = r;
      acc[0] += r * r;
      acc[1] += bb * bb;
    }
  }
  double tot[2];
  if (tile_finish<double, 2>(acc, tile, s, tl, partials, counters, tot)) {
    rnorm2[s] = tot[0];
    bnorm2[s] = tot[1];
  }
}

__global__ void k_cast_f64_f32(int64_t n, const double *a, float *b) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) b[i] = (float)a[i];
}

// plain SpMV for tests / timing (y = A x): the warps of the grid take 32-row chunks in turn
template <typename T>
__global__ void __launch_bounds__(kThreads) k_spmv_plain(int64_t n, const int64_t *rp, const int32_t *ci, const T *av, const T *x, T *y) {
  __shared__ T sm[kWarps][32 * kSpmvU];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int64_t gw = (int64_t)blockIdx.x * kWarps + w, nw = (int64_t)gridDim.x * kWarps;
  for (int64_t q0 = 32 * gw; q0 < n; q0 += 32 * nw) {
    const int nr = (int)(n - q0 < 32 ? n - q0 : 32);
    const T v = chunk_rowsums<T, kSpmvU, false>(rp, ci, av, x, q0, nr, sm[w]);
    if (lane < nr) y[q0 + lane] = v;
  }
}

}  // namespace vshe

// =====================================================================
// thin launchers (declared in kernels.h)
// =====================================================================
using namespace vshe;

static inline int grid_for(int64_t n) {
  int64_t g = (n + kThreads - 1) / kThreads;
  if (g > 65535LL * 16) g = 65535LL * 16;
  if (g < 1) g = 1;
  return (int)g;
}

static std::atomic<long long> g_launches{0};

template <typename T>
static int launch_trsv_t(int mode, int grid, const SysDev<T> *sys, const BiState<T> *st, const int32_t *act, Levels lL, Levels lU, int which, unsigned *bar, int32_t *err, cudaStream_t s) {
  if (mode == 1) {
    g_launches += 1;
    void *args[] = {(void *)&sys, (void *)&st, (void *)&act, (void *)&lL, (void *)&lU, (void *)&which, (void *)&bar, (void *)&err};
    return (int)cudaLaunchCooperativeKernel((void *)k_trsv_persistent<T>, dim3(grid), dim3(kThreads), args, 0, s);
  }
  g_launches += lL.nlev + lU.nlev;
  for (int pass = 0; pass < 2; ++pass) {
    const Levels &lv = pass == 0 ? lL : lU;
    for (int k = 0; k < lv.nlev; ++k) k_trsv_level<T><<<grid, kThreads, 0, s>>>(sys, st, act, lv, k, 1 - pass, which);
  }
  return (int)cudaGetLastError();
}

extern "C" {

int vk_threads() { return kThreads; }
void vk_count_launches(long long k) { g_launches += k; }
long long vk_launches_total() { return g_launches.load(); }

#define VK_BODY_T(T, SUF)                                                                                             \
  void vk_bicg_init_##SUF(int ntiles, const void *sys, void *st, const VkTiles *tl, T *part, int32_t *cnt,           \
                          const int32_t *act, cudaStream_t s) {                                                      \
    g_launches += 1;                                                                                                 \
    k_bicg_init<T><<<ntiles, kThreads, 0, s>>>((const SysDev<T> *)sys, (BiState<T> *)st, *(const Tiles *)tl, part, cnt, act); \
  }                                                                                                                  \
  void vk_update_p_##SUF(int ntiles, const void *sys, void *st, const VkTiles *tl, const int32_t *act,              \
                         cudaStream_t s) {                                                                           \
    g_launches += 1;                                                                                                 \
    k_update_p<T><<<ntiles, kThreads, 0, s>>>((const SysDev<T> *)sys, (BiState<T> *)st, *(const Tiles *)tl, act);    \
  }                                                                                                                  \
  void vk_spmv_dot_##SUF(int ntiles, const void *sys, void *st, const VkTiles *tl, T *part, int32_t *cnt,            \
                         const int32_t *act, int which, cudaStream_t s) {                                            \
    g_launches += 1;                                                                                                 \
    k_spmv_dot<T><<<ntiles, kThreads, 0, s>>>((const SysDev<T> *)sys, (BiState<T> *)st, *(const Tiles *)tl, part, cnt, act, which); \
  }                                                                                                                  \
  void vk_update_s_##SUF(int ntiles, const void *sys, void *st, const VkTiles *tl, T *part, int32_t *cnt,           \
                         const int32_t *act, cudaStream_t s) {                                                       \
    g_launches += 1;                                                                                                 \
    k_update_s<T><<<ntiles, kThreads, 0, s>>>((const SysDev<T> *)sys, (BiState<T> *)st, *(const Tiles *)tl, part, cnt, act); \
  }                                                                                                                  \
  void vk_update_xr_##SUF(int ntiles, const void *sys, void *st, const VkTiles *tl, T *part, int32_t *cnt,          \
                          const int32_t *act, int reliable, cudaStream_t s) {                                        \
    g_launches += 1;                                                                                                 \
    k_update_xr<T><<<ntiles, kThreads, 0, s>>>((const SysDev<T> *)sys, (BiState<T> *)st, *(const Tiles *)tl, part, cnt, act, reliable); \
  }                                                                                                                  \
  void vk_precond_copy_##SUF(int ntiles, const void *sys, const void *st, const VkTiles *tl, const int32_t *act,    \
                             int which, cudaStream_t s) {                                                            \
    g_launches += 1;                                                                                                 \
    k_precond_copy<T><<<ntiles, kThreads, 0, s>>>((const SysDev<T> *)sys, (const BiState<T> *)st, *(const Tiles *)tl, act, which); \
  }                                                                                                                  \
  int vk_trsv_##SUF(int mode, int grid, const void *sys, const void *st, const int32_t *act, const VkLevels *lL,     \
                    const VkLevels *lU, int which, unsigned *bar, int32_t *err, cudaStream_t s) {                    \
    return launch_trsv_t<T>(mode, grid, (const SysDev<T> *)sys, (const BiState<T> *)st, act, *(const Levels *)lL,   \
                            *(const Levels *)lU, which, bar, err, s);                                                \
  }                                                                                                                  \
  int vk_trsv_occupancy_##SUF(int *blocks_per_sm) {                                                                  \
    return (int)cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, (void *)k_trsv_persistent<T>, kThreads, 0); \
  }                                                                                                                  \
  void vk_split_factor_##SUF(int64_t nnz, int64_t n, const double *lu, const int64_t *fmap, const int64_t *diag,     \
                             const int64_t *dpos, T *lval, T *uval, T *udinv, cudaStream_t s) {                      \
    g_launches += 1;                                                                                                 \
    k_split_factor<T><<<grid_for(nnz > n ? nnz : n), kThreads, 0, s>>>(nnz, n, lu, fmap, diag, dpos, lval, uval, udinv); \
  }                                                                                                                  \
  void vk_spmv_plain_##SUF(int grid, int64_t n, const int64_t *rp, const int32_t *ci, const T *av, const T *x, T *y, \
                           cudaStream_t s) {                                                                         \
    g_launches += 1;                                                                                                 \
    k_spmv_plain<T><<<grid, kThreads, 0, s>>>(n, rp, ci, av, x, y);                                                  \
  }

VK_BODY_T(float, f32)
VK_BODY_T(double, f64)

void vk_reliable_x(int ntiles, const void *sys32, const void *st, const VkTiles *tl, const int32_t *act, cudaStream_t s) {
  g_launches += 1;
  k_reliable_x<<<ntiles, kThreads, 0, s>>>((const SysDev<float> *)sys32, (const BiState<float> *)st, *(const Tiles *)tl, act);
}

void vk_reliable_r(int ntiles, const void *sys32, void *st, const VkTiles *tl, double *part, int32_t *cnt,
                   const int32_t *act, double tol64, int force, cudaStream_t s) {
  const SysDev<float> *S = (const SysDev<float> *)sys32;
  BiState<float> *B = (BiState<float> *)st;
  const Tiles t = *(const Tiles *)tl;
  g_launches += 2;
  k_reliable_r<<<ntiles, kThreads, 0, s>>>(S, B, t, part, cnt, act, tol64, force);
  k_reliable_scale<<<ntiles, kThreads, 0, s>>>(S, B, t, part, cnt, act, tol64, force);
}

int vk_ilu0(int mode, int grid, const void *fs, const VkLevels *lv, unsigned *bar, int32_t *err, cudaStream_t s) {
  const FactDev *f = (const FactDev *)fs;
  Levels L = *(const Levels *)lv;
  if (mode == 1) {
    g_launches += 1;
    void *args[] = {(void *)&f, (void *)&L, (void *)&bar, (void *)&err};
    return (int)cudaLaunchCooperativeKernel((void *)k_ilu0_persistent, dim3(grid), dim3(kThreads), args, 0, s);
  }
  g_launches += L.nlev;
  for (int k = 0; k < L.nlev; ++k) k_ilu0_level<<<grid, kThreads, 0, s>>>(f, L, k, err);
  return (int)cudaGetLastError();
}

int vk_ilu0_occupancy(int *blocks_per_sm) {
  return (int)cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, (void *)k_ilu0_persistent, kThreads, 0);
}

void vk_gather_values(int64_t nnz, const int64_t *amap, const double *av, double *lu, cudaStream_t s) {
  g_launches += 1;
  k_gather_values<<<grid_for(nnz), kThreads, 0, s>>>(nnz, amap, av, lu);
}

size_t vk_factdev_size() { return sizeof(FactDev); }
size_t vk_refdev_size() { return sizeof(RefDev); }
size_t vk_sysdev_size_f32() { return sizeof(SysDev<float>); }
size_t vk_sysdev_size_f64() { return sizeof(SysDev<double>); }
size_t vk_bistate_size_f32() { return sizeof(BiState<float>); }
size_t vk_bistate_size_f64() { return sizeof(BiState<double>); }

void vk_residual64(int ntiles, const void *ref, const VkTiles *tl, double *part, int32_t *cnt, const int32_t *act,
                   double *rnorm2, double *bnorm2, cudaStream_t s) {
  g_launches += 1;
  k_residual64<<<ntiles, kThreads, 0, s>>>((const RefDev *)ref, *(const Tiles *)tl, part, cnt, act, rnorm2, bnorm2);
}

void vk_cast_f64_f32(int64_t n, const double *a, float *b, cudaStream_t s) {
  g_launches += 1;
  k_cast_f64_f32<<<grid_for(n), kThreads, 0, s>>>(n, a, b);
}

}  // extern "C"

// solver_kernels.cu -- sm_100a kernels of the Krylov solver (thin launchers at the end).
//
// Everything here is memory-bound sparse work: SELL-32 SpMV fused with the dot products that
// follow it, BiCGStab vector updates fused with their reductions, level-scheduled ILU(0)
// factorisation and triangular solves run as persistent cooperative kernels with a bounded
// grid barrier per level.  No tensor cores: nothing on this path is a dense contraction.
//
// Data layout (solver_kernels.cuh): every system is solved in a level-sorted "solver order"
// and A, L, U are SELL-32 slices, one row per lane, so value and column loads are coalesced
// lines, every row is summed by one thread in index order (deterministic, launch-shape
// independent) and the triangular solves read and write their vectors without index maps.
//
// Batches: each kernel works on a batch of independent systems described by per-system
// pointer tables (SysDev) and row tiles that never straddle two systems; reductions are per
// tile and are finished by the last tile of each system, in a fixed order, so a system's
// iterates do not depend on what else is in the batch.
//
// BiCGStab follows van der Vorst (1992), right-preconditioned, in FP64.  The shadow residual
// r^ is a fixed dense pseudo-random vector rather than r_0: the SHE right-hand side lives on
// the few contact rows only, and with r^ = r_0 the inner products (r^, r_k) collapse to
// rounding noise.  Mixed precision stores the ILU(0) factors in FP32 and reads them into FP64
// triangular solves; SpMV, dot products and vector updates stay FP64.  A fixed FP32 rounding
// of the factors is just another (linear) preconditioner of the same quality, while FP32
// arithmetic in the solves or FP32 Krylov vectors turn the preconditioner into a noisy one
// that BiCGStab's short recurrences do not tolerate: on the 2D bar they cost 2-6x the
// iterations or break down.

#include <cooperative_groups.h>
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
constexpr int kWarps = kThreads / 32;
constexpr int kSpmvU = 8;  // SELL entries per lane whose loads are issued together
constexpr int kVecU = 4;   // rows per thread whose loads the vector updates issue together
constexpr int kDotU = 6;   // the same inside the tile kernels, which also carry reduction state
constexpr int kTrsvU = 8;  // entries of a factor row loaded at once (factor rows hold ~5 entries)
// CTAs per SM the grid-wide sweeps are compiled for (40 registers, some spilled): up to 6 CTAs
// of slices in flight per SM.  The autotuner picks 1 .. 6; on the 2D bar 6 beat 4 by 3 %.
constexpr int kTrsvCtasPerSm = 6;

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Block-wide sums; results valid in thread 0.
template <typename T, int NV>
__device__ __forceinline__ void block_sum(T (&v)[NV]) {
  __shared__ T sh[NV][kWarps];
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
      T x = lane < kWarps ? sh[i][lane] : T(0);
      v[i] = warp_sum(x);
    }
  }
  __syncthreads();
}

// Writes this tile's partial sums; if this block is the last tile of its
// system to arrive, sums all partials of the system in tile order into tot[]
// and returns true (in thread 0 only).
template <int NV>
__device__ bool tile_finish(double (&v)[NV], int tile, int sys, const Tiles &tl, double *partials, int32_t *counters, double (&tot)[NV]) {
  block_sum<double, NV>(v);
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
  double acc[NV];
#pragma unroll
  for (int i = 0; i < NV; ++i) acc[i] = 0.0;
  for (int t = t0 + (int)threadIdx.x; t < t1; t += kThreads) {
#pragma unroll
    for (int i = 0; i < NV; ++i) acc[i] += ((volatile double *)partials)[(size_t)t * 3 + i];
  }
  block_sum<double, NV>(acc);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int i = 0; i < NV; ++i) tot[i] = acc[i];
    counters[sys] = 0;
  }
  return threadIdx.x == 0;
}

// ------------------------------------------------------------ SELL-32 rows
// Lane `lane` of a warp sums row `lane` of one SELL-32 slice: sum_k val[off + 32 k + lane] *
// x[col[off + 32 k + lane]] for k < width, in index order with FP64 fused multiply-adds, so the
// result does not depend on the launch shape.  All column and value loads of a group of kU
// entries are issued before their gathers of x.  Values and columns are read once per sweep
// (streaming loads, evict-first); CG: x is written by other CTAs of the same launch and is
// read through L2 only.
template <typename V, bool CG, int kU>
__device__ __forceinline__ double sell_rowsum(int64_t off, int width, const int32_t *__restrict__ col, const V *__restrict__ val,
                                              const double *x) {
  const int lane = threadIdx.x & 31;
  const int32_t *c = col + off + lane;
  const V *a = val + off + lane;
  double sum = 0.0;
  for (int k = 0; k < width; k += kU) {
    // the width is the same for all lanes of the slice: the masks below are warp-uniform
    int32_t cc[kU];
    V aa[kU];
#pragma unroll
    for (int u = 0; u < kU; ++u) {
      cc[u] = 0; aa[u] = V(0);
      if (k + u < width) { cc[u] = __ldcs(c + 32 * u); aa[u] = __ldcs(a + 32 * u); }
    }
    double xx[kU];
#pragma unroll
    for (int u = 0; u < kU; ++u) {
      xx[u] = 0.0;
      if (k + u < width) xx[u] = CG ? __ldcg(x + cc[u]) : __ldg(x + cc[u]);
    }
#pragma unroll
    for (int u = 0; u < kU; ++u)
      if (k + u < width) sum = fma((double)aa[u], xx[u], sum);
    c += 32 * kU; a += 32 * kU;
  }
  return sum;
}

// Continues a SELL-32 row sum from entry k0 (entries below k0 already summed into `sum`), kU
// entries per round trip; CG: x is written by other CTAs of the same launch (L2 reads).  The
// global-load sweeps use kU = 1: 8 per round trip cost registers and spills, and measured slower
// on the 2D bar with ILU(1) (cluster sweep 1.00 vs 0.76 ms per apply).
template <typename V, bool CG, int kU>
__device__ __forceinline__ double sell_rowsum_from(int64_t off, int width, int k0, const int32_t *__restrict__ col, const V *__restrict__ val,
                                                const double *x, double sum) {
  const int lane = threadIdx.x & 31;
  for (int k = k0; k < width; k += kU) {
    int32_t cc[kU];
    V aa[kU];
#pragma unroll
    for (int u = 0; u < kU; ++u) {
      cc[u] = 0; aa[u] = V(0);
      if (k + u < width) { const int64_t e = off + 32 * (k + u) + lane; cc[u] = __ldcs(col + e); aa[u] = __ldcs(val + e); }
    }
    double xx[kU];
#pragma unroll
    for (int u = 0; u < kU; ++u) xx[u] = k + u < width ? (CG ? __ldcg(x + cc[u]) : x[cc[u]]) : 0.0;
#pragma unroll
    for (int u = 0; u < kU; ++u)
      if (k + u < width) sum = fma((double)aa[u], xx[u], sum);
  }
  return sum;
}

// deterministic dense shadow residual in [0.5, 1.5): a hash of the row index
__device__ __forceinline__ double shadow_value(int64_t i) {
  uint32_t h = (uint32_t)((uint64_t)i * 2654435761ull) ^ (uint32_t)((uint64_t)i >> 32);
  h ^= h >> 16; h *= 0x7feb352dU; h ^= h >> 15; h *= 0x846ca68bU; h ^= h >> 16;
  return 0.5 + (double)(h >> 8) * (1.0 / 16777216.0);
}

typedef SysDev<double> SysK;  // the Krylov kernels touch only the FP64 members

// ------------------------------------------------------------------ BiCGStab
// init (x0 = 0): r = b, rh = shadow (or r_0), x = p = v = 0; ||b||, (rh, r) -> state
__device__ __forceinline__ void k_bicg_init_tile(const SysK *sys, BiState *st, const Tiles &tl, double *partials, int32_t *counters, const int32_t *active, int tile) {
  const int s = tl.tile_sys[tile];
  if (!active[s]) return;
  const SysK S = sys[s];
  const bool r0 = st[s].shadow_r0 != 0;
  double acc[2] = {0.0, 0.0};
  for (int64_t i = tl.tile_row0[tile] + threadIdx.x; i < tl.tile_row1[tile]; i += kThreads) {
    const double r = S.b[i];
    const double h = r0 ? r : shadow_value(i);
    S.r[i] = r;
    S.rh[i] = h;
    S.x[i] = 0.0; S.p[i] = 0.0; S.v[i] = 0.0;
    acc[0] += r * r;
    acc[1] += h * r;
  }
  double tot[2];
  if (tile_finish<2>(acc, tile, s, tl, partials, counters, tot)) {
    BiState &b = st[s];
    b.bnorm = sqrt(tot[0]);
    b.rho = tot[1]; b.rho_old = 1.0; b.alpha = 1.0; b.omega = 1.0;
    b.res = 1.0; b.iter = 0; b.s_conv = 0; b.status = 0; b.restart = 1;
    b.done = (tot[0] == 0.0) ? 1 : 0;
    if (b.done) b.res = 0.0;
  }
}
__global__ void __launch_bounds__(kThreads) k_bicg_init(const SysK *sys, BiState *st, Tiles tl, double *partials, int32_t *counters, const int32_t *active) {
  k_bicg_init_tile(sys, st, tl, partials, counters, active, blockIdx.x);
}

// resume after a residual replacement: r holds b - A x (true residual); restart the recurrence
__device__ __forceinline__ void k_bicg_resume_tile(const SysK *sys, BiState *st, const Tiles &tl, double *partials, int32_t *counters, const int32_t *active, int tile) {
  const int s = tl.tile_sys[tile];
  if (!active[s]) return;
  const SysK S = sys[s];
  double acc[2] = {0.0, 0.0};
  for (int64_t i = tl.tile_row0[tile] + threadIdx.x; i < tl.tile_row1[tile]; i += kThreads) {
    const double r = S.r[i];
    acc[0] += r * r;
    acc[1] += S.rh[i] * r;
  }
  double tot[2];
  if (tile_finish<2>(acc, tile, s, tl, partials, counters, tot)) {
    BiState &b = st[s];
    b.rho = tot[1]; b.rho_old = 1.0; b.alpha = 1.0; b.omega = 1.0;
    b.res = b.bnorm > 0.0 ? sqrt(tot[0]) / b.bnorm : 0.0;
    b.s_conv = 0; b.status = 0; b.restart = 1; b.done = 0;
  }
}
__global__ void __launch_bounds__(kThreads) k_bicg_resume(const SysK *sys, BiState *st, Tiles tl, double *partials, int32_t *counters, const int32_t *active) {
  k_bicg_resume_tile(sys, st, tl, partials, counters, active, blockIdx.x);
}

// p = r + beta (p - omega v), or p = r after a (re)start
__device__ __forceinline__ void k_update_p_tile(const SysK *sys, BiState *st, const Tiles &tl, const int32_t *active, int tile) {
  const int s = tl.tile_sys[tile];
  if (!active[s] || st[s].done) return;
  const SysK S = sys[s];
  const BiState b = st[s];
  if (b.restart) {
    for (int64_t i = tl.tile_row0[tile] + threadIdx.x; i < tl.tile_row1[tile]; i += kThreads) S.p[i] = S.r[i];
  } else {
    const double beta = (b.rho / b.rho_old) * (b.alpha / b.omega);
    const double *__restrict__ r = S.r;
    const double *__restrict__ v = S.v;
    double *__restrict__ p = S.p;
    const int64_t i1 = tl.tile_row1[tile];
    // kVecU rows per thread in flight: all loads of a group, then the updates
    for (int64_t i0 = tl.tile_row0[tile] + threadIdx.x; i0 < i1; i0 += kVecU * kThreads) {
      double rr[kVecU], pp[kVecU], vv[kVecU];
#pragma unroll
      for (int u = 0; u < kVecU; ++u) {
        const int64_t i = i0 + u * kThreads;
        rr[u] = i < i1 ? r[i] : 0.0; pp[u] = i < i1 ? p[i] : 0.0; vv[u] = i < i1 ? v[i] : 0.0;
      }
#pragma unroll
      for (int u = 0; u < kVecU; ++u)
        if (i0 + u * kThreads < i1) p[i0 + u * kThreads] = rr[u] + beta * (pp[u] - b.omega * vv[u]);
    }
  }
}
__global__ void __launch_bounds__(kThreads) k_update_p(const SysK *sys, BiState *st, Tiles tl, const int32_t *active) {
  k_update_p_tile(sys, st, tl, active, blockIdx.x);
}

// y = A x over one tile (one SELL-32 slice per warp in turn), fused dots.
// which = 0: v = A ph, (rh, v) -> alpha.   which = 1: t = A sh, (t, s), (t, t) -> omega.
__device__ __forceinline__ void k_spmv_dot_tile(const SysK *sys, BiState *st, const Tiles &tl, double *partials, int32_t *counters, const int32_t *active, int which, int tile) {
  const int s = tl.tile_sys[tile];
  if (!active[s] || st[s].done) return;
  if (which == 1 && st[s].s_conv) return;
  const SysK &S = sys[s];
  const int64_t *__restrict__ aoff = S.aoff;
  const int32_t *__restrict__ acol = S.acol;
  const double *__restrict__ aval = S.aval;
  const double *xin = which == 0 ? S.ph : S.sh;
  double *yout = which == 0 ? S.v : S.t;
  const double *dv = which == 0 ? S.rh : S.s;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int64_t r0 = tl.tile_row0[tile], r1 = tl.tile_row1[tile];
  double acc[2] = {0.0, 0.0};
  for (int64_t q0 = r0 + 32 * w; q0 < r1; q0 += 32 * kWarps) {
    const int64_t j = q0 >> 5, off = aoff[j];
    const double y = sell_rowsum<double, false, kSpmvU>(off, (int)((aoff[j + 1] - off) >> 5), acol, aval, xin);
    const int64_t row = q0 + lane;
    if (row < r1) {
      yout[row] = y;
      const double d = dv[row];
      if (which == 0) acc[0] += d * y;
      else { acc[0] += y * d; acc[1] += y * y; }
    }
  }
  double tot[2];
  if (tile_finish<2>(acc, tile, s, tl, partials, counters, tot)) {
    BiState &b = st[s];
    if (which == 0) {
      if (tot[0] == 0.0) { b.alpha = 0.0; b.s_conv = 0; b.status = VSHE_E_BREAKDOWN_DEV; }
      else b.alpha = b.rho / tot[0];
    } else {
      b.omega = tot[1] == 0.0 ? 0.0 : tot[0] / tot[1];
    }
  }
}
__global__ void __launch_bounds__(kThreads, 4) k_spmv_dot(const SysK *sys, BiState *st, Tiles tl, double *partials, int32_t *counters, const int32_t *active, int which) {
  k_spmv_dot_tile(sys, st, tl, partials, counters, active, which, blockIdx.x);
}

// s = r - alpha v, ||s|| -> s_conv
__device__ __forceinline__ void k_update_s_tile(const SysK *sys, BiState *st, const Tiles &tl, double *partials, int32_t *counters, const int32_t *active, int tile) {
  const int s = tl.tile_sys[tile];
  if (!active[s] || st[s].done) return;
  const SysK S = sys[s];
  const double alpha = st[s].alpha;
  double acc[1] = {0.0};
  const double *__restrict__ r = S.r;
  const double *__restrict__ vp = S.v;
  double *__restrict__ sp = S.s;
  const int64_t i1 = tl.tile_row1[tile];
  for (int64_t i0 = tl.tile_row0[tile] + threadIdx.x; i0 < i1; i0 += kVecU * kThreads) {
    double rr[kVecU], vv[kVecU];
#pragma unroll
    for (int u = 0; u < kVecU; ++u) {
      const int64_t i = i0 + u * kThreads;
      rr[u] = i < i1 ? r[i] : 0.0; vv[u] = i < i1 ? vp[i] : 0.0;
    }
#pragma unroll
    for (int u = 0; u < kVecU; ++u) {
      const int64_t i = i0 + u * kThreads;
      if (i < i1) {
        const double v = rr[u] - alpha * vv[u];
        sp[i] = v;
        acc[0] += v * v;
      }
    }
  }
  double tot[1];
  if (tile_finish<1>(acc, tile, s, tl, partials, counters, tot)) {
    BiState &b = st[s];
    const double sres = sqrt(tot[0]) / b.bnorm;
    b.s_conv = (sres < b.tol) ? 1 : 0;
    if (b.s_conv) b.res = sres;
  }
}
__global__ void __launch_bounds__(kThreads) k_update_s(const SysK *sys, BiState *st, Tiles tl, double *partials, int32_t *counters, const int32_t *active) {
  k_update_s_tile(sys, st, tl, partials, counters, active, blockIdx.x);
}

// x += alpha ph + omega sh; r = s - omega t; ||r||, (rh, r) -> next rho, convergence.
__device__ __forceinline__ void k_update_xr_tile(const SysK *sys, BiState *st, const Tiles &tl, double *partials, int32_t *counters, const int32_t *active, int tile) {
  const int s = tl.tile_sys[tile];
  if (!active[s] || st[s].done) return;
  const SysK S = sys[s];
  const BiState b0 = st[s];
  double acc[2] = {0.0, 0.0};
  if (b0.s_conv) {
    for (int64_t i = tl.tile_row0[tile] + threadIdx.x; i < tl.tile_row1[tile]; i += kThreads) {
      S.x[i] += b0.alpha * S.ph[i];
      const double r = S.s[i];
      S.r[i] = r;
      acc[0] += r * r;
      acc[1] += S.rh[i] * r;
    }
  } else {
    double *__restrict__ x = S.x;
    double *__restrict__ rp = S.r;
    const double *__restrict__ ph = S.ph;
    const double *__restrict__ sh = S.sh;
    const double *__restrict__ sv = S.s;
    const double *__restrict__ tv = S.t;
    const double *__restrict__ rh = S.rh;
    const int64_t i1 = tl.tile_row1[tile];
    for (int64_t i0 = tl.tile_row0[tile] + threadIdx.x; i0 < i1; i0 += kVecU * kThreads) {
      double xx[kVecU], pp[kVecU], ss[kVecU], sv_[kVecU], tt[kVecU], hh[kVecU];
#pragma unroll
      for (int u = 0; u < kVecU; ++u) {
        const int64_t i = i0 + u * kThreads;
        const bool in = i < i1;
        xx[u] = in ? x[i] : 0.0; pp[u] = in ? ph[i] : 0.0; ss[u] = in ? sh[i] : 0.0;
        sv_[u] = in ? sv[i] : 0.0; tt[u] = in ? tv[i] : 0.0; hh[u] = in ? rh[i] : 0.0;
      }
#pragma unroll
      for (int u = 0; u < kVecU; ++u) {
        const int64_t i = i0 + u * kThreads;
        if (i < i1) {
          x[i] = xx[u] + (b0.alpha * pp[u] + b0.omega * ss[u]);
          const double r = sv_[u] - b0.omega * tt[u];
          rp[i] = r;
          acc[0] += r * r;
          acc[1] += hh[u] * r;
        }
      }
    }
  }
  double tot[2];
  if (tile_finish<2>(acc, tile, s, tl, partials, counters, tot)) {
    BiState &b = st[s];
    b.iter += 1;
    b.restart = 0;
    b.res = sqrt(tot[0]) / b.bnorm;
    b.rho_old = b.rho;
    b.rho = tot[1];
    const bool broke = (b.status == VSHE_E_BREAKDOWN_DEV) || b.rho == 0.0 || (!b.s_conv && b.omega == 0.0) ||
                       !isfinite(b.res) || !isfinite(b.rho);
    if (b.s_conv || b.res < b.tol) { b.done = 1; b.status = 0; return; }
    if (broke) { b.done = 1; b.status = VSHE_E_BREAKDOWN_DEV; return; }
    if (b.iter >= b.max_iter) { b.done = 1; b.status = VSHE_E_NOT_CONVERGED_DEV; }
  }
}
__global__ void __launch_bounds__(kThreads) k_update_xr(const SysK *sys, BiState *st, Tiles tl, double *partials, int32_t *counters, const int32_t *active) {
  k_update_xr_tile(sys, st, tl, partials, counters, active, blockIdx.x);
}

// copy (no preconditioner): which 0: ph = p, which 1: sh = s
__device__ __forceinline__ void k_precond_copy_tile(const SysK *sys, const BiState *st, const Tiles &tl, const int32_t *active, int which, int tile) {
  const int s = tl.tile_sys[tile];
  if (!active[s] || st[s].done) return;
  if (which == 1 && st[s].s_conv) return;
  const SysK S = sys[s];
  const double *in = which == 0 ? S.p : S.s;
  double *out = which == 0 ? S.ph : S.sh;
  for (int64_t i = tl.tile_row0[tile] + threadIdx.x; i < tl.tile_row1[tile]; i += kThreads) out[i] = in[i];
}
__global__ void __launch_bounds__(kThreads) k_precond_copy(const SysK *sys, const BiState *st, Tiles tl, const int32_t *active, int which) {
  k_precond_copy_tile(sys, st, tl, active, which, blockIdx.x);
}

// ------------------------------------------------------------ grid barrier
// Generation barrier for a cooperative launch (all CTAs resident).  The spin is
// bounded: after `limit` polls the kernel records a timeout and every CTA leaves.
// bar[0] counts arrivals, bar[1] is the generation, bar[2..3] hold the poll limit (uint64) the
// host sets (vshe_set_spin_limit) for every wait of the batch's kernels.
__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned *p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release_u32(unsigned *p, unsigned v) {
  asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

__device__ __forceinline__ unsigned atom_add_acq_rel_u32(unsigned *p, unsigned v) {
  unsigned old;
  asm volatile("atom.acq_rel.gpu.global.add.u32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v) : "memory");
  return old;
}

// The arrival is one acquire-release atomic: its release half publishes the CTA's writes
// (ordered before it by the CTA barrier), its acquire half gives the last arriver everyone
// else's.  The generation is read before arriving, so the release cannot be missed.  A CTA that
// arrives after another has given up still arrives and leaves through the error check in its spin.
__device__ __forceinline__ unsigned long long spin_limit_of(const unsigned *bar) {
  return *((const volatile unsigned long long *)(bar + 2));
}

__device__ bool grid_barrier(unsigned *bar, int32_t *err) {
  __shared__ int ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    ok = 1;
    const unsigned nb = gridDim.x * gridDim.y * gridDim.z;
    const unsigned gen = ld_acquire_u32(&bar[1]);
    if (atom_add_acq_rel_u32(&bar[0], 1u) == nb - 1) {
      bar[0] = 0;
      st_release_u32(&bar[1], gen + 1u);
    } else {
      unsigned long long spins = 0;
      const unsigned long long limit = spin_limit_of(bar);  // default 20 M: ~ 1-2 s with the backoff below
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
// Barrier-free ("flow") sweeps: every row of ytmp and of the output starts the launch holding
// kPending, a NaN bit pattern that no arithmetic produces, and a row that reads a solved value
// polls that word until the row that produces it has written it.  The value is its own flag
// (one 8-byte word, written once per launch), so no fence is needed between a value and a flag.
constexpr unsigned long long kPending = 0x7FF4DEAD7FF4DEADull;

__device__ __forceinline__ double ld_flow(const double *p) {
  unsigned long long v;
  asm volatile("ld.relaxed.gpu.global.b64 %0, [%1];" : "=l"(v) : "l"(p));
  return __longlong_as_double((long long)v);
}
__device__ __forceinline__ void st_flow(double *p, double v) {
  asm volatile("st.relaxed.gpu.global.b64 [%0], %1;" ::"l"(p), "l"((unsigned long long)__double_as_longlong(v)) : "memory");
}
__device__ __forceinline__ bool is_pending(double v) { return (unsigned long long)__double_as_longlong(v) == kPending; }

// Polls *p until it holds a solved value; v is the value already loaded.  Gives up after
// `limit` polls (error word set to VSHE_E_TIMEOUT) or once another warp has set the error word,
// returning 0.
__device__ __noinline__ double wait_flow(const double *p, double v, int32_t *err, unsigned long long limit) {
  unsigned long long spins = 0;
  unsigned ns = 32;
  while (is_pending(v)) {
    if (++spins > limit) { atomicExch(err, VSHE_E_TIMEOUT_DEV); return 0.0; }
    if ((spins & 255) == 0 && *((volatile int32_t *)err) != 0) return 0.0;
    __nanosleep(ns);  // polls back off so that waiting lanes leave L2 to the working ones
    if (ns < 512) ns <<= 1;
    v = ld_flow(p);
  }
  return v;
}


// out = U^{-1} L^{-1} in (solver order) over SELL-32 factor slices stored in precision P;
// the arithmetic and the work vector ytmp are FP64 in both modes.  which 0: ph = M^{-1} p,
// 1: sh = M^{-1} s.  A level is a list of (system, slice) entries; the warps of the grid take
// them in turn, one slice per warp, one row per lane.  Forward slices are runs of consecutive
// solver rows; backward slices list their rows through urow.  ytmp and out are written by
// other CTAs of the same launch and read through L2 only.
// One SELL-32 slice of a triangular sweep as one warp holds it: lane = row.  The phases are
// split so that a warp can keep several slices' loads in flight: load() issues the slice's first
// kTrsvU entry loads together with the row's own operand (in[row] forward; urow, ytmp[row] and
// the inverse diagonal backward); finish() gathers the solved values at those columns, walks any
// further entries and writes the row.  Rows are summed in index order (FMA), as sell_rowsum.
template <typename P, bool CG, bool FLOW = false>
struct TrsvSlice {
  bool on = false;
  int width = 0, nr = 0;
  int64_t off = 0;
  const int32_t *col = nullptr;
  const P *val = nullptr;
  const double *src = nullptr;  // solved values gathered at the columns (ytmp / out)
  double *dst = nullptr;        // where the row's result goes (ytmp / out)
  int32_t row = 0;
  double base = 0.0, dinv = 1.0;
  int32_t cc[kTrsvU];
  P aa[kTrsvU];
  int32_t *err = nullptr;  // flow sweeps: the launch's error word and poll limit
  unsigned long long limit = 0;

  __device__ __forceinline__ void load(const SysDev<P> *sys, const BiState *st, const int32_t *active, const Levels &lv, int64_t c,
                                       bool lower, int which) {
    on = false;
    if (c < 0) return;
    const int s = lv.ent_sys[c];
    if (!active[s] || st[s].done || (which == 1 && st[s].s_conv)) return;
    load_slice(sys[s], lv.ent_row[c], lower, which);
  }

  __device__ __forceinline__ void load_slice(const SysDev<P> &S, int j, bool lower, int which) {
    const int lane = threadIdx.x & 31;
    on = true;
    if (lower) {
      off = S.loff[j];
      width = (int)((S.loff[j + 1] - off) >> 5);
      const int32_t q0 = S.lrow0[j];
      nr = S.lrow0[j + 1] - q0;
      col = S.lcol; val = S.lval; src = S.ytmp; dst = S.ytmp;
      row = q0 + lane;
      const double *in = which == 0 ? S.p : S.s;
      base = lane < nr ? in[row] : 0.0;
      dinv = 1.0;
    } else {
      off = S.uoff[j];
      width = (int)((S.uoff[j + 1] - off) >> 5);
      const int32_t t0 = S.uslot0[j];
      nr = S.uslot0[j + 1] - t0;
      col = S.ucol; val = S.uval;
      double *out = which == 0 ? S.ph : S.sh;
      src = out; dst = out;
      row = 0; base = 0.0; dinv = 1.0;
      if (lane < nr) {
        row = S.urow[t0 + lane];
        dinv = (double)S.udinv[t0 + lane];
        if constexpr (FLOW) {
          base = ld_flow(&S.ytmp[row]);
          if (is_pending(base)) base = wait_flow(&S.ytmp[row], base, err, limit);
        } else {
          base = CG ? __ldcg(&S.ytmp[row]) : S.ytmp[row];
        }
      }
    }
#pragma unroll
    for (int u = 0; u < kTrsvU; ++u) {
      cc[u] = 0; aa[u] = P(0);
      if (u < width) {
        const int64_t k = off + 32 * u + lane;
        cc[u] = __ldcs(col + k); aa[u] = __ldcs(val + k);
      }
    }
  }

  __device__ __forceinline__ void finish() {
    if (!on) return;
    const int lane = threadIdx.x & 31;
    double xx[kTrsvU];
    if constexpr (FLOW) {
#pragma unroll
      for (int u = 0; u < kTrsvU; ++u) xx[u] = u < width ? ld_flow(src + cc[u]) : 0.0;
#pragma unroll
      for (int u = 0; u < kTrsvU; ++u)
        if (u < width && is_pending(xx[u])) xx[u] = wait_flow(src + cc[u], xx[u], err, limit);
    } else {
#pragma unroll
      for (int u = 0; u < kTrsvU; ++u) xx[u] = u < width ? (CG ? __ldcg(src + cc[u]) : src[cc[u]]) : 0.0;
    }
    double sum = 0.0;
#pragma unroll
    for (int u = 0; u < kTrsvU; ++u)
      if (u < width) sum = fma((double)aa[u], xx[u], sum);
    if constexpr (FLOW) {
      for (int k = kTrsvU; k < width; ++k) {
        const int64_t e = off + 32 * k + lane;
        const int32_t c = __ldcs(col + e);
        const P a = __ldcs(val + e);
        double x = ld_flow(src + c);
        if (is_pending(x)) x = wait_flow(src + c, x, err, limit);
        sum = fma((double)a, x, sum);
      }
      if (lane < nr) st_flow(dst + row, (base - sum) * dinv);
    } else {
      if (width > kTrsvU) sum = sell_rowsum_from<P, CG, 1>(off, width, kTrsvU, col, val, src, sum);
      if (lane < nr) dst[row] = (base - sum) * dinv;
    }
  }
};

// out = U^{-1} L^{-1} in (solver order) over SELL-32 factor slices stored in precision P;
// the arithmetic and the work vector ytmp are FP64 in both modes.  which 0: ph = M^{-1} p,
// 1: sh = M^{-1} s.  A level is a list of (system, slice) entries; the warps of the grid take
// them two at a time, one row per lane.  ytmp and out are written by other CTAs of the same
// launch and read through L2 only.
template <typename P>
__device__ __forceinline__ void trsv_level_rows(const SysDev<P> *sys, const BiState *st, const int32_t *active, const Levels &lv, int k,
                                                bool lower, int which) {
  const int64_t gw = ((int64_t)blockIdx.x * kThreads + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * kThreads) >> 5;
  const int64_t c1 = lv.lvl_ptr[k + 1];
  for (int64_t c = lv.lvl_ptr[k] + gw; c < c1; c += nw) {
    TrsvSlice<P, true> a;
    a.load(sys, st, active, lv, c, lower, which);
    a.finish();
  }
}

template <typename P>
__global__ void __launch_bounds__(kThreads, kTrsvCtasPerSm) k_trsv_persistent(const SysDev<P> *sys, const BiState *st, const int32_t *active, Levels lL, Levels lU, int which, unsigned *bar, int32_t *err) {
  for (int k = 0; k < lL.nlev; ++k) {
    trsv_level_rows<P>(sys, st, active, lL, k, true, which);
    if (!grid_barrier(bar, err)) return;
  }
  for (int k = 0; k < lU.nlev; ++k) {
    trsv_level_rows<P>(sys, st, active, lU, k, false, which);
    if (k + 1 < lU.nlev && !grid_barrier(bar, err)) return;
  }
}

// Barrier-free sweeps in one cooperative launch.  Phase 1 marks every row that the launch will
// solve (ytmp for the forward slices, the output for the backward ones) as kPending; one grid
// barrier; phase 2 deals the forward then the backward slices of the merged level lists out to
// the warps in turn (entry g to warp g mod W, each warp in increasing g), and a row waits only on
// the rows it reads.  Deadlock-free because every warp is resident and takes its entries in
// increasing order: the lowest unfinished entry reads only finished rows.  Each row is summed in
// the same order as in k_trsv_persistent, so the results are bitwise the same.
template <typename P>
__global__ void __launch_bounds__(kThreads, kTrsvCtasPerSm) k_trsv_flow(const SysDev<P> *sys, const BiState *st, const int32_t *active, Levels lL, Levels lU, int which, unsigned *bar, int32_t *err) {
  const int lane = threadIdx.x & 31;
  const int64_t gw = ((int64_t)blockIdx.x * kThreads + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * kThreads) >> 5;
  const int64_t nL = lL.lvl_ptr[lL.nlev], nU = lU.lvl_ptr[lU.nlev];
  const double pend = __longlong_as_double((long long)kPending);
  const unsigned long long limit = spin_limit_of(bar);
  for (int64_t g = gw; g < nL + nU; g += nw) {
    const bool lower = g < nL;
    const int64_t c = lower ? g : g - nL;
    const int s = lower ? lL.ent_sys[c] : lU.ent_sys[c];
    if (!active[s] || st[s].done || (which == 1 && st[s].s_conv)) continue;
    const SysDev<P> &S = sys[s];
    const int j = lower ? lL.ent_row[c] : lU.ent_row[c];
    if (lower) {
      const int32_t q0 = S.lrow0[j];
      if (lane < S.lrow0[j + 1] - q0) S.ytmp[q0 + lane] = pend;
    } else {
      const int32_t t0 = S.uslot0[j];
      if (lane < S.uslot0[j + 1] - t0) (which == 0 ? S.ph : S.sh)[S.urow[t0 + lane]] = pend;
    }
  }
  if (!grid_barrier(bar, err)) return;
  for (int64_t g = gw; g < nL + nU; g += nw) {
    if (*((volatile int32_t *)err) != 0) return;
    const bool lower = g < nL;
    TrsvSlice<P, true, true> a;
    a.err = err;
    a.limit = limit;
    a.load(sys, st, active, lower ? lL : lU, lower ? g : g - nL, lower, which);
    a.finish();
  }
}

template <typename P>
__global__ void __launch_bounds__(kThreads) k_trsv_level(const SysDev<P> *sys, const BiState *st, const int32_t *active, Levels lv, int k, int lower, int which) {
  trsv_level_rows<P>(sys, st, active, lv, k, lower != 0, which);
}

// ------------------------------------------- per-task sweeps staged through shared memory
// mbarrier and bulk-copy primitives (PTX ISA 8.x; sm_90 and later).
__device__ __forceinline__ unsigned smem_u32(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Waits for the phase of the given parity to complete; gives up after `limit` polls (the error
// word is then set to VSHE_E_TIMEOUT) or once the error word is set by another thread.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, unsigned parity, unsigned long long limit, int32_t *err) {
  unsigned long long spins = 0;
  while (!mbar_try_wait(bar, parity)) {
    if (++spins > limit) { atomicExch(err, VSHE_E_TIMEOUT_DEV); return false; }
    if ((spins & 63) == 0 && *((volatile int32_t *)err) != 0) return false;
    if (spins > 16) __nanosleep(64);
  }
  return true;
}
// Waits for a phase regardless of the error word, at most kDrainPolls polls: copies in flight
// complete within microseconds, and shared memory must not be released under them.
constexpr unsigned long long kDrainPolls = 1ull << 24;
__device__ __forceinline__ void mbar_drain(uint64_t *bar, unsigned parity) {
  for (unsigned long long spins = 0; !mbar_try_wait(bar, parity) && spins < kDrainPolls; ++spins)
    if (spins > 16) __nanosleep(64);
}
// Bulk copy (the untiled TMA form) of `bytes` from global memory into this CTA's shared memory;
// completion is counted on the mbarrier.  Source, destination and size are multiples of 16 bytes.
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, unsigned bytes, uint64_t *bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}
// Barrier of the consumer warps only (named barrier 1; the producer warp does not take part).
__device__ __forceinline__ void consumers_sync(int nthreads) { asm volatile("bar.sync 1, %0;" ::"r"(nthreads) : "memory"); }

// One slice of a sweep read straight from global memory (a slice wider than a stage).
template <typename P>
__device__ __noinline__ void trsv_slice_direct(const SysDev<P> &S, int j, bool lower, int which) {
  TrsvSlice<P, true> a;
  a.load_slice(S, j, lower, which);
  a.finish();
}

constexpr int kTaskThreads = 32 * (kTaskConsumers + 1);     // + one warp that issues the bulk copies
constexpr int kStages = 3;                                  // chunks of 64 KB in flight per CTA (6 of 32 KB: 3.5 % slower)
// gathers of a row issued together: 4 with FP32 factor values (5 or more spill at 64 registers, and
// 8 measured 13 % slower on the 2D bar), 8 with FP64 ones (3 % faster than 4)
template <typename P>
__host__ __device__ constexpr int task_gathers() { return sizeof(P) == 4 ? 4 : 8; }
constexpr int kTaskSmem = kStages * kTaskStageBytes;

// Row sum of one slice row from a stage: sum_k val[32 k] * src[col[32 k]] in index order with
// FP64 FMAs, task_gathers<P>() gathers in flight; the values are read from shared memory as they
// are multiplied (loading them into registers first measured 3.5x slower).
template <typename P>
__device__ __forceinline__ double task_row_sum(const double *src, const int32_t *cj, const P *vj, int width) {
  constexpr int G = task_gathers<P>();
  double sum = 0.0;
  for (int k = 0; k < width; k += G) {
    double xx[G];
#pragma unroll
    for (int u = 0; u < G; ++u) xx[u] = k + u < width ? __ldcg(src + cj[32 * (k + u)]) : 0.0;
#pragma unroll
    for (int u = 0; u < G; ++u)
      if (k + u < width) sum = fma((double)vj[32 * (k + u)], xx[u], sum);
  }
  return sum;
}

// The incomplete-LU apply of one task (a preconditioner block, or a whole system) on one CTA:
// out = U^{-1} L^{-1} in over the task's SELL-32 slices, level after level, a CTA barrier
// between levels instead of a grid barrier.  Everything a slice needs except the solved values
// it gathers -- its descriptor (slot offset, width, rows), the factor columns and values, and its
// rows' operands (the input vector's entries in the forward sweep; urow and udinv in the
// backward sweep) -- does not depend on the sweep, so one producer thread streams it chunk by
// chunk (the layout of solver_kernels.cuh) into a ring of kStages shared-memory stages with bulk
// copies, chunks of later levels in flight while the consumer warps work on the current one.
// A consumer then reads global memory only for the gathers of solved values and, in the
// backward sweep, its row's forward result.
// Slice j of a chunk is summed by consumer warp (rot + j - s0) mod kTaskConsumers, one row per
// lane, in index order with FP64 FMAs: the same arithmetic as k_trsv_persistent, so both give
// bitwise the same results.  The gathers of solved values (written by other warps of this CTA
// before the last CTA barrier) read through L2.  Grid = one CTA per task, tasks ordered by
// decreasing work, so the CTAs that start late take the smallest tasks.  Every wait is bounded
// (bar[2..3] polls); after a failed wait a consumer stops reading the stages but keeps arriving
// on the barriers and taking the level barriers (their sequence comes from the chunk flags in
// global memory, never from a stage), and the producer stops issuing and drains its copies in
// flight.
template <typename P>
__global__ void __launch_bounds__(kTaskThreads, 1) k_trsv_task(const SysDev<P> *sys, const BiState *st, const int32_t *active,
                                                                const TaskDev *tasks, const ChunkDev *chunks,
                                                                const SliceDesc *sdesc, int which, const unsigned *bar,
                                                                int32_t *err) {
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ __align__(8) uint64_t full[kStages], empty[kStages];
  __shared__ int4 smeta[kStages][2];  // per stage: (s0, s1, rot, r0), (values, rows, udinv byte offsets, flags)
  const TaskDev T = tasks[blockIdx.x];
  const int s = T.sys;
  if (!active[s] || st[s].done || (which == 1 && st[s].s_conv)) return;
  const SysDev<P> &S = sys[s];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    for (int i = 0; i < kStages; ++i) { mbar_init(&full[i], 1); mbar_init(&empty[i], kTaskConsumers); }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  const int nL = T.cL1 - T.cL0, nch = nL + (T.cU1 - T.cU0);
  const unsigned long long spin_limit = spin_limit_of(bar);
  const double *in = which == 0 ? S.p : S.s;

  if (warp == kTaskConsumers) {
    // producer: one thread issues the chunks in sweep order, each into the stage its
    // predecessor kStages chunks back has released
    if (lane != 0) return;
    int issued = 0;
    for (int g = 0; g < nch; ++g) {
      const bool lower = g < nL;
      const ChunkDev c = chunks[lower ? T.cL0 + g : T.cU0 + (g - nL)];
      const int stg = g % kStages, round = g / kStages;
      if (round > 0 && !mbar_wait(&empty[stg], (round - 1) & 1, spin_limit, err)) break;
      if (*((volatile int32_t *)err) != 0) break;  // after a failed wait the stages may hold copies in flight
      const unsigned ns = (unsigned)(c.s1 - c.s0), nslot = (unsigned)c.nslot, nrow = (unsigned)(c.r1 - c.r0);
      const unsigned offA = 16u * ns, offB = offA + 4u * nslot, offC = offB + (unsigned)sizeof(P) * nslot, offD = offC + 4u * nrow;
      smeta[stg][0] = make_int4(c.s0, c.s1, c.rot, c.r0);
      smeta[stg][1] = make_int4((int)offB, (int)offC, (int)offD, c.flags);
      if (c.flags & kChunkDirect) { mbar_arrive(&full[stg]); issued = g + 1; continue; }
      unsigned char *base = smem + stg * kTaskStageBytes;
      mbar_arrive_expect_tx(&full[stg], offC + nrow * (lower ? 8u : 4u + (unsigned)sizeof(P)));
      bulk_g2s(base, sdesc + c.d0, offA, &full[stg]);
      if (nslot) {
        bulk_g2s(base + offA, (lower ? S.lcol : S.ucol) + c.o0, 4u * nslot, &full[stg]);
        bulk_g2s(base + offB, (lower ? S.lval : S.uval) + c.o0, (unsigned)sizeof(P) * nslot, &full[stg]);
      }
      if (lower) {
        bulk_g2s(base + offC, in + c.r0, 8u * nrow, &full[stg]);
      } else {
        bulk_g2s(base + offC, S.urow + c.r0, 4u * nrow, &full[stg]);
        bulk_g2s(base + offD, S.udinv + c.r0, (unsigned)sizeof(P) * nrow, &full[stg]);
      }
      issued = g + 1;
    }
    // leave only once this thread's copies have landed: every chunk before the last kStages
    // issued had its stage released before the next copy into it, so only these can be in
    // flight (a fixed bound, independent of the error word and of the caller's poll limit)
    for (int g = issued > kStages ? issued - kStages : 0; g < issued; ++g) mbar_drain(&full[g % kStages], (g / kStages) & 1);
    return;
  }

  // consumers
  double *out = which == 0 ? S.ph : S.sh;
  double *ytmp = S.ytmp;
  bool ok = true;
  for (int g = 0; g < nch; ++g) {
    const bool lower = g < nL;
    const int stg = g % kStages;
    if (ok && !mbar_wait(&full[stg], (g / kStages) & 1, spin_limit, err)) ok = false;
    // the chunk's flags: from its stage, or from global memory once a wait has failed (the stage
    // may then be stale, and every consumer warp must take the same level barriers)
    int32_t flags;
    if (ok) {
      const int4 m0 = smeta[stg][0], m1 = smeta[stg][1];
      flags = m1.w;
      const int s0 = m0.x, s1 = m0.y;
      int j = s0 + (warp - m0.z + kTaskConsumers) % kTaskConsumers;
      if (flags & kChunkDirect) {
        for (; j < s1; j += kTaskConsumers) trsv_slice_direct<P>(S, j, lower, which);
      } else {
        const unsigned char *stage = smem + stg * kTaskStageBytes;
        const int4 *sd = (const int4 *)stage;
        const int32_t *scol = (const int32_t *)(stage + 16 * (s1 - s0));
        const P *sval = (const P *)(stage + m1.x);
        if (lower) {
          const double *sin = (const double *)(stage + m1.y);
          for (; j < s1; j += kTaskConsumers) {
            const int4 d = sd[j - s0];
            const int row = d.z + lane;
            const double base = lane < d.w ? sin[row - m0.w] : 0.0;
            const double sum = task_row_sum<P>(ytmp, scol + d.x + lane, sval + d.x + lane, d.y);
            if (lane < d.w) ytmp[row] = base - sum;
          }
        } else {
          const int32_t *surow = (const int32_t *)(stage + m1.y);
          const P *sdinv = (const P *)(stage + m1.z);
          for (; j < s1; j += kTaskConsumers) {
            const int4 d = sd[j - s0];
            int32_t row = 0;
            double base = 0.0, dinv = 1.0;
            if (lane < d.w) {
              const int t = d.z + lane - m0.w;
              row = surow[t];
              dinv = (double)sdinv[t];
              base = __ldcg(ytmp + row);
            }
            const double sum = task_row_sum<P>(out, scol + d.x + lane, sval + d.x + lane, d.y);
            if (lane < d.w) out[row] = (base - sum) * dinv;
          }
        }
      }
    } else {
      flags = chunks[lower ? T.cL0 + g : T.cU0 + (g - nL)].flags;
    }
    __syncwarp();
    if (lane == 0) mbar_arrive(&empty[stg]);
    if (flags & kChunkLevelEnd) consumers_sync(32 * kTaskConsumers);
  }
}

// ------------------------------------------------- per-task sweeps on thread-block clusters
// The incomplete-LU apply of one task (a preconditioner block, or a whole system) on one
// thread-block cluster of K CTAs: the cluster's warps take the slices of a level in turn (one
// slice per warp, one row per lane, the arithmetic of k_trsv_persistent, so both give bitwise
// the same results) and a cluster barrier (barrier.cluster, release / acquire at cluster scope)
// closes each level instead of a grid barrier.  Clusters are independent: tasks need no
// co-residency, and tasks ordered by decreasing work put the smallest last.  A warp loads its
// first slice of the next level (factor entries and the row's own operand, which do not depend
// on the sweep) before the barrier that closes the current level; only the gathers of solved
// values wait for it.  Solved values written by other CTAs of the cluster are read through L2.
template <typename P>
__global__ void __launch_bounds__(kThreads, 4) k_trsv_cluster(const SysDev<P> *sys, const BiState *st, const int32_t *active,
                                                          const ClusterTask *tasks, const int64_t *lv, int which) {
  namespace cg = cooperative_groups;
  cg::cluster_group cl = cg::this_cluster();
  const int nb = (int)cl.num_blocks();
  const ClusterTask T = tasks[blockIdx.x / nb];
  const int s = T.sys;
  if (!active[s] || st[s].done || (which == 1 && st[s].s_conv)) return;  // uniform over the cluster
  const SysDev<P> &S = sys[s];
  const int w = (int)cl.block_rank() * kWarps + (threadIdx.x >> 5), nw = nb * kWarps;
  for (int pass = 0; pass < 2; ++pass) {
    const bool lower = pass == 0;
    const int nlev = lower ? T.nlevL : T.nlevU;
    const int64_t *lvp = lv + (lower ? T.offL : T.offU);
    TrsvSlice<P, true> cur;
    if (nlev > 0 && lvp[0] + w < lvp[1]) cur.load_slice(S, (int)(lvp[0] + w), lower, which);
    for (int k = 0; k < nlev; ++k) {
      const int64_t j0 = lvp[2 * k], j1 = lvp[2 * k + 1];
      TrsvSlice<P, true> nxt;
      if (k + 1 < nlev && lvp[2 * k + 2] + w < lvp[2 * k + 3]) nxt.load_slice(S, (int)(lvp[2 * k + 2] + w), lower, which);
      cur.finish();
      for (int64_t j = j0 + w + nw; j < j1; j += nw) {
        TrsvSlice<P, true> extra;
        extra.load_slice(S, (int)j, lower, which);
        extra.finish();
      }
      cl.sync();
      cur = nxt;
    }
  }
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

// Keeps the pkeep largest |entries| of lu[lo, hi) (ties: the lower column wins), zeroing the
// others; one warp, entries already zero stay zero and do not count.  In the order "|value|
// descending, then position ascending" the nonzero entries have the distinct ranks 0 .. cnt-1;
// the entry of rank pkeep-1 (magnitude bits vb at position kb) is the last one kept, and every
// entry after it in that order is zeroed.  Short parts find it by ranking every entry against
// the part; long ones (more than kRankMax entries) bisect the bits of vb (|x| of a double orders
// like its bit pattern with the sign cleared) and then walk the ties in position order.
constexpr int64_t kRankMax = 256;
__device__ __forceinline__ unsigned long long abs_bits(double v) {
  return (unsigned long long)__double_as_longlong(v) & 0x7FFFFFFFFFFFFFFFull;
}
__device__ void keep_largest(double *lu, int64_t lo, int64_t hi, int pkeep) {
  const int lane = threadIdx.x & 31;
  int cnt = 0;
  for (int64_t k = lo + lane; k < hi; k += 32) cnt += __ldcg(&lu[k]) != 0.0 ? 1 : 0;
  cnt = warp_sum(cnt);
  if (cnt <= pkeep) return;
  __syncwarp();
  unsigned long long vb = 0;
  int64_t kb = -1;
  if (pkeep > 0 && hi - lo <= kRankMax) {
    for (int64_t k = lo + lane; k < hi; k += 32) {
      const unsigned long long v = abs_bits(__ldcg(&lu[k]));
      if (v == 0) continue;
      int rank = 0;
      for (int64_t k2 = lo; k2 < hi && rank < pkeep; ++k2) {
        const unsigned long long v2 = abs_bits(__ldcg(&lu[k2]));
        if (v2 > v || (v2 == v && k2 < k)) ++rank;
      }
      if (rank == pkeep - 1) { vb = v; kb = k; }
    }
    const unsigned found = __ballot_sync(0xffffffffu, kb >= 0);
    if (!found) return;
    const int src = __ffs(found) - 1;
    vb = __shfl_sync(0xffffffffu, vb, src);
    kb = __shfl_sync(0xffffffffu, kb, src);
  } else if (pkeep > 0) {
    // vb = the largest bit pattern t with at least pkeep entries >= t
    for (int bit = 62; bit >= 0; --bit) {
      const unsigned long long t = vb | (1ull << bit);
      int c = 0;
      for (int64_t k = lo + lane; k < hi; k += 32) c += abs_bits(__ldcg(&lu[k])) >= t ? 1 : 0;
      if (warp_sum(c) >= pkeep) vb = t;
    }
    // the entries equal to vb that stay: pkeep minus those above vb, the lowest positions first
    int above = 0;
    for (int64_t k = lo + lane; k < hi; k += 32) above += abs_bits(__ldcg(&lu[k])) > vb ? 1 : 0;
    int need = pkeep - warp_sum(above);
    for (int64_t k0 = lo; k0 < hi && kb < 0; k0 += 32) {
      const int64_t k = k0 + lane;
      const bool tie = k < hi && abs_bits(__ldcg(&lu[k])) == vb;
      const unsigned m = __ballot_sync(0xffffffffu, tie);
      const int before = __popc(m & ((1u << lane) - 1u));
      const unsigned hit = __ballot_sync(0xffffffffu, tie && before == need - 1);
      if (hit) kb = k0 + (__ffs(hit) - 1);
      else need -= __popc(m);
    }
    if (kb < 0) return;
  }
  __syncwarp();
  for (int64_t k = lo + lane; k < hi; k += 32) {
    const unsigned long long v = abs_bits(__ldcg(&lu[k]));
    if (kb < 0 || v < vb || (v == vb && k > kb)) lu[k] = 0.0;
  }
  __syncwarp();
}

// One row of the IKJ elimination (ILU(0) / ILU(k), no dropping) on a group of kRowLanes lanes,
// with the row's columns and values held in the group's shared-memory row cache: the same
// operations in the same order as the general path below, with the searches and updates of row
// i in shared memory instead of global memory.  Rows of earlier levels (the pivots and the U
// parts) are read from global memory, where they are final.  A warp works on 32 / kRowLanes rows
// at once (the U part of a pivot row is rarely wider than 8 entries).
constexpr int kRowCache = 64;
constexpr int kRowLanes = 8;
constexpr int kRowGroups = kWarps * (32 / kRowLanes);
__device__ __forceinline__ void ilu_row_cached(const FactDev &F, int64_t a, int64_t b, int64_t d, int32_t bi, int32_t *scol,
                                               double *sval, unsigned mask, int32_t *err) {
  const int g = threadIdx.x & (kRowLanes - 1);
  const int w = (int)(b - a);
  for (int k = g; k < w; k += kRowLanes) { scol[k] = F.ci[a + k]; sval[k] = __ldcg(&F.lu[a + k]); }
  __syncwarp(mask);
  for (int64_t kp = a; kp < d; ++kp) {
    const int q = (int)(kp - a);
    const int32_t c = scol[q];
    if (F.blk[c] != bi) continue;
    const double piv = __ldcg(&F.lu[F.diag[c]]);
    if (piv == 0.0) {
      if (g == 0) atomicExch(err, VSHE_E_ZERO_PIVOT_DEV);
      break;
    }
    const double l = sval[q] / piv;
    __syncwarp(mask);
    if (g == 0) sval[q] = l;
    for (int64_t kk = F.diag[c] + 1 + g; kk < F.rp[c + 1]; kk += kRowLanes) {
      const int32_t j = F.ci[kk];
      if (F.blk[j] != bi) continue;
      int lo = q + 1, hi = w - 1, pos = -1;
      while (lo <= hi) {
        const int mid = (lo + hi) >> 1;
        const int32_t cm = scol[mid];
        if (cm == j) { pos = mid; break; }
        if (cm < j) lo = mid + 1; else hi = mid - 1;
      }
      if (pos >= 0) sval[pos] = sval[pos] - l * __ldcg(&F.lu[kk]);
    }
    __syncwarp(mask);
  }
  for (int k = g; k < w; k += kRowLanes) F.lu[a + k] = sval[k];
  __syncwarp(mask);
}

// level entries are solver rows ent_row[e] of system ent_sys[e] (row e of system 0 when NULL).
// ILU(0) / ILU(k) / ILU on a pattern: Saad's IKJ elimination inside the row's pattern.  With
// F.ilut the two ILUT dropping rules (Saad Alg. 10.6) are applied on the way: multipliers below
// tau ||a_i|| are dropped before they eliminate, and after the row is reduced its entries below
// tau ||a_i|| are dropped and only the pkeep largest of L and of U stay; a zero pivot is replaced
// by tau ||a_i|| (or 1), as ILUT does.
__device__ void ilu0_level_rows(const FactDev *fs, Levels lv, int k, int32_t *err) {
  __shared__ int32_t s_col[kRowGroups][kRowCache];
  __shared__ double s_val[kRowGroups][kRowCache];
  const int lane = threadIdx.x & 31;
  const int64_t gid = ((int64_t)blockIdx.x * kThreads + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * kThreads) >> 5;
  const int64_t e0 = lv.lvl_ptr[k], e1 = lv.lvl_ptr[k + 1];
  // pass 1: rows without dropping that fit the row cache, one lane group each
  {
    const int grp = threadIdx.x / kRowLanes;
    const unsigned mask = ((1u << kRowLanes) - 1u) << (lane & ~(kRowLanes - 1));
    const int64_t gg = (int64_t)blockIdx.x * kRowGroups + grp, ng = (int64_t)gridDim.x * kRowGroups;
    for (int64_t e = e0 + gg; e < e1; e += ng) {
      const FactDev &F = fs[lv.ent_sys ? lv.ent_sys[e] : 0];
      const int64_t i = lv.ent_row ? lv.ent_row[e] : e;
      const int64_t a = F.rp[i], b = F.rp[i + 1];
      if (F.ilut || b - a > kRowCache) continue;
      ilu_row_cached(F, a, b, F.diag[i], F.blk[i], s_col[grp], s_val[grp], mask, err);
    }
  }
  __syncwarp();
  // pass 2: the other rows (ILUT, or longer than the cache), one warp each
  for (int64_t e = e0 + gid; e < e1; e += nw) {
    const int s = lv.ent_sys ? lv.ent_sys[e] : 0;
    const FactDev F = fs[s];
    const int64_t i = lv.ent_row ? lv.ent_row[e] : e;
    const int64_t a = F.rp[i], b = F.rp[i + 1], d = F.diag[i];
    const int32_t bi = F.blk[i];
    if (!F.ilut && b - a <= kRowCache) continue;  // done in pass 1
    double ti = 0.0;
    if (F.ilut) {
      double ss = 0.0;
      for (int64_t kk = a + lane; kk < b; kk += 32) { const double v = __ldcg(&F.lu[kk]); ss += v * v; }
      ss = warp_sum(ss);
      ti = F.tau * sqrt(ss);
    }
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
      if (F.ilut && fabs(l) < ti) {  // dropped multiplier: no elimination with row c
        if (lane == 0) F.lu[kp] = 0.0;
        __syncwarp();
        continue;
      }
      if (lane == 0) F.lu[kp] = l;
      for (int64_t kk = F.diag[c] + 1 + lane; kk < F.rp[c + 1]; kk += 32) {
        const int32_t j = F.ci[kk];
        if (F.blk[j] != bi) continue;
        const int64_t pos = find_col(F.ci, kp + 1, b, j);
        if (pos >= 0) F.lu[pos] = __ldcg(&F.lu[pos]) - l * __ldcg(&F.lu[kk]);
      }
      __syncwarp();
    }
    if (F.ilut) {
      for (int64_t kk = a + lane; kk < b; kk += 32)
        if (kk != d && fabs(__ldcg(&F.lu[kk])) < ti) F.lu[kk] = 0.0;
      __syncwarp();
      keep_largest(F.lu, a, d, F.pkeep);
      keep_largest(F.lu, d + 1, b, F.pkeep);
      if (lane == 0 && __ldcg(&F.lu[d]) == 0.0) F.lu[d] = ti > 0.0 ? ti : 1.0;
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

// solver-order values from A: out[k] = av[amap[k]], 0 where amap[k] < 0 (SELL padding)
__global__ void k_gather_values(int64_t nnz, const int64_t *amap, const double *av, double *out) {
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < nnz; k += (int64_t)gridDim.x * blockDim.x) {
    const int64_t m = amap[k];
    out[k] = m >= 0 ? av[m] : 0.0;
  }
}

// out[q] = in[perm[q]] (gather == 1) or out[perm[q]] = in[q] (gather == 0)
__global__ void k_permute(int64_t n, const int32_t *perm, const double *in, double *out, int gather) {
  for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (int64_t)gridDim.x * blockDim.x) {
    if (gather) out[q] = in[perm[q]];
    else out[perm[q]] = in[q];
  }
}

// Split the solver-order factor (FP64 CSR) into the SELL-32 slices of L and U and the inverse
// diagonal, in precision P: fmap[k] >= 0 -> L slot, <= -2 -> U slot -(fmap+2), -1 -> not part
// of the factor; dpos[row] is the backward-sweep slot of the row.  Padding slots stay 0.
template <typename P>
__global__ void k_split_factor(int64_t nnz, int64_t n, const double *lu, const int64_t *fmap, const int64_t *diag, const int64_t *dpos,
                               P *lval, P *uval, P *udinv) {
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < nnz; k += (int64_t)gridDim.x * blockDim.x) {
    const int64_t m = fmap[k];
    if (m >= 0) lval[m] = (P)lu[k];
    else if (m <= -2) uval[-(m + 2)] = (P)lu[k];
  }
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    udinv[dpos[i]] = (P)(1.0 / lu[diag[i]]);
}

// ------------------------------------------------------- FP64 residual
// r = b - A x (FP64, solver order), ||r||^2 and ||b||^2 per system -> rnorm2 / bnorm2.
__device__ __forceinline__ void k_residual64_tile(const RefDev *sys, const Tiles &tl, double *partials, int32_t *counters, const int32_t *active, double *rnorm2, double *bnorm2, int tile) {
  const int s = tl.tile_sys[tile];
  if (!active[s]) return;
  const RefDev &S = sys[s];
  const int64_t *__restrict__ aoff = S.aoff;
  const int32_t *__restrict__ acol = S.acol;
  const double *__restrict__ aval = S.aval;
  const double *xv = S.x, *bv = S.b;
  double *rv = S.r;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int64_t r0 = tl.tile_row0[tile], r1 = tl.tile_row1[tile];
  double acc[2] = {0.0, 0.0};
  for (int64_t q0 = r0 + 32 * w; q0 < r1; q0 += 32 * kWarps) {
    const int64_t j = q0 >> 5, off = aoff[j];
    const double ax = sell_rowsum<double, false, kDotU>(off, (int)((aoff[j + 1] - off) >> 5), acol, aval, xv);
    const int64_t row = q0 + lane;
    if (row < r1) {
      const double bb = bv[row];
      const double r = bb - ax;
      rv[row] = r;
      acc[0] += r * r;
      acc[1] += bb * bb;
    }
  }
  double tot[2];
  if (tile_finish<2>(acc, tile, s, tl, partials, counters, tot)) {
    rnorm2[s] = tot[0];
    bnorm2[s] = tot[1];
  }
}
__global__ void __launch_bounds__(kThreads, 4) k_residual64(const RefDev *sys, Tiles tl, double *partials, int32_t *counters, const int32_t *active, double *rnorm2, double *bnorm2) {
  k_residual64_tile(sys, tl, partials, counters, active, rnorm2, bnorm2, blockIdx.x);
}

// plain SELL-32 SpMV for tests / timing (y = A x, solver order): one slice per warp in turn
__global__ void __launch_bounds__(kThreads, 4) k_spmv_plain(int64_t n, const int64_t *aoff, const int32_t *acol, const double *aval, const double *x, double *y) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int64_t gw = (int64_t)blockIdx.x * kWarps + w, nw = (int64_t)gridDim.x * kWarps;
  for (int64_t j = gw; 32 * j < n; j += nw) {
    const int64_t off = aoff[j];
    const double v = sell_rowsum<double, false, kSpmvU>(off, (int)((aoff[j + 1] - off) >> 5), acol, aval, x);
    if (32 * j + lane < n) y[32 * j + lane] = v;
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

// CTAs of the tile kernels: one per tile.  (Persistent CTAs looping over the tiles measured 10%
// slower on the 2D bar: a CTA's per-tile reduction tail then stalls its next tile, where
// separate CTAs overlap it with other CTAs' work.)
static int tile_grid(int ntiles) { return ntiles; }

template <typename P>
static int launch_trsv_t(int mode, int grid, const SysDev<P> *sys, const BiState *st, const int32_t *act, Levels lL, Levels lU, int which, unsigned *bar, int32_t *err, cudaStream_t s) {
  if (mode == 1 || mode == 3) {
    g_launches += 1;
    void *args[] = {(void *)&sys, (void *)&st, (void *)&act, (void *)&lL, (void *)&lU, (void *)&which, (void *)&bar, (void *)&err};
    return (int)cudaLaunchCooperativeKernel(mode == 1 ? (void *)k_trsv_persistent<P> : (void *)k_trsv_flow<P>, dim3(grid), dim3(kThreads),
                                            args, 0, s);
  }
  g_launches += lL.nlev + lU.nlev;
  for (int pass = 0; pass < 2; ++pass) {
    const Levels &lv = pass == 0 ? lL : lU;
    for (int k = 0; k < lv.nlev; ++k) k_trsv_level<P><<<grid, kThreads, 0, s>>>(sys, st, act, lv, k, 1 - pass, which);
  }
  return (int)cudaGetLastError();
}

extern "C" {

int vk_threads() { return kThreads; }
void vk_count_launches(long long k) { g_launches += k; }
long long vk_launches_total() { return g_launches.load(); }

void vk_bicg_init(int ntiles, const void *sys, void *st, const VkTiles *tl, double *part, int32_t *cnt, const int32_t *act, cudaStream_t s) {
  g_launches += 1;
  k_bicg_init<<<tile_grid(ntiles), kThreads, 0, s>>>((const SysK *)sys, (BiState *)st, *(const Tiles *)tl, part, cnt, act);
}
void vk_bicg_resume(int ntiles, const void *sys, void *st, const VkTiles *tl, double *part, int32_t *cnt, const int32_t *act, cudaStream_t s) {
  g_launches += 1;
  k_bicg_resume<<<tile_grid(ntiles), kThreads, 0, s>>>((const SysK *)sys, (BiState *)st, *(const Tiles *)tl, part, cnt, act);
}
void vk_update_p(int ntiles, const void *sys, void *st, const VkTiles *tl, const int32_t *act, cudaStream_t s) {
  g_launches += 1;
  k_update_p<<<tile_grid(ntiles), kThreads, 0, s>>>((const SysK *)sys, (BiState *)st, *(const Tiles *)tl, act);
}
void vk_spmv_dot(int ntiles, const void *sys, void *st, const VkTiles *tl, double *part, int32_t *cnt, const int32_t *act, int which, cudaStream_t s) {
  g_launches += 1;
  k_spmv_dot<<<tile_grid(ntiles), kThreads, 0, s>>>((const SysK *)sys, (BiState *)st, *(const Tiles *)tl, part, cnt, act, which);
}
void vk_update_s(int ntiles, const void *sys, void *st, const VkTiles *tl, double *part, int32_t *cnt, const int32_t *act, cudaStream_t s) {
  g_launches += 1;
  k_update_s<<<tile_grid(ntiles), kThreads, 0, s>>>((const SysK *)sys, (BiState *)st, *(const Tiles *)tl, part, cnt, act);
}
void vk_update_xr(int ntiles, const void *sys, void *st, const VkTiles *tl, double *part, int32_t *cnt, const int32_t *act, cudaStream_t s) {
  g_launches += 1;
  k_update_xr<<<tile_grid(ntiles), kThreads, 0, s>>>((const SysK *)sys, (BiState *)st, *(const Tiles *)tl, part, cnt, act);
}
void vk_precond_copy(int ntiles, const void *sys, const void *st, const VkTiles *tl, const int32_t *act, int which, cudaStream_t s) {
  g_launches += 1;
  k_precond_copy<<<tile_grid(ntiles), kThreads, 0, s>>>((const SysK *)sys, (const BiState *)st, *(const Tiles *)tl, act, which);
}

#define VK_BODY_P(P, SUF)                                                                                             \
  int vk_trsv_task_##SUF(int ntasks, const void *sys, const void *st, const int32_t *act, const void *tasks,          \
                         const void *chunks, const void *sdesc, int which, const unsigned *bar, int32_t *err,      \
                         cudaStream_t s) {                                                                          \
    static bool attr = false;                                                                                        \
    if (!attr) {                                                                                                     \
      cudaError_t e = cudaFuncSetAttribute((const void *)k_trsv_task<P>, cudaFuncAttributeMaxDynamicSharedMemorySize, \
                                           kTaskSmem);                                                               \
      if (e != cudaSuccess) return (int)e;                                                                           \
      attr = true;                                                                                                   \
    }                                                                                                                \
    g_launches += 1;                                                                                                 \
    k_trsv_task<P><<<ntasks, kTaskThreads, kTaskSmem, s>>>((const SysDev<P> *)sys, (const BiState *)st, act,         \
                                                           (const TaskDev *)tasks, (const ChunkDev *)chunks,          \
                                                           (const SliceDesc *)sdesc, which, bar, err);                \
    return (int)cudaGetLastError();                                                                                  \
  }                                                                                                                  \
  int vk_trsv_cluster_##SUF(int ntasks, int csize, const void *sys, const void *st, const int32_t *act, const void *tasks, \
                            const int64_t *lv, int which, cudaStream_t s) {                                          \
    cudaLaunchConfig_t cfg = {};                                                                                     \
    cudaLaunchAttribute at[1];                                                                                       \
    at[0].id = cudaLaunchAttributeClusterDimension;                                                                  \
    at[0].val.clusterDim.x = (unsigned)csize; at[0].val.clusterDim.y = 1; at[0].val.clusterDim.z = 1;                \
    cfg.gridDim = dim3((unsigned)(ntasks * csize));                                                                  \
    cfg.blockDim = dim3(kThreads);                                                                                   \
    cfg.dynamicSmemBytes = 0;                                                                                        \
    cfg.stream = s;                                                                                                  \
    cfg.attrs = at;                                                                                                  \
    cfg.numAttrs = 1;                                                                                                \
    g_launches += 1;                                                                                                 \
    return (int)cudaLaunchKernelEx(&cfg, k_trsv_cluster<P>, (const SysDev<P> *)sys, (const BiState *)st, act,        \
                                   (const ClusterTask *)tasks, lv, which);                                           \
  }                                                                                                                  \
  int vk_trsv_##SUF(int mode, int grid, const void *sys, const void *st, const int32_t *act, const VkLevels *lL,     \
                    const VkLevels *lU, int which, unsigned *bar, int32_t *err, cudaStream_t s) {                    \
    return launch_trsv_t<P>(mode, grid, (const SysDev<P> *)sys, (const BiState *)st, act, *(const Levels *)lL,       \
                            *(const Levels *)lU, which, bar, err, s);                                                \
  }                                                                                                                  \
  int vk_trsv_occupancy_##SUF(int *blocks_per_sm) {                                                                  \
    int b1 = 0, b2 = 0;                                                                                              \
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b1, (void *)k_trsv_persistent<P>, kThreads, 0);   \
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b2, (void *)k_trsv_flow<P>, kThreads, 0); \
    *blocks_per_sm = b1 < b2 ? b1 : b2;                                                                              \
    return (int)e;                                                                                                   \
  }                                                                                                                  \
  void vk_split_factor_##SUF(int64_t nnz, int64_t n, const double *lu, const int64_t *fmap, const int64_t *diag,     \
                             const int64_t *dpos, P *lval, P *uval, P *udinv, cudaStream_t s) {                      \
    g_launches += 1;                                                                                                 \
    k_split_factor<P><<<grid_for(nnz > n ? nnz : n), kThreads, 0, s>>>(nnz, n, lu, fmap, diag, dpos, lval, uval, udinv); \
  }

VK_BODY_P(float, f32)
VK_BODY_P(double, f64)

void vk_spmv_plain(int grid, int64_t n, const int64_t *aoff, const int32_t *acol, const double *aval, const double *x, double *y, cudaStream_t s) {
  g_launches += 1;
  k_spmv_plain<<<grid, kThreads, 0, s>>>(n, aoff, acol, aval, x, y);
}

void vk_permute(int64_t n, const int32_t *perm, const double *in, double *out, int gather, cudaStream_t s) {
  g_launches += 1;
  k_permute<<<grid_for(n), kThreads, 0, s>>>(n, perm, in, out, gather);
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

void vk_gather_values(int64_t nnz, const int64_t *amap, const double *av, double *out, cudaStream_t s) {
  g_launches += 1;
  k_gather_values<<<grid_for(nnz), kThreads, 0, s>>>(nnz, amap, av, out);
}

size_t vk_factdev_size() { return sizeof(FactDev); }
size_t vk_refdev_size() { return sizeof(RefDev); }
size_t vk_sysdev_size() { return sizeof(SysDev<double>); }
size_t vk_bistate_size() { return sizeof(BiState); }

void vk_residual64(int ntiles, const void *ref, const VkTiles *tl, double *part, int32_t *cnt, const int32_t *act,
                   double *rnorm2, double *bnorm2, cudaStream_t s) {
  g_launches += 1;
  k_residual64<<<tile_grid(ntiles), kThreads, 0, s>>>((const RefDev *)ref, *(const Tiles *)tl, part, cnt, act, rnorm2, bnorm2);
}

}  // extern "C"

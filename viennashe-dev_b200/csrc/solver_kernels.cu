// solver_kernels.cu -- sm_100a kernels of the Krylov solver (thin launchers at the end).
//
// Everything here is memory-bound sparse work: CSR SpMV with sub-warp row
// groups and fused dot products, BiCGStab vector updates fused with their
// reductions, level-scheduled ILU(0) factorisation and triangular solves run
// as persistent cooperative kernels with a bounded grid barrier per level,
// and the FP64 refinement residual.  No tensor cores: nothing on this path is
// a dense contraction.
//
// Batches: each kernel works on a batch of independent systems described by
// per-system pointer tables (SysDev) and row tiles that never straddle two
// systems; reductions are per tile and are finished by the last tile of each
// system, in a fixed order, so a system's iterates do not depend on what else
// is in the batch.

#include <cuda_runtime.h>
#include <cooperative_groups.h>
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

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

template <typename T, int G>
__device__ __forceinline__ T group_sum(T v) {
#pragma unroll
  for (int o = G / 2; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Block-wide sum of up to 3 values; result valid in thread 0.
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
  // last block: deterministic fixed-shape reduction over the system's tiles
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

template <typename T>
__device__ __forceinline__ T dsqrt(T x);
template <>
__device__ __forceinline__ float dsqrt<float>(float x) { return sqrtf(x); }
template <>
__device__ __forceinline__ double dsqrt<double>(double x) { return sqrt(x); }

// ------------------------------------------------------------------ BiCGStab
// init: rh = r (= b of this solve), x = p = v = 0; ||b|| -> state
template <typename T>
__global__ void __launch_bounds__(kThreads) k_bicg_init(const SysDev<T> *sys, BiState<T> *st, Tiles tl, T *partials, int32_t *counters, const int32_t *active) {
  const int tile = blockIdx.x;
  const int s = tl.tile_sys[tile];
  if (!active[s]) return;
  const SysDev<T> S = sys[s];
  T acc[1] = {T(0)};
  for (int64_t i = tl.tile_row0[tile] + threadIdx.x; i < tl.tile_row1[tile]; i += kThreads) {
    T r = S.r[i];
    S.rh[i] = r;
    S.x[i] = T(0); S.p[i] = T(0); S.v[i] = T(0);
    acc[0] += r * r;
  }
  T tot[1];
  if (tile_finish<T, 1>(acc, tile, s, tl, partials, counters, tot)) {
    BiState<T> &b = st[s];
    b.bnorm = dsqrt(tot[0]);
    b.rho = tot[0]; b.rho_old = T(1); b.alpha = T(1); b.omega = T(1);
    b.res = T(1); b.iter = 0; b.s_conv = 0; b.status = 0;
    b.done = (tot[0] == T(0)) ? 1 : 0;
    if (b.done) b.res = T(0);
  }
}

// p = r + beta (p - omega v)
template <typename T>
__global__ void __launch_bounds__(kThreads) k_update_p(const SysDev<T> *sys, const BiState<T> *st, Tiles tl, const int32_t *active) {
  const int tile = blockIdx.x;
  const int s = tl.tile_sys[tile];
  if (!active[s] || st[s].done) return;
  const SysDev<T> S = sys[s];
  const BiState<T> b = st[s];
  if (b.iter == 0) {
    for (int64_t i = tl.tile_row0[tile] + threadIdx.x; i < tl.tile_row1[tile]; i += kThreads) S.p[i] = S.r[i];
  } else {
    const T beta = (b.rho / b.rho_old) * (b.alpha / b.omega);
    for (int64_t i = tl.tile_row0[tile] + threadIdx.x; i < tl.tile_row1[tile]; i += kThreads)
      S.p[i] = S.r[i] + beta * (S.p[i] - b.omega * S.v[i]);
  }
}

// y = A x over one tile with G lanes per row; optional dots with y.
// which = 0: v = A ph, dot (rh, v) -> alpha.   which = 1: t = A sh, dots (t, s), (t, t) -> omega.
template <typename T, int G>
__global__ void __launch_bounds__(kThreads) k_spmv_dot(const SysDev<T> *sys, BiState<T> *st, Tiles tl, T *partials, int32_t *counters, const int32_t *active, int which) {
  const int tile = blockIdx.x;
  const int s = tl.tile_sys[tile];
  if (!active[s] || st[s].done) return;
  if (which == 1 && st[s].s_conv) return;
  const SysDev<T> S = sys[s];
  const T *xin = which == 0 ? S.ph : S.sh;
  T *yout = which == 0 ? S.v : S.t;
  const int lane = threadIdx.x % G;
  const int grp = threadIdx.x / G;
  const int wgrp = (threadIdx.x & ~31) / G;  // first group of this warp (loop bound is warp-uniform)
  constexpr int NG = kThreads / G;
  const int64_t r0 = tl.tile_row0[tile], r1 = tl.tile_row1[tile];
  T acc[2] = {T(0), T(0)};
  for (int64_t base = r0 + wgrp; base < r1; base += NG) {
    const int64_t row = base + (grp - wgrp);
    const bool valid = row < r1;
    T sum = T(0);
    if (valid) {
      const int64_t a = S.rp[row], e = S.rp[row + 1];
      for (int64_t k = a + lane; k < e; k += G) sum += S.av[k] * xin[S.ci[k]];
    }
    sum = group_sum<T, G>(sum);
    if (valid && lane == 0) {
      yout[row] = sum;
      if (which == 0) acc[0] += S.rh[row] * sum;
      else { acc[0] += sum * S.s[row]; acc[1] += sum * sum; }
    }
  }
  T tot[2];
  if (tile_finish<T, 2>(acc, tile, s, tl, partials, counters, tot)) {
    BiState<T> &b = st[s];
    if (which == 0) {
      if (tot[0] == T(0)) { b.status = VSHE_E_BREAKDOWN_DEV; b.done = 1; }
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

// x += alpha ph + omega sh; r = s - omega t; ||r||, (rh, r) -> next rho, convergence
template <typename T>
__global__ void __launch_bounds__(kThreads) k_update_xr(const SysDev<T> *sys, BiState<T> *st, Tiles tl, T *partials, int32_t *counters, const int32_t *active) {
  const int tile = blockIdx.x;
  const int s = tl.tile_sys[tile];
  if (!active[s] || st[s].done) return;
  const SysDev<T> S = sys[s];
  const BiState<T> b0 = st[s];
  T acc[2] = {T(0), T(0)};
  if (b0.s_conv) {
    for (int64_t i = tl.tile_row0[tile] + threadIdx.x; i < tl.tile_row1[tile]; i += kThreads) S.x[i] += b0.alpha * S.ph[i];
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
    if (b.s_conv) { b.done = 1; return; }
    b.res = dsqrt(tot[0]) / b.bnorm;
    b.rho_old = b.rho;
    b.rho = tot[1];
    if (b.res < b.tol) { b.done = 1; return; }
    if (b.rho == T(0) || b.omega == T(0)) { b.done = 1; b.status = VSHE_E_BREAKDOWN_DEV; return; }
    if (b.iter >= b.max_iter) { b.done = 1; b.status = VSHE_E_NOT_CONVERGED_DEV; }
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
// Sense-free generation barrier for a cooperative launch (all CTAs resident).
// The spin is bounded: after `limit` polls the kernel records a timeout and
// every CTA leaves; the host sees the error flag.
__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned *p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release_u32(unsigned *p, unsigned v) {
  asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

__device__ bool grid_barrier(unsigned *bar, int32_t *err) {
  // bar[0] = arrival count, bar[1] = generation
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
        if (spins > 64) __nanosleep(64);
      }
    }
    if (ok && *((volatile int32_t *)err) != 0) ok = 0;
  }
  __syncthreads();
  return ok != 0;
}

// ------------------------------------------------- triangular solves (ILU apply)
// out = U^{-1} L^{-1} in, level by level.  which 0: ph = M^{-1} p, 1: sh = M^{-1} s.
template <typename T, int G>
__device__ __forceinline__ void trsv_level_rows(const SysDev<T> *sys, const BiState<T> *st, const int32_t *active, const Levels lv, int k, bool lower, int which) {
  const int lane = threadIdx.x % G;
  const int64_t gid = ((int64_t)blockIdx.x * kThreads + threadIdx.x) / G;
  const int64_t wgid = ((int64_t)blockIdx.x * kThreads + (threadIdx.x & ~31)) / G;  // warp-uniform loop bound
  const int64_t ngrp = ((int64_t)gridDim.x * kThreads) / G;
  const int64_t e0 = lv.lvl_ptr[k], e1 = lv.lvl_ptr[k + 1];
  for (int64_t eb = e0 + wgid; eb < e1; eb += ngrp) {
    const int64_t e = eb + (gid - wgid);
    bool valid = e < e1;
    int s = 0;
    if (valid) {
      s = lv.ent_sys ? lv.ent_sys[e] : 0;
      valid = active[s] && !st[s].done && !(which == 1 && st[s].s_conv);
    }
    const SysDev<T> *S = &sys[s];
    const int64_t row = valid ? (int64_t)lv.ent_row[e] : 0;
    T *out = which == 0 ? S->ph : S->sh;
    T sum = T(0);
    if (lower) {
      if (valid)
        for (int64_t q = S->lrp[row] + lane; q < S->lrp[row + 1]; q += G) sum += S->lv[q] * __ldcg(&out[S->lci[q]]);
      sum = group_sum<T, G>(sum);
      if (valid && lane == 0) {
        const T *in = which == 0 ? S->p : S->s;
        out[row] = in[row] - sum;
      }
    } else {
      if (valid)
        for (int64_t q = S->urp[row] + lane; q < S->urp[row + 1]; q += G) sum += S->uv[q] * __ldcg(&out[S->uci[q]]);
      sum = group_sum<T, G>(sum);
      if (valid && lane == 0) out[row] = (__ldcg(&out[row]) - sum) * S->dinv[row];
    }
  }
}

template <typename T, int G>
__global__ void __launch_bounds__(kThreads) k_trsv_persistent(const SysDev<T> *sys, const BiState<T> *st, const int32_t *active, Levels lL, Levels lU, int which, unsigned *bar, int32_t *err) {
  for (int k = 0; k < lL.nlev; ++k) {
    trsv_level_rows<T, G>(sys, st, active, lL, k, true, which);
    if (!grid_barrier(bar, err)) return;
  }
  for (int k = 0; k < lU.nlev; ++k) {
    trsv_level_rows<T, G>(sys, st, active, lU, k, false, which);
    if (k + 1 < lU.nlev && !grid_barrier(bar, err)) return;
  }
}

template <typename T, int G>
__global__ void __launch_bounds__(kThreads) k_trsv_level(const SysDev<T> *sys, const BiState<T> *st, const int32_t *active, Levels lv, int k, int lower, int which) {
  trsv_level_rows<T, G>(sys, st, active, lv, k, lower != 0, which);
}

// ------------------------------------------------------ ILU(0) factorisation
// Row-wise IKJ ILU(0) (Saad, Alg. 10.4) restricted to within-block entries,
// one warp per row, rows of a level in parallel.  Values in FP64.

__device__ __forceinline__ int64_t find_col(const int32_t *ci, int64_t a, int64_t b, int32_t j) {
  // binary search for column j in ci[a, b)
  int64_t lo = a, hi = b - 1;
  while (lo <= hi) {
    int64_t mid = (lo + hi) >> 1;
    int32_t c = ci[mid];
    if (c == j) return mid;
    if (c < j) lo = mid + 1; else hi = mid - 1;
  }
  return -1;
}

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

// Split the factor (in A's pattern, FP64) into strict L, strict U and 1/diag(U) in precision T.
template <typename T>
__global__ void k_split_factor(int64_t n, const int64_t *rp, const int32_t *ci, const double *lu, const int32_t *blk,
                               const int64_t *lrp, T *lv, const int64_t *urp, T *uv, T *dinv) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    int64_t lp = lrp[i], up = urp[i];
    const int32_t bi = blk[i];
    for (int64_t k = rp[i]; k < rp[i + 1]; ++k) {
      const int32_t j = ci[k];
      if (j == i) { dinv[i] = (T)(1.0 / lu[k]); continue; }
      if (blk[j] != bi) continue;
      if (j < i) lv[lp++] = (T)lu[k];
      else uv[up++] = (T)lu[k];
    }
  }
}

// ------------------------------------------------------- FP64 refinement
// r = b - A x (FP64), ||r||^2 per system -> rnorm[s]; counters/partials as for the Krylov kernels.

template <int G>
__global__ void __launch_bounds__(kThreads) k_residual64(const RefDev *sys, Tiles tl, double *partials, int32_t *counters, const int32_t *active, double *rnorm2, double *bnorm2) {
  const int tile = blockIdx.x;
  const int s = tl.tile_sys[tile];
  if (!active[s]) return;
  const RefDev S = sys[s];
  const int lane = threadIdx.x % G, grp = threadIdx.x / G;
  const int wgrp = (threadIdx.x & ~31) / G;
  constexpr int NG = kThreads / G;
  const int64_t r0 = tl.tile_row0[tile], r1 = tl.tile_row1[tile];
  double acc[2] = {0.0, 0.0};
  for (int64_t base = r0 + wgrp; base < r1; base += NG) {
    const int64_t row = base + (grp - wgrp);
    const bool valid = row < r1;
    double sum = 0.0;
    if (valid)
      for (int64_t k = S.rp[row] + lane; k < S.rp[row + 1]; k += G) sum += S.av[k] * S.x[S.ci[k]];
    sum = group_sum<double, G>(sum);
    if (valid && lane == 0) {
      double bb = S.b[row];
      double r = bb - sum;
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

// inner rhs: r32 = r64 / ||r64||
__global__ void k_scale_to_f32(const RefDev *ref, const SysDev<float> *sys, Tiles tl, const int32_t *active, const double *rnorm2) {
  const int tile = blockIdx.x;
  const int s = tl.tile_sys[tile];
  if (!active[s]) return;
  const double inv = rnorm2[s] > 0.0 ? 1.0 / sqrt(rnorm2[s]) : 0.0;
  const double *r = ref[s].r;
  float *r32 = sys[s].r;
  for (int64_t i = tl.tile_row0[tile] + threadIdx.x; i < tl.tile_row1[tile]; i += blockDim.x) r32[i] = (float)(r[i] * inv);
}

// x64 += ||r64|| * x32
__global__ void k_accumulate_x(const RefDev *ref, const SysDev<float> *sys, Tiles tl, const int32_t *active, const double *rnorm2) {
  const int tile = blockIdx.x;
  const int s = tl.tile_sys[tile];
  if (!active[s]) return;
  const double sc = sqrt(rnorm2[s]);
  double *x = ref[s].x;
  const float *d = sys[s].x;
  for (int64_t i = tl.tile_row0[tile] + threadIdx.x; i < tl.tile_row1[tile]; i += blockDim.x) x[i] += sc * (double)d[i];
}

__global__ void k_cast_f64_f32(int64_t n, const double *a, float *b) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) b[i] = (float)a[i];
}

// plain SpMV for tests / timing (y = A x), G lanes per row
template <typename T, int G>
__global__ void __launch_bounds__(kThreads) k_spmv_plain(int64_t n, const int64_t *rp, const int32_t *ci, const T *av, const T *x, T *y) {
  const int lane = threadIdx.x % G;
  const int64_t grp = ((int64_t)blockIdx.x * kThreads + threadIdx.x) / G;
  const int64_t wgrp = ((int64_t)blockIdx.x * kThreads + (threadIdx.x & ~31)) / G;
  const int64_t ngrp = ((int64_t)gridDim.x * kThreads) / G;
  for (int64_t base = wgrp; base < n; base += ngrp) {
    const int64_t row = base + (grp - wgrp);
    const bool valid = row < n;
    T sum = T(0);
    if (valid)
      for (int64_t k = rp[row] + lane; k < rp[row + 1]; k += G) sum += av[k] * x[ci[k]];
    sum = group_sum<T, G>(sum);
    if (valid && lane == 0) y[row] = sum;
  }
}

}  // namespace vshe

// =====================================================================
// thin launchers (declared in kernels.h)
// =====================================================================
using namespace vshe;

template <typename T, int G>
static void launch_spmv_dot_g(int ntiles, const SysDev<T> *sys, BiState<T> *st, Tiles tl, T *part, int32_t *cnt, const int32_t *act, int which, cudaStream_t s) {
  k_spmv_dot<T, G><<<ntiles, kThreads, 0, s>>>(sys, st, tl, part, cnt, act, which);
}

template <typename T>
static void launch_spmv_dot_t(int group, int ntiles, const SysDev<T> *sys, BiState<T> *st, Tiles tl, T *part, int32_t *cnt, const int32_t *act, int which, cudaStream_t s) {
  switch (group) {
    case 2: launch_spmv_dot_g<T, 2>(ntiles, sys, st, tl, part, cnt, act, which, s); break;
    case 4: launch_spmv_dot_g<T, 4>(ntiles, sys, st, tl, part, cnt, act, which, s); break;
    case 8: launch_spmv_dot_g<T, 8>(ntiles, sys, st, tl, part, cnt, act, which, s); break;
    case 16: launch_spmv_dot_g<T, 16>(ntiles, sys, st, tl, part, cnt, act, which, s); break;
    default: launch_spmv_dot_g<T, 32>(ntiles, sys, st, tl, part, cnt, act, which, s); break;
  }
}

template <typename T>
static int launch_trsv_t(int mode, int group, int grid, const SysDev<T> *sys, const BiState<T> *st, const int32_t *act, Levels lL, Levels lU, int which, unsigned *bar, int32_t *err, cudaStream_t s) {
  if (mode == 1) {
    void *args[] = {(void *)&sys, (void *)&st, (void *)&act, (void *)&lL, (void *)&lU, (void *)&which, (void *)&bar, (void *)&err};
    void *fn;
    switch (group) {
      case 1: fn = (void *)k_trsv_persistent<T, 1>; break;
      case 2: fn = (void *)k_trsv_persistent<T, 2>; break;
      case 4: fn = (void *)k_trsv_persistent<T, 4>; break;
      default: fn = (void *)k_trsv_persistent<T, 8>; break;
    }
    return (int)cudaLaunchCooperativeKernel(fn, dim3(grid), dim3(kThreads), args, 0, s);
  }
  for (int k = 0; k < lL.nlev; ++k) {
    switch (group) {
      case 1: k_trsv_level<T, 1><<<grid, kThreads, 0, s>>>(sys, st, act, lL, k, 1, which); break;
      case 2: k_trsv_level<T, 2><<<grid, kThreads, 0, s>>>(sys, st, act, lL, k, 1, which); break;
      case 4: k_trsv_level<T, 4><<<grid, kThreads, 0, s>>>(sys, st, act, lL, k, 1, which); break;
      default: k_trsv_level<T, 8><<<grid, kThreads, 0, s>>>(sys, st, act, lL, k, 1, which); break;
    }
  }
  for (int k = 0; k < lU.nlev; ++k) {
    switch (group) {
      case 1: k_trsv_level<T, 1><<<grid, kThreads, 0, s>>>(sys, st, act, lU, k, 0, which); break;
      case 2: k_trsv_level<T, 2><<<grid, kThreads, 0, s>>>(sys, st, act, lU, k, 0, which); break;
      case 4: k_trsv_level<T, 4><<<grid, kThreads, 0, s>>>(sys, st, act, lU, k, 0, which); break;
      default: k_trsv_level<T, 8><<<grid, kThreads, 0, s>>>(sys, st, act, lU, k, 0, which); break;
    }
  }
  return (int)cudaGetLastError();
}

template <typename T>
static int occupancy_persistent_t(int group, int *blocks_per_sm) {
  void *fn;
  switch (group) {
    case 1: fn = (void *)k_trsv_persistent<T, 1>; break;
    case 2: fn = (void *)k_trsv_persistent<T, 2>; break;
    case 4: fn = (void *)k_trsv_persistent<T, 4>; break;
    default: fn = (void *)k_trsv_persistent<T, 8>; break;
  }
  return (int)cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, fn, kThreads, 0);
}

extern "C" {

int vk_threads() { return kThreads; }

#define VK_BODY_T(T, SUF)                                                                                             \
  void vk_bicg_init_##SUF(int ntiles, const void *sys, void *st, const VkTiles *tl, T *part, int32_t *cnt,           \
                          const int32_t *act, cudaStream_t s) {                                                      \
    k_bicg_init<T><<<ntiles, kThreads, 0, s>>>((const SysDev<T> *)sys, (BiState<T> *)st, *(const Tiles *)tl, part, cnt, act); \
  }                                                                                                                  \
  void vk_update_p_##SUF(int ntiles, const void *sys, const void *st, const VkTiles *tl, const int32_t *act,        \
                         cudaStream_t s) {                                                                           \
    k_update_p<T><<<ntiles, kThreads, 0, s>>>((const SysDev<T> *)sys, (const BiState<T> *)st, *(const Tiles *)tl, act); \
  }                                                                                                                  \
  void vk_spmv_dot_##SUF(int group, int ntiles, const void *sys, void *st, const VkTiles *tl, T *part, int32_t *cnt, \
                         const int32_t *act, int which, cudaStream_t s) {                                            \
    launch_spmv_dot_t<T>(group, ntiles, (const SysDev<T> *)sys, (BiState<T> *)st, *(const Tiles *)tl, part, cnt, act, which, s); \
  }                                                                                                                  \
  void vk_update_s_##SUF(int ntiles, const void *sys, void *st, const VkTiles *tl, T *part, int32_t *cnt,           \
                         const int32_t *act, cudaStream_t s) {                                                       \
    k_update_s<T><<<ntiles, kThreads, 0, s>>>((const SysDev<T> *)sys, (BiState<T> *)st, *(const Tiles *)tl, part, cnt, act); \
  }                                                                                                                  \
  void vk_update_xr_##SUF(int ntiles, const void *sys, void *st, const VkTiles *tl, T *part, int32_t *cnt,          \
                          const int32_t *act, cudaStream_t s) {                                                      \
    k_update_xr<T><<<ntiles, kThreads, 0, s>>>((const SysDev<T> *)sys, (BiState<T> *)st, *(const Tiles *)tl, part, cnt, act); \
  }                                                                                                                  \
  void vk_precond_copy_##SUF(int ntiles, const void *sys, const void *st, const VkTiles *tl, const int32_t *act,    \
                             int which, cudaStream_t s) {                                                            \
    k_precond_copy<T><<<ntiles, kThreads, 0, s>>>((const SysDev<T> *)sys, (const BiState<T> *)st, *(const Tiles *)tl, act, which); \
  }                                                                                                                  \
  int vk_trsv_##SUF(int mode, int group, int grid, const void *sys, const void *st, const int32_t *act,             \
                    const VkLevels *lL, const VkLevels *lU, int which, unsigned *bar, int32_t *err, cudaStream_t s) {  \
    return launch_trsv_t<T>(mode, group, grid, (const SysDev<T> *)sys, (const BiState<T> *)st, act, *(const Levels *)lL, \
                            *(const Levels *)lU, which, bar, err, s);                                                \
  }                                                                                                                  \
  int vk_trsv_occupancy_##SUF(int group, int *blocks_per_sm) { return occupancy_persistent_t<T>(group, blocks_per_sm); } \
  void vk_split_factor_##SUF(int64_t n, const int64_t *rp, const int32_t *ci, const double *lu, const int32_t *blk,  \
                             const int64_t *lrp, T *lv, const int64_t *urp, T *uv, T *dinv, cudaStream_t s) {        \
    int grid = (int)((n + kThreads - 1) / kThreads);                                                                 \
    if (grid > 65535 * 16) grid = 65535 * 16;                                                                        \
    if (grid < 1) grid = 1;                                                                                          \
    k_split_factor<T><<<grid, kThreads, 0, s>>>(n, rp, ci, lu, blk, lrp, lv, urp, uv, dinv);                        \
  }                                                                                                                  \
  void vk_spmv_plain_##SUF(int group, int grid, int64_t n, const int64_t *rp, const int32_t *ci, const T *av,       \
                           const T *x, T *y, cudaStream_t s) {                                                       \
    switch (group) {                                                                                                 \
      case 2: k_spmv_plain<T, 2><<<grid, kThreads, 0, s>>>(n, rp, ci, av, x, y); break;                             \
      case 4: k_spmv_plain<T, 4><<<grid, kThreads, 0, s>>>(n, rp, ci, av, x, y); break;                             \
      case 8: k_spmv_plain<T, 8><<<grid, kThreads, 0, s>>>(n, rp, ci, av, x, y); break;                             \
      case 16: k_spmv_plain<T, 16><<<grid, kThreads, 0, s>>>(n, rp, ci, av, x, y); break;                           \
      default: k_spmv_plain<T, 32><<<grid, kThreads, 0, s>>>(n, rp, ci, av, x, y); break;                           \
    }                                                                                                                \
  }

VK_BODY_T(float, f32)
VK_BODY_T(double, f64)

int vk_ilu0(int mode, int grid, const void *fs, const VkLevels *lv, unsigned *bar, int32_t *err, cudaStream_t s) {
  const FactDev *f = (const FactDev *)fs;
  Levels L = *(const Levels *)lv;
  if (mode == 1) {
    void *args[] = {(void *)&f, (void *)&L, (void *)&bar, (void *)&err};
    return (int)cudaLaunchCooperativeKernel((void *)k_ilu0_persistent, dim3(grid), dim3(kThreads), args, 0, s);
  }
  for (int k = 0; k < L.nlev; ++k) k_ilu0_level<<<grid, kThreads, 0, s>>>(f, L, k, err);
  return (int)cudaGetLastError();
}

int vk_ilu0_occupancy(int *blocks_per_sm) {
  return (int)cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, (void *)k_ilu0_persistent, kThreads, 0);
}

size_t vk_factdev_size() { return sizeof(FactDev); }
size_t vk_refdev_size() { return sizeof(RefDev); }
size_t vk_sysdev_size_f32() { return sizeof(SysDev<float>); }
size_t vk_sysdev_size_f64() { return sizeof(SysDev<double>); }
size_t vk_bistate_size_f32() { return sizeof(BiState<float>); }
size_t vk_bistate_size_f64() { return sizeof(BiState<double>); }

void vk_residual64(int group, int ntiles, const void *ref, const VkTiles *tl, double *part, int32_t *cnt, const int32_t *act,
                   double *rnorm2, double *bnorm2, cudaStream_t s) {
  const Tiles t = *(const Tiles *)tl;
  const RefDev *r = (const RefDev *)ref;
  switch (group) {
    case 2: k_residual64<2><<<ntiles, kThreads, 0, s>>>(r, t, part, cnt, act, rnorm2, bnorm2); break;
    case 4: k_residual64<4><<<ntiles, kThreads, 0, s>>>(r, t, part, cnt, act, rnorm2, bnorm2); break;
    case 8: k_residual64<8><<<ntiles, kThreads, 0, s>>>(r, t, part, cnt, act, rnorm2, bnorm2); break;
    case 16: k_residual64<16><<<ntiles, kThreads, 0, s>>>(r, t, part, cnt, act, rnorm2, bnorm2); break;
    default: k_residual64<32><<<ntiles, kThreads, 0, s>>>(r, t, part, cnt, act, rnorm2, bnorm2); break;
  }
}

void vk_scale_to_f32(int ntiles, const void *ref, const void *sys32, const VkTiles *tl, const int32_t *act, const double *rnorm2, cudaStream_t s) {
  k_scale_to_f32<<<ntiles, kThreads, 0, s>>>((const RefDev *)ref, (const SysDev<float> *)sys32, *(const Tiles *)tl, act, rnorm2);
}

void vk_accumulate_x(int ntiles, const void *ref, const void *sys32, const VkTiles *tl, const int32_t *act, const double *rnorm2, cudaStream_t s) {
  k_accumulate_x<<<ntiles, kThreads, 0, s>>>((const RefDev *)ref, (const SysDev<float> *)sys32, *(const Tiles *)tl, act, rnorm2);
}

void vk_cast_f64_f32(int64_t n, const double *a, float *b, cudaStream_t s) {
  int grid = (int)((n + kThreads - 1) / kThreads);
  if (grid > 65535 * 16) grid = 65535 * 16;
  if (grid < 1) grid = 1;
  k_cast_f64_f32<<<grid, kThreads, 0, s>>>(n, a, b);
}

}  // extern "C"

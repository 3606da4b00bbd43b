// solver_kernels.cuh -- device-side data layout shared by the solver kernels
// (solver_kernels.cu) and the C++ host driver (host_solver.cpp).
#pragma once
#include <cstdint>

namespace vshe {

// One linear system of a batch, as the kernels see it (all device pointers).
// T is the arithmetic type of the Krylov iteration (float or double).
template <typename T>
struct SysDev {
  int64_t n;
  // A in precision T (pattern shared with the FP64 copy)
  const int64_t *rp;
  const int32_t *ci;
  const T *av;
  // incomplete factors: strict lower L (unit diagonal), strict upper U, 1 / diag(U)
  const int64_t *lrp; const int32_t *lci; const T *lv;
  const int64_t *urp; const int32_t *uci; const T *uv;
  const T *dinv;
  // Krylov vectors (length n)
  T *x, *r, *rh, *p, *v, *s, *t, *ph, *sh;
};

// Per-system BiCGStab state, resident on the device.
template <typename T>
struct BiState {
  T rho, rho_old, alpha, omega;
  T bnorm;        // ||b|| of the current (inner) solve
  T res;          // ||r|| / ||b||
  T tol;          // relative tolerance of the current (inner) solve
  int32_t iter;   // iterations done in the current solve
  int32_t max_iter;
  int32_t done;   // 1 = converged or stopped
  int32_t s_conv; // 1 = ||s|| already below tol in this iteration
  int32_t status; // 0 ok, VSHE_E_BREAKDOWN, ...
};

// Tiles: contiguous row ranges inside one system.  Reductions are per tile,
// finished by the last tile of the system (sys_tile0[s] .. sys_tile0[s+1]).
struct Tiles {
  int32_t ntiles;
  const int32_t *tile_sys;
  const int64_t *tile_row0;
  const int64_t *tile_row1;
  const int32_t *sys_tile0;
};

// Level schedule of a batch: entries of global level k are
// [lvl_ptr[k], lvl_ptr[k+1]) of (ent_sys, ent_row).
struct Levels {
  int32_t nlev;
  const int64_t *lvl_ptr;
  const int32_t *ent_sys;
  const int32_t *ent_row;
};

// ILU(0) factorisation view of one system (values in FP64, in A's pattern).
struct FactDev {
  int64_t n;
  const int64_t *rp;
  const int32_t *ci;
  double *lu;
  const int64_t *diag;
  const int32_t *blk;
};

// FP64 refinement view of one system: r = b - A x.
struct RefDev {
  int64_t n;
  const int64_t *rp; const int32_t *ci; const double *av;
  const double *b; double *x; double *r;
};

}  // namespace vshe

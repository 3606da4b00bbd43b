// solver_kernels.cuh -- device-side data layout shared by the solver kernels
// (solver_kernels.cu) and the C++ host driver (host_solver.cpp).
#pragma once
#include <cstdint>

namespace vshe {

// One linear system of a batch, as the kernels see it (all device pointers).
//
// The Krylov iteration (SpMV, dot products, vector updates) runs in FP64 on A in the
// caller's row order.  P is the storage and arithmetic type of the ILU(0) triangular
// solves: float for the mixed-precision solver, double for the plain FP64 solver.
//
// The incomplete factors belong to the permuted matrix P A P^T and are stored level by
// level: entry k of the forward solve is row lrow[k] (permuted numbering) with strict
// lower entries [lptr[k], lptr[k+1]) of (lcol, lval); entry k of the backward solve is
// row urow[k] with strict upper entries [uptr[k], uptr[k+1]) and the inverse diagonal
// udinv[k].  lgat[k] / ugat[k] are the original rows of those entries.
template <typename P>
struct SysDev {
  int64_t n;
  const int64_t *rp;
  const int32_t *ci;
  const double *av;
  const double *b;
  const int32_t *lrow; const int64_t *lptr; const int32_t *lcol; const P *lval;
  const int32_t *urow; const int64_t *uptr; const int32_t *ucol; const P *uval; const P *udinv;
  const int32_t *lgat, *ugat;
  P *ytmp;  // permuted-order work vector of the triangular solves
  // Krylov vectors (original order, FP64)
  double *x, *r, *rh, *p, *v, *s, *t, *ph, *sh;
};

// Per-system BiCGStab state, resident on the device.
struct BiState {
  double rho, rho_old, alpha, omega;
  double bnorm;    // ||b||
  double res;      // ||r|| / ||b|| (recursive residual)
  double tol;      // relative tolerance
  int32_t iter;    // iterations done
  int32_t max_iter;
  int32_t done;    // 1 = converged or stopped
  int32_t s_conv;  // 1 = ||s|| already below tol in this iteration
  int32_t status;  // 0 ok, VSHE_E_BREAKDOWN, ...
  int32_t restart; // next iteration restarts the Krylov recurrence (p = r)
  int32_t shadow_r0; // 1: r^ = r_0 instead of the dense pseudo-random shadow
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

// Level schedule of a batch: entries of global level k are [lvl_ptr[k], lvl_ptr[k+1]).
// Triangular solves: entry e is a chunk of ent_cnt[e] <= 32 consecutive level-ordered
// positions of system ent_sys[e] starting at ent_row[e].  Factorisation: entry e is the
// permuted row ent_row[e] of system ent_sys[e] (ent_sys NULL for a single system, ent_cnt NULL).
struct Levels {
  int32_t nlev;
  const int64_t *lvl_ptr;
  const int32_t *ent_sys;
  const int32_t *ent_row;
  const int32_t *ent_cnt;
};

// ILU(0) factorisation view of one system: values in FP64 in the permuted
// matrix's CSR (prp, pci), filled from A's values through amap (permuted entry
// -> original entry); diag[i] = position of the diagonal in row i.
struct FactDev {
  int64_t n;
  const int64_t *rp;
  const int32_t *ci;
  double *lu;
  const int64_t *diag;
  const int32_t *blk;
};

// FP64 residual view of one system: r = b - A x.
struct RefDev {
  int64_t n;
  const int64_t *rp; const int32_t *ci; const double *av;
  const double *b; const double *x; double *r;
};

}  // namespace vshe

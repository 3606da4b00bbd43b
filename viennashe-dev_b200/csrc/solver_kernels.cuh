// solver_kernels.cuh -- device-side data layout shared by the solver kernels
// (solver_kernels.cu) and the C++ host driver (host_solver.cpp).
//
// Solver order.  Every system is solved in its own row order q = 0..n-1, a symmetric
// permutation of the caller's rows (perm[q] = caller row): the preconditioner's base
// ordering (natural, multicolour or caller-given), then stably sorted by the level of the
// forward (L) sweep, then, inside a level, by preconditioner block and by row length.  Rows of one forward level are
// therefore contiguous, and because a level never holds two structurally coupled rows, the
// ILU(0) factors in solver order are those of the base ordering, relabelled.  The Krylov
// vectors live in solver order; b is gathered in and x scattered out once per solve.
//
// SELL-32.  A (in solver order) and the incomplete factors L, U are stored as slices of 32
// rows: entry k of the slice's row `lane` is at off + 32 k + lane, for k below the slice's
// width (the longest row of the slice; shorter rows are padded with value 0 and a column
// that points at a finite entry).  Lane = row, so every value and column load of a warp is
// one coalesced 128/256-byte line and each row is summed by one thread in index order.
#pragma once
#include <cstdint>

namespace vshe {

// One linear system of a batch, as the kernels see it (all device pointers).
//
// The Krylov iteration (SpMV, dot products, vector updates) runs in FP64.  P is the storage
// type of the ILU(0) factors: float for the mixed-precision solver, double for the plain
// FP64 solver; the triangular solves compute in FP64 either way.
//
// A: slices j = rows [32 j, 32 j + 32), entries [aoff[j], aoff[j+1]).
// L: slices in forward-level order; slice j = solver rows [lrow0[j], lrow0[j+1]),
//    entries [loff[j], loff[j+1]) (strict lower part inside the row's block; unit diagonal).
// U: slices in backward-level order over slots; slice j = slots [uslot0[j], uslot0[j+1]),
//    slot t is solver row urow[t] with inverse diagonal udinv[t]; entries [uoff[j], uoff[j+1]).
template <typename P>
struct SysDev {
  int64_t n;
  const int64_t *aoff; const int32_t *acol; const double *aval;
  const double *b;   // rhs, solver order
  const int32_t *lrow0; const int64_t *loff; const int32_t *lcol; const P *lval;
  const int32_t *uslot0; const int64_t *uoff; const int32_t *ucol; const P *uval; const P *udinv; const int32_t *urow;
  double *ytmp;      // forward-sweep result (FP64)
  // level -> slice ranges of this system alone
  const int64_t *lvsL; const int64_t *lvsU; int32_t nlevL, nlevU;
  // Krylov vectors (solver order, FP64)
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

// Tiles: contiguous row ranges of 2048 rows (64 A-slices) inside one system.  Reductions are
// per tile, finished by the last tile of the system (sys_tile0[s] .. sys_tile0[s+1]).
struct Tiles {
  int32_t ntiles;
  const int32_t *tile_sys;
  const int64_t *tile_row0;
  const int64_t *tile_row1;
  const int32_t *sys_tile0;
};

// Level schedule of a batch: entries of global level k are [lvl_ptr[k], lvl_ptr[k+1]).
// Triangular solves: entry e is slice ent_row[e] (of L or U) of system ent_sys[e].
// Factorisation: entry e is the solver row ent_row[e] of system ent_sys[e]; for a single
// system both are NULL and entry e is row e (forward levels are contiguous row ranges).
struct Levels {
  int32_t nlev;
  const int64_t *lvl_ptr;
  const int32_t *ent_sys;
  const int32_t *ent_row;
  const int32_t *ent_cnt;  // unused (NULL)
};

// ILU(0) factorisation view of one system: values in FP64 in the solver-order CSR (rp, ci),
// diag[i] = position of the diagonal in row i; blk[i] = preconditioner block of row i.
struct FactDev {
  int64_t n;
  const int64_t *rp;
  const int32_t *ci;
  double *lu;
  const int64_t *diag;
  const int32_t *blk;
  // ILUT dropping (ilut != 0): a multiplier or entry below tau * ||a_i||_2 is dropped, then only
  // the pkeep largest entries of the row's L part and of its U part are kept
  int32_t ilut, pkeep;
  double tau;
};

// Sweep tasks.  A task is one independent unit of the incomplete-LU apply that one CTA walks
// alone: a preconditioner block of one system (an energy slab of block-ILU: its factor has no
// entry outside the block, so blocks sweep independently), or a whole system.  Its forward
// (L) and backward (U) sweeps are lists of chunks [cL0, cL1) and [cU0, cU1).
//
// A chunk is a run of consecutive SELL slices [s0, s1) of one level whose operands fit one
// shared-memory stage of kTaskStageBytes, staged there by bulk copies in this layout (byte
// offsets, each a multiple of 16):
//   [0, 16 ns)                       ns = s1 - s0 slice descriptors (SliceDesc), from desc + d0
//   [16 ns, +4 nslot)                factor columns of the chunk's slots [o0, o0 + nslot)
//   [.., +sizeof(P) nslot)           factor values of the same slots
//   [.., ..)                         forward sweep: the input vector's rows [r0, r1) (FP64);
//                                    backward sweep: urow[r0, r1), then udinv[r0, r1)
// r0 and r1 are the chunk's first row (L) or slot (U) rounded down, and its end rounded up, to
// a multiple of 4, so that every copy starts and ends on a 16-byte boundary.  A slice too wide
// for a stage is a chunk of its own (kChunkDirect) and is read from global memory.
// kChunkLevelEnd marks the last chunk of a level: the CTA synchronises before the next level.
// rot = (s0 - first slice of the level) mod the consumer warps: slice j of the chunk is summed by
// consumer warp (rot + j - s0) mod the consumer warps, so the slices of a level go round the warps.
constexpr int32_t kChunkLevelEnd = 1;
constexpr int32_t kChunkDirect = 2;
constexpr int32_t kTaskStageBytes = 65536;
constexpr int32_t kTaskConsumers = 31;  // consumer warps of k_trsv_task (one more warp issues the copies)
struct TaskDev {
  int32_t sys, cL0, cL1, cU0, cU1, pad;
};
struct ChunkDev {
  int32_t s0, s1, flags, nslot;
  int64_t o0, d0;
  int32_t r0, r1, rot, pad;
};
struct SliceDesc {
  int32_t soff;   // first slot of the slice, relative to the chunk's o0
  int32_t width;  // entries per row (slots / 32)
  int32_t r0;     // first solver row (L) or slot (U) of the slice
  int32_t nr;     // rows of the slice (at most 32)
};
// Bytes one chunk occupies in a stage (the layout above), for factor values of `vbytes` bytes.
inline constexpr int64_t task_chunk_bytes(int64_t ns, int64_t nslot, int64_t r0, int64_t r1, bool lower, int vbytes) {
  return 16 * ns + (4 + vbytes) * nslot + (r1 - r0) * (lower ? 8 : 4 + vbytes);
}

// Cluster sweep tasks (k_trsv_cluster): the same units as TaskDev, walked by one thread-block
// cluster each, level by level, with the slices of level k of the forward (backward) sweep in
// [lv[offL + 2k], lv[offL + 2k + 1]) ([lv[offU + 2k], ...)).
struct ClusterTask {
  int32_t sys, nlevL, nlevU, pad;
  int64_t offL, offU;
};

// FP64 residual view of one system (solver order): r = b - A x.
struct RefDev {
  int64_t n;
  const int64_t *aoff; const int32_t *acol; const double *aval;
  const double *b; const double *x; double *r;
};

}  // namespace vshe

// she_kernels.h -- device views of one SHE problem and the launchers of she_kernels.cu
// (part of the thin internal C ABI between the C++ host code and the kernels).
#pragma once
#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

namespace vshe {

// Read-only tables of one SHE problem on the device (see she_host.h for their meaning).
struct SheDev {
  int32_t dim, nc, nf, NH, D, L;
  double T;
  // cells
  const int32_t *mat, *contact, *cf_ptr, *cf_idx, *inc_dir_even;
  const double *vol, *cen, *shift_c;
  const char *mask_c;
  // facets
  const int32_t *fcell, *inc_dir_odd;
  const double *fvol, *fnorm, *shift_f;
  // (x, H) space
  const double *Hval, *bnd_c;
  const int32_t *ord_c, *ord_f;
  const int64_t *idx_c, *idx_f;
  const int32_t *even_nodes, *odd_nodes;
  int64_t n_even_nodes, n_odd_nodes;
  int64_t n_even, n_odd;
  const int32_t *even_harm, *odd_harm;
  const double *cblocks;
  // physics
  int32_t acoustic, optical, bnd_type, scaling_type;
  double rate_ac, rate_op, n_op, hbar_omega, tau;
  double ax01[3], ay01[3];
};

// The assembled full (even + odd) system in CSR.
struct FullDev {
  const int64_t *rp;
  const int32_t *ci;
  const double *val;
  const double *rhs;
};

}  // namespace vshe

extern "C" {
int vk_she_assemble_even(const vshe::SheDev *P, int pass, int64_t *rowlen, const int64_t *rp, int32_t *ci, double *val,
                         double *rhs, int32_t *err, cudaStream_t s);
int vk_she_assemble_odd(const vshe::SheDev *P, int pass, int64_t *rowlen, const int64_t *rp, int32_t *ci, double *val,
                        double *rhs, int32_t *err, cudaStream_t s);
int vk_she_schur(const vshe::FullDev *A, int64_t n_even, int pass, int64_t *rowlen, const int64_t *rrp, int32_t *rci,
                 double *rval, double *rrhs, uint8_t *ins_diag, int32_t *err, cudaStream_t s);
int vk_scan_rowptr(int64_t *rp, int64_t n, void *tmp, size_t *tmp_bytes, cudaStream_t s);
int vk_she_normalise(const vshe::SheDev *P, int64_t n, const int64_t *rp, const int32_t *ci, double *val, double *rhs,
                     const uint8_t *ins_diag, int scale, double *s_vec, double *sf, int64_t *diag_pos, int64_t *cptr,
                     int64_t *cursor, int64_t *cpos, void *tmp, size_t tmp_bytes, cudaStream_t s);
int vk_she_finish(const vshe::SheDev *P, const vshe::FullDev *A, const double *x_red, const double *s_vec,
                  const double *sf, int scale, double *xf, double *part, double *dens, int ncontacts, double *cur,
                  cudaStream_t s);
int vk_she_residual_blocks(int64_t n_full);
}

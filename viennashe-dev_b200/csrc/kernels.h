// kernels.h -- the thin internal C ABI between the C++ host code and the CUDA
// kernels: every launcher takes plain pointers, sizes and a stream.
#pragma once
#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

extern "C" {

// Same layout as vshe::Tiles / vshe::Levels (solver_kernels.cuh).
typedef struct VkTiles {
  int32_t ntiles;
  const int32_t *tile_sys;
  const int64_t *tile_row0;
  const int64_t *tile_row1;
  const int32_t *sys_tile0;
} VkTiles;

typedef struct VkLevels {
  int32_t nlev;
  const int64_t *lvl_ptr;
  const int32_t *ent_sys;
  const int32_t *ent_row;
  const int32_t *ent_cnt;
} VkLevels;

int vk_threads(void);
// process-wide count of this library's kernel launches (library kernels such as CUB scans excluded)
void vk_count_launches(long long k);
long long vk_launches_total(void);
size_t vk_factdev_size(void);
size_t vk_refdev_size(void);
size_t vk_sysdev_size(void);   // SysDev<float> and SysDev<double> have the same layout
size_t vk_bistate_size(void);

// BiCGStab (FP64), one launch per step over all tiles of a batch
void vk_bicg_init(int ntiles, const void *sys, void *st, const VkTiles *tl, double *part, int32_t *cnt, const int32_t *act, cudaStream_t s);
void vk_bicg_resume(int ntiles, const void *sys, void *st, const VkTiles *tl, double *part, int32_t *cnt, const int32_t *act, cudaStream_t s);
void vk_update_p(int ntiles, const void *sys, void *st, const VkTiles *tl, const int32_t *act, cudaStream_t s);
void vk_spmv_dot(int ntiles, const void *sys, void *st, const VkTiles *tl, double *part, int32_t *cnt, const int32_t *act, int which, cudaStream_t s);
void vk_update_s(int ntiles, const void *sys, void *st, const VkTiles *tl, double *part, int32_t *cnt, const int32_t *act, cudaStream_t s);
void vk_update_xr(int ntiles, const void *sys, void *st, const VkTiles *tl, double *part, int32_t *cnt, const int32_t *act, cudaStream_t s);
void vk_precond_copy(int ntiles, const void *sys, const void *st, const VkTiles *tl, const int32_t *act, int which, cudaStream_t s);

// ILU(0) apply in factor precision P (f32 / f64); mode 1 = one persistent cooperative launch,
// 2 = one launch per level.  bar: 4 words (arrival count, generation, poll limit as uint64) that
// every bounded device-side wait of the batch reads; k_trsv_task sweeps one task per CTA.
#define VK_DECL_P(P, SUF)                                                                                               \
  int vk_trsv_##SUF(int mode, int grid, const void *sys, const void *st, const int32_t *act,                          \
                    const VkLevels *lL, const VkLevels *lU, int which, unsigned *bar, int32_t *err, cudaStream_t s);    \
  int vk_trsv_occupancy_##SUF(int *blocks_per_sm);                                                                     \
  int vk_trsv_task_##SUF(int ntasks, const void *sys, const void *st, const int32_t *act, const void *tasks,          \
                         const void *chunks, const void *sdesc, int which, const unsigned *bar, int32_t *err,      \
                         cudaStream_t s);                                                                           \
  int vk_trsv_cluster_##SUF(int ntasks, int csize, const void *sys, const void *st, const int32_t *act, const void *tasks, \
                            const int64_t *lv, int which, cudaStream_t s);                                           \
  void vk_split_factor_##SUF(int64_t nnz, int64_t n, const double *lu, const int64_t *fmap, const int64_t *diag,       \
                             const int64_t *dpos, P *lval, P *uval, P *udinv, cudaStream_t s);

VK_DECL_P(float, f32)
VK_DECL_P(double, f64)

// y = A x on a SELL-32 matrix (solver order)
void vk_spmv_plain(int grid, int64_t n, const int64_t *aoff, const int32_t *acol, const double *aval, const double *x, double *y, cudaStream_t s);
// out[q] = in[perm[q]] (gather = 1) or out[perm[q]] = in[q] (gather = 0)
void vk_permute(int64_t n, const int32_t *perm, const double *in, double *out, int gather, cudaStream_t s);

int vk_ilu0(int mode, int grid, const void *fs, const VkLevels *lv, unsigned *bar, int32_t *err, cudaStream_t s);
int vk_ilu0_occupancy(int *blocks_per_sm);
// out[k] = av[amap[k]] (0 where amap[k] < 0)
void vk_gather_values(int64_t nnz, const int64_t *amap, const double *av, double *out, cudaStream_t s);

// r = b - A x in FP64 (solver order, written to the RefDev's r), ||r||^2 and ||b||^2 per system
void vk_residual64(int ntiles, const void *ref, const VkTiles *tl, double *part, int32_t *cnt,
                   const int32_t *act, double *rnorm2, double *bnorm2, cudaStream_t s);

}  // extern "C"

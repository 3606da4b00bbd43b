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
size_t vk_sysdev_size_f32(void);
size_t vk_sysdev_size_f64(void);
size_t vk_bistate_size_f32(void);
size_t vk_bistate_size_f64(void);

#define VK_DECL_T(T, SUF)                                                                                               \
  void vk_bicg_init_##SUF(int ntiles, const void *sys, void *st, const VkTiles *tl, T *part, int32_t *cnt,             \
                          const int32_t *act, cudaStream_t s);                                                         \
  void vk_update_p_##SUF(int ntiles, const void *sys, void *st, const VkTiles *tl, const int32_t *act,                \
                         cudaStream_t s);                                                                              \
  void vk_spmv_dot_##SUF(int ntiles, const void *sys, void *st, const VkTiles *tl, T *part, int32_t *cnt,              \
                         const int32_t *act, int which, cudaStream_t s);                                               \
  void vk_update_s_##SUF(int ntiles, const void *sys, void *st, const VkTiles *tl, T *part, int32_t *cnt,             \
                         const int32_t *act, cudaStream_t s);                                                          \
  void vk_update_xr_##SUF(int ntiles, const void *sys, void *st, const VkTiles *tl, T *part, int32_t *cnt,            \
                          const int32_t *act, int reliable, cudaStream_t s);                                           \
  void vk_precond_copy_##SUF(int ntiles, const void *sys, const void *st, const VkTiles *tl, const int32_t *act,      \
                             int which, cudaStream_t s);                                                               \
  int vk_trsv_##SUF(int mode, int grid, const void *sys, const void *st, const int32_t *act,                          \
                    const VkLevels *lL, const VkLevels *lU, int which, unsigned *bar, int32_t *err, cudaStream_t s);    \
  int vk_trsv_occupancy_##SUF(int *blocks_per_sm);                                                                     \
  void vk_split_factor_##SUF(int64_t nnz, int64_t n, const double *lu, const int64_t *fmap, const int64_t *diag,       \
                             const int64_t *dpos, T *lval, T *uval, T *udinv, cudaStream_t s);                         \
  void vk_spmv_plain_##SUF(int grid, int64_t n, const int64_t *rp, const int32_t *ci, const T *av,                    \
                           const T *x, T *y, cudaStream_t s);

VK_DECL_T(float, f32)
VK_DECL_T(double, f64)

int vk_ilu0(int mode, int grid, const void *fs, const VkLevels *lv, unsigned *bar, int32_t *err, cudaStream_t s);
int vk_ilu0_occupancy(int *blocks_per_sm);

void vk_residual64(int ntiles, const void *ref, const VkTiles *tl, double *part, int32_t *cnt,
                   const int32_t *act, double *rnorm2, double *bnorm2, cudaStream_t s);
void vk_reliable_x(int ntiles, const void *sys32, const void *st, const VkTiles *tl, const int32_t *act, cudaStream_t s);
// r64 = b - A x64, then r32 = r64 / ||r64|| with p, v carried to the new scale (two launches);
// force = 1 starts the mixed solve (x64 = 0) and initialises the FP32 recurrence.
void vk_reliable_r(int ntiles, const void *sys32, void *st, const VkTiles *tl, double *part, int32_t *cnt,
                   const int32_t *act, double tol64, int force, cudaStream_t s);
void vk_gather_values(int64_t nnz, const int64_t *amap, const double *av, double *lu, cudaStream_t s);
void vk_cast_f64_f32(int64_t n, const double *a, float *b, cudaStream_t s);

}  // extern "C"

// poisson_kernels.h -- device view of the outer loop's Poisson problem (poisson_kernels.cu) and
// its launchers, shared with the host driver (poisson.cpp).
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

namespace vshe {

// The cell mesh (vshe_device_desc, on the device), the unknown numbering (the non-contact cells
// in cell order) and the CSR of the linearised Poisson system: row u is cell row_cell[u]; the
// diagonal entry of row u is at diag_pos[u]; the entry of the neighbour across the cell's facet
// slot k (an index into cf_idx) is at fpos[k] when that neighbour is an unknown.
struct PoissonDev {
  int32_t n_cells, n_facets, dim, n_unk;
  double temperature;
  const int32_t *row_cell, *unk, *material;
  const double *volume, *centroid, *doping_n, *doping_p;
  const int32_t *facet_cells;
  const double *facet_volume, *facet_normal, *facet_centroid;
  const int32_t *cf_ptr, *cf_idx;
  const int64_t *diag_pos, *fpos;
  const double *bval;  // boundary value of every contact cell (its description potential)
};

}  // namespace vshe

int vk_poisson_assemble(const vshe::PoissonDev *P, const double *psi, const double *n, const double *p, double *val,
                        double *rhs, cudaStream_t s);
int vk_poisson_update(const vshe::PoissonDev *P, const double *psi, const double *dpsi, double alpha, double *out,
                      cudaStream_t s);

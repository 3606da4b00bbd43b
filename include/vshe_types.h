/*
 * vshe_types.h -- plain-C descriptions of a SHE problem, shared by the GPU
 * library (vshe_gpu.h) and by any host that feeds it.
 *
 * Everything is flat arrays + sizes: no C++ or CUDA types cross this boundary.
 * Units are SI throughout (m, m^-3, V, J, K, s), as in ViennaSHE.
 */
#ifndef VSHE_TYPES_H
#define VSHE_TYPES_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Material ids, same numbering as viennashe/materials/all.hpp (si::id = 0, metal::id = 100). */
#define VSHE_MATERIAL_SI     0    /* materials/all.hpp: si, the semiconductor */
#define VSHE_MATERIAL_SIO2   1    /* insulators (Poisson only): sio2, hfo2, sion, gas */
#define VSHE_MATERIAL_HFO2   2
#define VSHE_MATERIAL_SION   3
#define VSHE_MATERIAL_GAS    4
#define VSHE_MATERIAL_METAL  100

/* SHE boundary condition types (viennashe/forwards.h boundary_type_id subset used by SHE). */
#define VSHE_BOUNDARY_GENERATION_RECOMBINATION 0
#define VSHE_BOUNDARY_DIRICHLET                1

/* Unknown scaling (viennashe/config.hpp she_scaling_type_id). */
#define VSHE_SCALING_KINETIC_ENERGY 0
#define VSHE_SCALING_TOTAL_ENERGY   1

/*
 * A device on a mesh of cells (boxes) and facets, the information ViennaSHE
 * reads from its ViennaGrid mesh + device container during SHE assembly.
 *
 * Facets:   facet_cells[2f], facet_cells[2f+1] are the two cells of facet f in
 *           coboundary order (c1, c2); c2 = -1 on the domain boundary.
 * Cells:    the facets of cell c, in the cell's local facet order, are
 *           cell_facet_idx[cell_facet_ptr[c] .. cell_facet_ptr[c+1]).
 * Potential is the electrostatic potential per cell (contact cells carry their
 * Dirichlet value: contact potential + built-in potential).
 */
typedef struct vshe_device_desc {
  int32_t dim;                    /* 1 or 2 */
  int32_t n_cells;
  int32_t n_facets;
  const int32_t *cell_material;   /* n_cells: VSHE_MATERIAL_* */
  const double  *cell_volume;     /* n_cells: length (1D) or area (2D) */
  const double  *cell_centroid;   /* n_cells * dim */
  const double  *doping_n;        /* n_cells, m^-3 */
  const double  *doping_p;        /* n_cells, m^-3 */
  const double  *potential;       /* n_cells, V */
  const int32_t *contact_id;      /* n_cells: -1, or the contact (terminal) this metal cell belongs to */
  const int32_t *facet_cells;     /* n_facets * 2 */
  const double  *facet_volume;    /* n_facets: 1 in 1D, edge length in 2D */
  const double  *facet_normal;    /* n_facets * dim: unit normal, pointing from c1 to c2 */
  const int32_t *cell_facet_ptr;  /* n_cells + 1 */
  const int32_t *cell_facet_idx;  /* cell_facet_ptr[n_cells] */
  double         temperature;     /* lattice temperature, K */
} vshe_device_desc;

/*
 * SHE configuration: the subset of viennashe::config the SHE linear-solve path
 * reads (electrons only, phonon scattering, Modena dispersion, even/odd DF
 * discretisation, H-transformation on).
 */
typedef struct vshe_she_config {
  int32_t max_expansion_order;        /* L (odd: 1, 3, 5, 7) */
  double  energy_spacing;             /* J */
  double  min_kinetic_energy_range;   /* J */
  double  max_kinetic_energy_range;   /* J (reference default 5 eV) */
  int32_t acoustic_phonon;            /* enable flags */
  int32_t optical_phonon;
  double  acoustic_fit_factor;        /* reference default 1.05 (electrons) */
  double  optical_fit_factor;         /* reference default 0.7 */
  int32_t boundary_type;              /* VSHE_BOUNDARY_* */
  double  gr_tau;                     /* generation/recombination time, s (default 1e-16) */
  int32_t scaling_type;               /* VSHE_SCALING_* */
  int32_t scale;                      /* linear_solver_config::scale() */
} vshe_she_config;

/*
 * Spherical-harmonics coupling tables a_{x,y,z}, b_{x,y,z} of order L, each a
 * dense D x D row-major block with D = (L+1)^2, in that order (6 blocks).
 * An entry is "stored" (part of the coupling matrix's sparsity pattern) iff it
 * is non-zero, as in viennashe/she/harmonics_coupling.hpp.
 */
typedef struct vshe_coupling_tables {
  int32_t       L;
  const double *data;   /* 6 * D * D */
} vshe_coupling_tables;

#ifdef __cplusplus
}
#endif

#endif /* VSHE_TYPES_H */

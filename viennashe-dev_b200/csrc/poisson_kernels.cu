// poisson_kernels.cu -- the Gummel-linearised Poisson system of the outer loop and the damped
// potential update (viennashe/assemble.hpp:165-345, viennashe/simulator.hpp:606-647).
// Compiled without FMA contraction: the assembly is the reference's FP64 arithmetic term by
// term, so that it agrees with the oracle's restatement to rounding.
#include <cuda_runtime.h>
#include <cstdint>

#include "poisson_kernels.h"

namespace vshe {

namespace {
constexpr double kQ = 1.602176565e-19;   // As (physics/constants.hpp)
constexpr double kKB = 1.3806488e-23;    // J/K
constexpr double kPi = 3.1415926535897932384626433832795;
constexpr double kC0 = 299792458.0;

__device__ __forceinline__ double eps0() { return 1.0e7 / (4.0 * kPi * kC0 * kC0); }

// materials/all.hpp: relative permittivities of si, sio2, hfo2, sion, gas (metal cells are
// contacts and take no row)
__device__ __forceinline__ double permittivity(int32_t m) {
  switch (m) {
    case 0: return 11.9 * eps0();
    case 1: return 3.9 * eps0();
    case 2: return 25.0 * eps0();
    case 3: return 10.0 * eps0();
    case 4: return 1.0 * eps0();
    default: return 0.0;
  }
}

__device__ __forceinline__ double dist(const double *a, const double *b, int dim) {
  double s = 0.0;
  for (int d = 0; d < dim; ++d) s += (a[d] - b[d]) * (a[d] - b[d]);
  return sqrt(s);
}
}  // namespace

// One thread per unknown row (a non-contact cell): its row of A and its rhs entry, facet by
// facet in the cell's facet order, then the cell's volume terms, in the reference's order of
// operations (assemble.hpp:215-300).
__global__ void k_poisson_assemble(PoissonDev P, const double *__restrict__ psi, const double *__restrict__ n,
                                   const double *__restrict__ p, double *__restrict__ val, double *__restrict__ rhs) {
  const int u = blockIdx.x * blockDim.x + threadIdx.x;
  if (u >= P.n_unk) return;
  const int c = P.row_cell[u];
  const int dim = P.dim;
  const double *cc = P.centroid + (size_t)c * dim;
  const double psi_c = psi[c];
  const double eps_c = permittivity(P.material[c]);
  double a = 0.0, b = 0.0;
  for (int k = P.cf_ptr[c]; k < P.cf_ptr[c + 1]; ++k) {
    const int f = P.cf_idx[k];
    const int c1 = P.facet_cells[2 * f], c2 = P.facet_cells[2 * f + 1];
    const int o = c1 == c ? c2 : c1;
    if (o < 0) continue;  // domain boundary: homogeneous Neumann
    const double *co = P.centroid + (size_t)o * dim;
    double conn[3], len = 0.0;
    for (int d = 0; d < dim; ++d) { conn[d] = co[d] - cc[d]; len += conn[d] * conn[d]; }
    len = sqrt(len);
    double ip = 0.0;
    const double sgn = c1 == c ? 1.0 : -1.0;  // the outer normal of c at f
    for (int d = 0; d < dim; ++d) ip += (sgn * P.facet_normal[(size_t)f * dim + d]) * (conn[d] / len);
    const double wia = P.facet_volume[f] * ip;
    const int col = P.unk[o];
    if (col >= 0) {
      const double *fc = P.facet_centroid + (size_t)f * dim;
      const double dc = dist(fc, cc, dim), dn = dist(fc, co, dim);
      const double em = (dc + dn) / (dc / eps_c + dn / permittivity(P.material[o]));
      val[P.fpos[k]] = em * wia / len;
      a -= em * wia / len;
      b -= em * wia * (psi[o] - psi_c) / len;
    } else {
      a -= eps_c * wia / len;
      b -= eps_c * wia / len * (P.bval[o] - psi_c);
    }
  }
  const double vol = P.volume[c];
  if (P.material[c] == 0) {
    const double vt = (kKB * P.temperature) / kQ;
    a -= vol * kQ * (n[c] + p[c]) / vt;
    b += vol * kQ * (n[c] - P.doping_n[c] - p[c] + P.doping_p[c]);
  }
  val[P.diag_pos[u]] = a;
  rhs[u] = b;
}

// psi_out = (1 - alpha) psi + alpha psi_new with psi_new = psi + dpsi on unknown cells and the
// boundary value on contact cells (simulator.hpp:616-645, no logarithmic damping).
__global__ void k_poisson_update(PoissonDev P, const double *__restrict__ psi, const double *__restrict__ dpsi,
                                 double alpha, double *__restrict__ out) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= P.n_cells) return;
  const double cur = psi[c];
  const int u = P.unk[c];
  const double nv = u < 0 ? P.bval[c] : cur + dpsi[u];
  out[c] = cur * (1.0 - alpha) + nv * alpha;
}

}  // namespace vshe

using namespace vshe;

int vk_poisson_assemble(const PoissonDev *P, const double *psi, const double *n, const double *p, double *val, double *rhs,
                        cudaStream_t s) {
  if (P->n_unk <= 0) return 0;
  k_poisson_assemble<<<(P->n_unk + 255) / 256, 256, 0, s>>>(*P, psi, n, p, val, rhs);
  return (int)cudaGetLastError();
}

int vk_poisson_update(const PoissonDev *P, const double *psi, const double *dpsi, double alpha, double *out, cudaStream_t s) {
  if (P->n_cells <= 0) return 0;
  k_poisson_update<<<(P->n_cells + 255) / 256, 256, 0, s>>>(*P, psi, dpsi, alpha, out);
  return (int)cudaGetLastError();
}

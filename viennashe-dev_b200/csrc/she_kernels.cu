// she_kernels.cu -- device-side SHE operator assembly, odd elimination,
// scaling/normalisation and post-processing (FP64).
//
// Each kernel runs twice over the same enumeration: a count pass that sizes
// the CSR rows and a fill pass that writes sorted columns and values, so the
// sparsity pattern is built on the GPU with no host-side matrix.  Values are
// accumulated per entry in the order the reference accumulates them, and this
// file is compiled without FMA contraction (-fmad=false) so the arithmetic is
// the reference's.
//
//   K1 assemble_even   viennashe/she/assemble_all.hpp:227-309 with assemble_boundary.hpp:69-183,
//                      assemble_scattering.hpp:116-335, assemble_streaming.hpp:73-365
//   K2 assemble_odd    viennashe/she/assemble_all.hpp:317-393 (+ zero erasure, eliminate.hpp:195-212)
//   K3 schur           viennashe/she/eliminate.hpp:226-293
//   K4 normalise       viennashe/she/rescaling.hpp:50-107, viennashe/math/linalg_util.hpp:202-282
//   K10 finish         viennashe/she/linear_solver.hpp:172-186, eliminate.hpp:305-354,
//                      she/postproc/carrier_density.hpp:68-130, current_density.hpp:66-131,
//                      postproc/terminal_current.hpp:47-105

#include <cuda_runtime.h>
#include <cub/cub.cuh>
#include <cstdint>

#include "she_kernels.h"
#include "kernels.h"

namespace vshe {
namespace she {

struct K {
  static constexpr double PI = 3.1415926535897932384626433832795;
  static constexpr double Q = 1.602176565e-19;
  static constexpr double KB = 1.3806488e-23;
  static constexpr double M0 = 9.10938291e-31;
};

__device__ __forceinline__ double m_dos() { return 0.32 * K::M0; }
__device__ __forceinline__ double m_long() { return 0.98 * K::M0; }
__device__ __forceinline__ double m_trans() { return 0.19 * K::M0; }
__device__ __forceinline__ double m_cond() { return 3.0 / (1.0 / m_long() + 1.0 / m_trans() + 1.0 / m_trans()); }
__device__ __forceinline__ double hbar() { return 6.62606896e-34 / (2.0 * 3.1415926535897932384626433832795); }

// Modena dispersion (viennashe/physics/dispersion.hpp:207-286)
__device__ double dos(double eps) {
  if (eps > 0.0) {
    const double alpha = 0.5 / K::Q;
    const double mstar = m_dos();
    const double hb = hbar();
    const double prefactor = mstar * sqrt(2.0 * mstar) / (8.0 * K::PI * K::PI * K::PI * hb * hb * hb);
    return prefactor * 4.0 * K::PI * (1.0 + 2.0 * alpha * eps) * sqrt(eps * (1.0 + alpha * eps));
  }
  return 0.0;
}
__device__ double velocity(double eps) {
  if (eps < 0) return 0;
  const double alpha = 0.5 / K::Q;
  double gamma = eps * (1.0 + alpha * eps);
  double dgam = 1.0 + 2.0 * alpha * eps;
  double mc = m_cond(), md = m_dos();
  return sqrt(mc / md) * sqrt(2.0 * gamma / m_dos()) / dgam;
}

__device__ __forceinline__ int even_on_node(int L) { int n = 0; for (int l = 0; l <= L; l += 2) n += 2 * l + 1; return n; }
__device__ __forceinline__ int odd_on_node(int L) { int n = 0; for (int l = 1; l <= L; l += 2) n += 2 * l + 1; return n; }

// kinetic energy of an element (cell: shift_c, facet: shift_f)
struct Elem {
  const SheDev *P;
  bool facet;
  int id;
  __device__ double ek(int H) const { return P->Hval[H] - (facet ? P->shift_f[id] : P->shift_c[id]); }
};

// assemble_common.hpp:412-427
__device__ double box_height(const Elem &e, int H) {
  double h = 0;
  if (H > 0) h = fabs(e.ek(H) - e.ek(H - 1));
  if (H < e.P->NH - 1) h += fabs(e.ek(H + 1) - e.ek(H));
  return h / 2.0;
}
// assemble_common.hpp:433-462
__device__ double avg_dos(const Elem &e, int H) {
  double Z = dos(e.ek(H));
  double n = 1;
  if (H < e.P->NH - 1) { Z += dos((e.ek(H) + e.ek(H + 1)) / 2.0); ++n; }
  if (H > 0) { Z += dos((e.ek(H) + e.ek(H - 1)) / 2.0); ++n; }
  return Z / n;
}
// assemble_common.hpp:521-551
__device__ double integral_vZ(const Elem &e, int H) {
  double kc = e.ek(H);
  double vZ = velocity(kc) * dos(kc);
  double n = 1;
  if (H < e.P->NH - 1) { double k = (e.ek(H) + e.ek(H + 1)) / 2.0; vZ += velocity(k) * dos(k); ++n; }
  if (H > 0) { double k = (e.ek(H) + e.ek(H - 1)) / 2.0; vZ += velocity(k) * dos(k); ++n; }
  vZ /= n;
  return vZ * box_height(e, H);
}
// assemble_common.hpp:153-164 (the interval is ordered for the energies used here)
__device__ double integral_Z_over_hk(double em, double ep) {
  return 0.5 * (dos(ep) * velocity(ep) - dos(em) * velocity(em));
}
__device__ double ekc(const SheDev &P, int c, int H) { return P.Hval[H] - P.shift_c[c]; }
// assemble_common.hpp:325-388
__device__ double lower_ke_facet(const SheDev &P, int f, int H) {
  int c1 = P.fcell[2 * f], c2 = P.fcell[2 * f + 1];
  if (c2 < 0) return ekc(P, c1, H);
  if (H == 0) return ekc(P, c1, H) + ekc(P, c2, H) / 2.0;
  return (ekc(P, c1, H - 1) + ekc(P, c2, H - 1) + ekc(P, c1, H) + ekc(P, c2, H)) / 4.0;
}
__device__ double upper_ke_facet(const SheDev &P, int f, int H) {
  int c1 = P.fcell[2 * f], c2 = P.fcell[2 * f + 1];
  if (c2 < 0) return ekc(P, c1, H);
  if (H == P.NH - 1) return ekc(P, c1, H) + ekc(P, c2, H) / 2.0;
  return (ekc(P, c1, H + 1) + ekc(P, c2, H + 1) + ekc(P, c1, H) + ekc(P, c2, H)) / 4.0;
}
__device__ double cell_dist(const SheDev &P, int a, int b) {
  double s = 0;
  for (int d = 0; d < P.dim; ++d) { double t = P.cen[a * P.dim + d] - P.cen[b * P.dim + d]; s += t * t; }
  return sqrt(s);
}
// assemble_scattering.hpp:65-105
__device__ int energy_index_H(const Elem &e, int hint, double kin) {
  int res = hint;
  const int NH = e.P->NH;
  if (kin < e.ek(res) || kin > e.ek(res)) {
    int inc = 1;
    double diff = kin - e.ek(res);
    double diff0 = diff;
    if (diff < 0) inc = -1;
    while (res < NH - 1 && res > 0 && diff * diff0 > 0) {
      res += inc;
      diff = kin - e.ek(res);
    }
    if (diff * diff0 > 0) return -1;
    double e1 = fabs(diff), e2 = e1;
    if (res - inc >= 0 && res - inc < NH) e2 = fabs(kin - e.ek(res - inc));
    if (e2 < e1) return res - inc;
  }
  return res;
}

// Scattering events of one (element, H) in the reference's process/event order
// (acoustic_phonon_scattering.hpp:83-114, optical_phonon_scattering.hpp:122-179).
struct Event { double coef_out, coef_in; int col_out, col_in; bool elastic; };

__device__ int scattering_events(const SheDev &P, const Elem &e, int H, double V, Event *ev) {
  const double kin = e.ek(H);
  int ne = 0;
  double ei[5], ef[5], rate[5];
  int nproc = 0;
  if (P.acoustic) {
    ei[nproc] = kin; ef[nproc] = kin; rate[nproc] = P.rate_ac; ++nproc;
  }
  if (P.optical) {
    const double w = P.hbar_omega;
    ei[nproc] = kin;     ef[nproc] = kin - w; rate[nproc] = P.rate_op * (P.n_op + 1.0); ++nproc;
    ei[nproc] = kin + w; ef[nproc] = kin;     rate[nproc] = P.rate_op * (P.n_op + 1.0); ++nproc;
    ei[nproc] = kin;     ef[nproc] = kin + w; rate[nproc] = P.rate_op * P.n_op;         ++nproc;
    ei[nproc] = kin - w; ef[nproc] = kin;     rate[nproc] = P.rate_op * P.n_op;         ++nproc;
  }
  const int NH = P.NH;
  for (int s = 0; s < nproc; ++s) {
    Event E; E.col_out = -1; E.col_in = -1; E.coef_out = 0; E.coef_in = 0; E.elastic = false;
    if (rate[s] <= 0) { ev[ne++] = E; continue; }
    int iHi = energy_index_H(e, H, ei[s]);
    int iHf = energy_index_H(e, H, ef[s]);
    if (iHi == -1 || iHf == -1) { ev[ne++] = E; continue; }
    const double Zi = avg_dos(e, iHi), Zf = avg_dos(e, iHf);
    const double h = fmin(box_height(e, iHi), box_height(e, iHf));
    E.elastic = (iHi == iHf) && !e.facet;
    const int64_t *idx = e.facet ? P.idx_f : P.idx_c;
    if (ei[s] <= kin && ei[s] >= kin) {
      int64_t col = idx[(int64_t)e.id * NH + iHf];
      if (col >= 0) { E.col_out = (int)col; E.coef_out = 2.0 * K::PI * rate[s] * Zi * Zf * V * h; }
    }
    if (ef[s] <= kin && ef[s] >= kin) {
      int64_t col = idx[(int64_t)e.id * NH + iHi];
      if (col >= 0) { E.col_in = (int)col; E.coef_in = -2.0 * K::PI * rate[s] * Zi * Zf * V * h - 0.0 * Zi * V * h; }
    }
    ev[ne++] = E;
  }
  return ne;
}

// streaming coefficients for (cell, facet, H): assemble_streaming.hpp:73-365
__device__ void streaming_coefs(const SheDev &P, int cell, int facet, int H, double &cd, double &cdr) {
  const int other = P.fcell[2 * facet] == cell ? P.fcell[2 * facet + 1] : P.fcell[2 * facet];
  double conn[2] = {0, 0};
  for (int d = 0; d < P.dim; ++d) conn[d] = P.cen[cell * P.dim + d] - P.cen[other * P.dim + d];
  double len = 0;
  for (int d = 0; d < P.dim; ++d) len += conn[d] * conn[d];
  len = sqrt(len);
  const double sgn = (P.fcell[2 * facet] == cell) ? 1.0 : -1.0;
  double dot = 0;
  for (int d = 0; d < P.dim; ++d) dot += sgn * P.fnorm[facet * P.dim + d] * (conn[d] / len);
  const double warea = P.fvol[facet] * fabs(dot);
  Elem fe{&P, true, facet};
  cd = integral_vZ(fe, H) * warea;
  const double lo = lower_ke_facet(P, facet, H), up = upper_ke_facet(P, facet, H);
  const double izhk = integral_Z_over_hk(lo, up);
  const double force = (ekc(P, cell, H) - ekc(P, other, H)) / cell_dist(P, other, cell);
  cdr = izhk * force * warea * len / 2.0;
}

// ------------------------------------------------------------------ K1: even rows
constexpr int kMaxFacets = 8;
constexpr int kMaxEvenCols = 8;

__global__ void k_assemble_even(SheDev P, int pass, int64_t *rowlen, const int64_t *rp, int32_t *ci, double *val, double *rhs, int32_t *err) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= P.n_even_nodes) return;
  const int C = P.even_nodes[2 * k], H = P.even_nodes[2 * k + 1];
  const int NH = P.NH;
  const int64_t row0 = P.idx_c[(int64_t)C * NH + H];
  const int ord = P.ord_c[(int64_t)C * NH + H];
  const int ne = even_on_node(ord);
  const bool metal = P.mat[C] == 100;
  Elem ce{&P, false, C};
  // boundary (generation/recombination or Dirichlet): assemble_boundary.hpp:69-183
  double coef_bnd = 0.0, bnd = 0.0;
  const bool has_bnd = P.contact[C] >= 0;
  if (has_bnd) {
    bnd = P.bnd_c[(int64_t)C * NH + H];
    const double height = box_height(ce, H);
    if (P.bnd_type == 1) coef_bnd = height * avg_dos(ce, H);
    else coef_bnd = P.vol[C] * height / P.tau * avg_dos(ce, H);
  }
  Event ev[5];
  int nev = 0;
  if (!metal) nev = scattering_events(P, ce, H, P.vol[C], ev);
  // facets of C carrying odd unknowns at H, sorted by their unknown index
  int fs[kMaxFacets], fslot[kMaxFacets];
  int64_t fbase[kMaxFacets];
  int nfac = 0;
  for (int q = P.cf_ptr[C]; q < P.cf_ptr[C + 1] && nfac < kMaxFacets; ++q) {
    const int f = P.cf_idx[q];
    const int c1 = P.fcell[2 * f], c2 = P.fcell[2 * f + 1];
    if (c2 < 0) continue;
    (void)c1;
    const int64_t b = P.idx_f[(int64_t)f * NH + H];
    if (b < 0) continue;
    int pos = nfac++;
    while (pos > 0 && fbase[pos - 1] > b) { fs[pos] = fs[pos - 1]; fslot[pos] = fslot[pos - 1]; fbase[pos] = fbase[pos - 1]; --pos; }
    fs[pos] = f; fslot[pos] = q; fbase[pos] = b;
  }
  double cdv[kMaxFacets], cdrv[kMaxFacets];
  for (int j = 0; j < nfac; ++j) streaming_coefs(P, C, fs[j], H, cdv[j], cdrv[j]);
  const int D = P.D;
  for (int p = 0; p < ne; ++p) {
    const int64_t row = row0 + p;
    const int h = P.even_harm[p];
    // even columns (diagonal and in-scattering), accumulated in the reference's order
    int64_t ecol[kMaxEvenCols];
    double evl[kMaxEvenCols];
    int nec = 0;
    auto add_even = [&](int64_t col, double v) {
      for (int t = 0; t < nec; ++t) if (ecol[t] == col) { evl[t] += v; return; }
      if (nec < kMaxEvenCols) { ecol[nec] = col; evl[nec] = 0.0 + v; ++nec; }
      else atomicExch(err, -1);
    };
    if (has_bnd) add_even(row, coef_bnd);
    for (int s = 0; s < nev; ++s) {
      if (ev[s].col_out >= 0 && !(ev[s].elastic && p == 0)) add_even(row, ev[s].coef_out);
      if (ev[s].col_in >= 0 && p == 0 && !ev[s].elastic) add_even(ev[s].col_in, ev[s].coef_in);
    }
    for (int a = 1; a < nec; ++a) {  // insertion sort by column
      int64_t c = ecol[a]; double v = evl[a]; int b = a - 1;
      while (b >= 0 && ecol[b] > c) { ecol[b + 1] = ecol[b]; evl[b + 1] = evl[b]; --b; }
      ecol[b + 1] = c; evl[b + 1] = v;
    }
    const bool erase_zero = (row == P.n_even - 1);
    int64_t cnt = 0;
    const int64_t out = (pass == 1) ? rp[row] : 0;
    const int64_t lim = (pass == 1) ? rp[row + 1] - rp[row] : 0;
    for (int t = 0; t < nec; ++t) {
      if (erase_zero && evl[t] == 0.0) continue;
      if (pass == 1 && cnt < lim) { ci[out + cnt] = (int32_t)ecol[t]; val[out + cnt] = evl[t]; }
      ++cnt;
    }
    for (int j = 0; j < nfac; ++j) {
      const int f = fs[j];
      const int ordf = P.ord_f[(int64_t)f * NH + H];
      const int no = odd_on_node(ordf);
      const int dk = P.inc_dir_even[fslot[j]];
      const double *Cd = P.cblocks + ((size_t)dk * 4 + 0) * D * D;
      const double *Cb = P.cblocks + ((size_t)dk * 4 + 1) * D * D;
      for (int q = 0; q < no; ++q) {
        const int g = P.odd_harm[q];
        const double a = Cd[h * D + g], b = Cb[h * D + g];
        if (a == 0.0 && b == 0.0) continue;
        double v = 0.0;
        if (a != 0.0) v += cdv[j] * a;
        if (b != 0.0) v += cdrv[j] * b;
        if (erase_zero && v == 0.0) continue;
        if (pass == 1 && cnt < lim) { ci[out + cnt] = (int32_t)(fbase[j] + q); val[out + cnt] = v; }
        ++cnt;
      }
    }
    if (pass == 0) rowlen[row] = cnt;
    else {
      if (cnt != lim) atomicExch(err, -100);  // pattern changed since the count pass
      // write_boundary (assemble_common.hpp:302-319): only the zeroth harmonic row gets the rhs
      double b = 0.0;
      if (has_bnd && p == 0) { const double pre = -bnd * coef_bnd; b = b - pre * 1.0; }
      rhs[row] = b;
    }
  }
}

// ------------------------------------------------------------------ K2: odd rows
__global__ void k_assemble_odd(SheDev P, int pass, int64_t *rowlen, const int64_t *rp, int32_t *ci, double *val, double *rhs, int32_t *err) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= P.n_odd_nodes) return;
  const int F = P.odd_nodes[2 * k], H = P.odd_nodes[2 * k + 1];
  const int NH = P.NH;
  const int64_t row0 = P.idx_f[(int64_t)F * NH + H];
  const int ord = P.ord_f[(int64_t)F * NH + H];
  const int no = odd_on_node(ord);
  const int c1 = P.fcell[2 * F], c2 = P.fcell[2 * F + 1];
  Elem fe{&P, true, F};
  const double V = P.fvol[F] * cell_dist(P, c1, c2) / (double)P.dim;
  Event ev[5];
  const int nev = scattering_events(P, fe, H, V, ev);
  double diag = 0.0;
  bool has_diag = false;
  for (int s = 0; s < nev; ++s)
    if (ev[s].col_out >= 0) { diag += ev[s].coef_out; has_diag = true; }
  // the two cells in order of their unknown index
  int cs[2] = {c1, c2}, side[2] = {0, 1};
  int64_t cb[2] = {P.idx_c[(int64_t)c1 * NH + H], P.idx_c[(int64_t)c2 * NH + H]};
  if (cb[1] < cb[0]) { int t = cs[0]; cs[0] = cs[1]; cs[1] = t; t = side[0]; side[0] = side[1]; side[1] = t; int64_t u = cb[0]; cb[0] = cb[1]; cb[1] = u; }
  double cdv[2], cdrv[2];
  for (int j = 0; j < 2; ++j) streaming_coefs(P, cs[j], F, H, cdv[j], cdrv[j]);
  const int D = P.D;
  for (int q = 0; q < no; ++q) {
    const int64_t row = row0 + q;
    const int g = P.odd_harm[q];
    int64_t cnt = 0;
    const int64_t out = (pass == 1) ? rp[row] : 0;
    const int64_t lim = (pass == 1) ? rp[row + 1] - rp[row] : 0;
    for (int j = 0; j < 2; ++j) {
      const int cc = cs[j];
      const int ordc = P.ord_c[(int64_t)cc * NH + H];
      const int ne = even_on_node(ordc);
      const int dk = P.inc_dir_odd[2 * F + side[j]];
      const double *Cd = P.cblocks + ((size_t)dk * 4 + 2) * D * D;
      const double *Cb = P.cblocks + ((size_t)dk * 4 + 3) * D * D;
      for (int p = 0; p < ne; ++p) {
        const int h = P.even_harm[p];
        const double a = Cd[g * D + h], b = Cb[g * D + h];
        if (a == 0.0 && b == 0.0) continue;
        double v = 0.0;
        if (a != 0.0) v += cdv[j] * a;
        if (b != 0.0) v += cdrv[j] * b;
        if (v == 0.0) continue;  // eliminate.hpp:195-212: zero entries leave the odd rows
        if (pass == 1 && cnt < lim) { ci[out + cnt] = (int32_t)(cb[j] + p); val[out + cnt] = v; }
        ++cnt;
      }
    }
    if (has_diag && diag != 0.0) {
      if (pass == 1 && cnt < lim) { ci[out + cnt] = (int32_t)row; val[out + cnt] = diag; }
      ++cnt;
    }
    if (pass == 0) rowlen[row] = cnt;
    else {
      rhs[row] = 0.0;
      if (cnt != lim) atomicExch(err, -100);
    }
  }
}

// ------------------------------------------------------------------ K3: Schur complement
constexpr int kMaxRed = 192;

// Columns and values of reduced row i, in the order eliminate.hpp:236-288 produces them.
__device__ int schur_row(const FullDev &A, int64_t i, int64_t n_even, int64_t *cols, double *vals, double &brow, bool want_vals, int32_t *err) {
  int n = 0;
  auto upsert = [&](int64_t c) -> int {
    int lo = 0, hi = n - 1;
    while (lo <= hi) { int mid = (lo + hi) >> 1; if (cols[mid] == c) return mid; if (cols[mid] < c) lo = mid + 1; else hi = mid - 1; }
    if (n >= kMaxRed) { atomicExch(err, -1); return -1; }
    for (int t = n; t > lo; --t) { cols[t] = cols[t - 1]; vals[t] = vals[t - 1]; }
    cols[lo] = c; vals[lo] = 0.0; ++n;
    return lo;
  };
  if (want_vals) brow = A.rhs[i];
  for (int64_t q = A.rp[i]; q < A.rp[i + 1]; ++q) {
    const int64_t c = A.ci[q];
    if (c < n_even) {
      int t = upsert(c);
      if (t >= 0 && want_vals) vals[t] += A.val[q];
      continue;
    }
    // odd unknown c: its diagonal is the last entry of the (diagonal) odd row
    const int64_t a = A.rp[c], b = A.rp[c + 1];
    double d = -1.0;
    for (int64_t r = a; r < b; ++r) if (A.ci[r] == c) { d = A.val[r]; break; }
    if (d <= 0.0) { atomicExch(err, -4); return n; }
    const double s = A.val[q];
    for (int64_t r = a; r < b; ++r) {
      const int64_t j = A.ci[r];
      if (j >= n_even) continue;
      int t = upsert(j);
      if (t >= 0 && want_vals) vals[t] -= s * A.val[r] / d;
    }
    if (want_vals) brow -= s * A.rhs[c] / d;
  }
  return n;
}

__global__ void k_schur(FullDev A, int64_t n_even, int pass, int64_t *rowlen, const int64_t *rrp, int32_t *rci, double *rval, double *rrhs, uint8_t *ins_diag, int32_t *err) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_even) return;
  int64_t cols[kMaxRed];
  double vals[kMaxRed];
  double brow = 0.0;
  int n = schur_row(A, i, n_even, cols, vals, brow, pass == 1, err);
  // the normalisation's non-const access A(i, i) inserts a zero diagonal if absent (linalg_util.hpp:232, :258)
  bool has_diag = false;
  for (int t = 0; t < n; ++t) if (cols[t] == i) { has_diag = true; break; }
  if (pass == 0) { rowlen[i] = n + (has_diag ? 0 : 1); return; }
  const int64_t out = rrp[i];
  if (rrp[i + 1] - out != n + (has_diag ? 0 : 1)) { atomicExch(err, -100); return; }
  int w = 0;
  bool placed = has_diag;
  for (int t = 0; t < n; ++t) {
    if (!placed && cols[t] > i) { rci[out + w] = (int32_t)i; rval[out + w] = 0.0; ++w; placed = true; }
    rci[out + w] = (int32_t)cols[t]; rval[out + w] = vals[t]; ++w;
  }
  if (!placed) { rci[out + w] = (int32_t)i; rval[out + w] = 0.0; ++w; }
  rrhs[i] = brow;
  ins_diag[i] = has_diag ? 0 : 1;
}

// ------------------------------------------------------------------ K4: scaling and normalisation
__global__ void k_unknown_scaling(SheDev P, double *s) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= P.n_even_nodes) return;
  const int C = P.even_nodes[2 * k], H = P.even_nodes[2 * k + 1];
  const int64_t base = P.idx_c[(int64_t)C * P.NH + H];
  const int num = even_on_node(P.ord_c[(int64_t)C * P.NH + H]);
  const double T = P.T;
  double v;
  if (P.scaling_type == 0) v = exp(-(P.Hval[H] - P.shift_c[C]) / (K::KB * T));
  else v = exp(-P.Hval[H] / (K::KB * T));
  for (int i = 0; i < num; ++i) s[base + i] = v;
}

__global__ void k_rescale(int64_t n, const int64_t *rp, const int32_t *ci, double *val, const double *s) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  for (int64_t q = rp[i]; q < rp[i + 1]; ++q) val[q] *= s[ci[q]];
}

__global__ void k_col_count(int64_t n, const int64_t *rp, const int32_t *ci, int64_t *ccnt) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  for (int64_t q = rp[i]; q < rp[i + 1]; ++q) atomicAdd((unsigned long long *)&ccnt[ci[q] + 1], 1ull);
}
__global__ void k_col_fill(int64_t n, const int64_t *rp, const int32_t *ci, const int64_t *cptr, int64_t *cursor, int64_t *cpos) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  for (int64_t q = rp[i]; q < rp[i + 1]; ++q) {
    const int32_t j = ci[q];
    const int64_t slot = cptr[j] + (int64_t)atomicAdd((unsigned long long *)&cursor[j], 1ull);
    cpos[slot] = q;
  }
}
// sort each column's entry positions by row (position order = row order in CSR)
__global__ void k_col_sort(int64_t n, const int64_t *cptr, int64_t *cpos) {
  const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  const int64_t a = cptr[j], b = cptr[j + 1];
  for (int64_t x = a + 1; x < b; ++x) {
    int64_t v = cpos[x], y = x - 1;
    while (y >= a && cpos[y] > v) { cpos[y + 1] = cpos[y]; --y; }
    cpos[y + 1] = v;
  }
}
// column geometric means (log-sums in ascending row order), linalg_util.hpp:214-243
__global__ void k_col_normalise(int64_t n, const int64_t *cptr, const int64_t *cpos, const int32_t *ci, const int64_t *rp_unused,
                                double *val, const uint8_t *ins_diag, const int64_t *diag_pos, double *sf) {
  const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  const int64_t a = cptr[j], b = cptr[j + 1];
  const int64_t dq = diag_pos[j];
  double sum = 0.0;
  int64_t cnt = 0;
  for (int64_t x = a; x < b; ++x) {
    const int64_t q = cpos[x];
    if (ins_diag[j] && q == dq) continue;  // inserted after the mean is taken
    sum += log(fabs(val[q]));
    ++cnt;
  }
  double nrm = exp(sum / (double)cnt);
  if (val[dq] < 0.0) nrm *= -1.0;
  for (int64_t x = a; x < b; ++x) { const int64_t q = cpos[x]; val[q] /= nrm; }
  sf[j] = 1.0 / nrm;
}
// row 2-norms with positive diagonal, linalg_util.hpp:247-277
__global__ void k_row_normalise(int64_t n, const int64_t *rp, const int32_t *ci, double *val, double *rhs, const int64_t *diag_pos) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double s = 0.0;
  for (int64_t q = rp[i]; q < rp[i + 1]; ++q) s += val[q] * val[q];
  s = sqrt(s);
  if (val[diag_pos[i]] < 0.0) s *= -1.0;
  for (int64_t q = rp[i]; q < rp[i + 1]; ++q) val[q] /= s;
  rhs[i] /= s;
}
__global__ void k_diag_pos(int64_t n, const int64_t *rp, const int32_t *ci, int64_t *dpos) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int64_t d = -1;
  for (int64_t q = rp[i]; q < rp[i + 1]; ++q) if (ci[q] == i) { d = q; break; }
  dpos[i] = d;
}

// ------------------------------------------------------------------ K10: finish
// x_even = x_red * (s * sf) (linear_solver.hpp:172-176)
__global__ void k_unscale(int64_t n, const double *xr, const double *s, const double *sf, int scale, double *xf) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  xf[i] = scale ? xr[i] * (s[i] * sf[i]) : xr[i];
}
// odd unknowns from the even ones (eliminate.hpp:305-354)
__global__ void k_recover_odd(FullDev A, int64_t n_even, int64_t n_full, double *xf) {
  const int64_t i = n_even + (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_full) return;
  double d = 0.0, x = A.rhs[i];
  for (int64_t q = A.rp[i]; q < A.rp[i + 1]; ++q) {
    const int64_t j = A.ci[q];
    if (j < n_even) x -= A.val[q] * xf[j];
    else if (j == i) d = A.val[q];
  }
  xf[i] = x / d;
}
// ||A x - b||^2 and ||b||^2 partials per block (summed on the host in block order)
__global__ void k_full_residual(FullDev A, int64_t n_full, const double *xf, double *part) {
  __shared__ double sh[2][256];
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  double r2 = 0.0, b2 = 0.0;
  if (i < n_full) {
    double s = 0.0;
    for (int64_t q = A.rp[i]; q < A.rp[i + 1]; ++q) s += A.val[q] * xf[A.ci[q]];
    const double t = s - A.rhs[i];
    r2 = t * t;
    b2 = A.rhs[i] * A.rhs[i];
  }
  sh[0][threadIdx.x] = r2; sh[1][threadIdx.x] = b2;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o) { sh[0][threadIdx.x] += sh[0][threadIdx.x + o]; sh[1][threadIdx.x] += sh[1][threadIdx.x + o]; }
    __syncthreads();
  }
  if (threadIdx.x == 0) { part[2 * blockIdx.x] = sh[0][0]; part[2 * blockIdx.x + 1] = sh[1][0]; }
}
// carrier density per cell (carrier_density.hpp:68-130)
__global__ void k_density(SheDev P, const double *xf, double *dens) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= P.nc) return;
  Elem e{&P, false, c};
  const int NH = P.NH;
  double d = 0;
  for (int H = 1; H < NH - 1; ++H) {
    const double lo = fmax((e.ek(H - 1) + e.ek(H)) / 2.0, 0.0);
    const double up = fmin((e.ek(H + 1) + e.ek(H)) / 2.0, 1.0);
    if (P.mask_c[c]) {
      const int64_t u = P.idx_c[(int64_t)c * NH + H];
      if (u < 0) continue;
      if (up >= 0 && lo < up) d += xf[u] * avg_dos(e, H) * box_height(e, H);
    } else {
      if (up >= 0 && lo < up) d += P.bnd_c[(int64_t)c * NH + H] * avg_dos(e, H) * box_height(e, H);
    }
  }
  dens[c] = d * 6.0;
}
// current through facet f (current_density.hpp:66-131)
__device__ double facet_current(const SheDev &P, const double *xf, int f) {
  const int c1 = P.fcell[2 * f], c2 = P.fcell[2 * f + 1];
  if (c2 < 0) return 0;
  double nrm[2] = {0, 0}, len = 0;
  for (int d = 0; d < P.dim; ++d) { nrm[d] = P.cen[c2 * P.dim + d] - P.cen[c1 * P.dim + d]; len += nrm[d] * nrm[d]; }
  len = sqrt(len);
  for (int d = 0; d < P.dim; ++d) nrm[d] /= len;
  const double mt = m_trans(), md = m_dos();
  Elem fe{&P, true, f};
  double vn = 0;
  for (int H = 1; H < P.NH - 1; ++H) {
    const int64_t u = P.idx_f[(int64_t)f * P.NH + H];
    if (u < 0) continue;
    const double factor = integral_vZ(fe, H) * 6.0;
    const double *v = xf + u;
    vn += (P.ax01[0] * v[0] + P.ax01[1] * v[1] + P.ax01[2] * v[2]) * factor * sqrt(md / mt) * nrm[0];
    if (P.dim > 1) vn += (P.ay01[0] * v[0] + P.ay01[1] * v[1] + P.ay01[2] * v[2]) * factor * sqrt(md / mt) * nrm[1];
  }
  const double Y00 = sqrt((2.0 * 0 + 1.0) * 1.0 / (2.0 * K::PI * 1.0)) * 1.0 / sqrt(2.0);
  return -(-1.0) * K::Q * vn / Y00;
}
// terminal current per contact, one thread per contact walking its cells in order (terminal_current.hpp:47-105)
__global__ void k_terminal_currents(SheDev P, const double *xf, int ncontacts, double *cur) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= ncontacts) return;
  double I = 0.0;
  for (int c = 0; c < P.nc; ++c) {
    if (P.contact[c] != k) continue;
    for (int j = P.cf_ptr[c]; j < P.cf_ptr[c + 1]; ++j) {
      const int f = P.cf_idx[j];
      const int c1 = P.fcell[2 * f], c2 = P.fcell[2 * f + 1];
      if (c2 < 0) continue;
      const int o = (c1 == c) ? c2 : c1;
      if (P.mat[o] != 0) continue;
      double conn[2] = {0, 0}, len = 0;
      for (int d = 0; d < P.dim; ++d) { conn[d] = P.cen[o * P.dim + d] - P.cen[c * P.dim + d]; len += conn[d] * conn[d]; }
      len = sqrt(len);
      const double sgn = (c1 == c) ? 1.0 : -1.0;
      double dt = 0;
      for (int d = 0; d < P.dim; ++d) dt += sgn * P.fnorm[f * P.dim + d] * conn[d] / len;
      const double wa = P.fvol[f] * dt;
      const double J = facet_current(P, xf, f);
      if (c1 == c) I += J * wa; else I -= J * wa;
    }
  }
  cur[k] = I;
}

}  // namespace she
}  // namespace vshe

// ======================================================================= launchers
using namespace vshe;
using namespace vshe::she;

static inline int blocks_for(int64_t n, int t = 256) { return (int)((n + t - 1) / t); }

extern "C" {

int vk_she_assemble_even(const SheDev *P, int pass, int64_t *rowlen, const int64_t *rp, int32_t *ci, double *val, double *rhs, int32_t *err, cudaStream_t s) {
  if (P->n_even_nodes == 0) return 0;
  vk_count_launches(1);
  k_assemble_even<<<blocks_for(P->n_even_nodes, 128), 128, 0, s>>>(*P, pass, rowlen, rp, ci, val, rhs, err);
  return (int)cudaGetLastError();
}
int vk_she_assemble_odd(const SheDev *P, int pass, int64_t *rowlen, const int64_t *rp, int32_t *ci, double *val, double *rhs, int32_t *err, cudaStream_t s) {
  if (P->n_odd_nodes == 0) return 0;
  vk_count_launches(1);
  k_assemble_odd<<<blocks_for(P->n_odd_nodes, 128), 128, 0, s>>>(*P, pass, rowlen, rp, ci, val, rhs, err);
  return (int)cudaGetLastError();
}
int vk_she_schur(const FullDev *A, int64_t n_even, int pass, int64_t *rowlen, const int64_t *rrp, int32_t *rci, double *rval, double *rrhs, uint8_t *ins_diag, int32_t *err, cudaStream_t s) {
  vk_count_launches(1);
  k_schur<<<blocks_for(n_even, 64), 64, 0, s>>>(*A, n_even, pass, rowlen, rrp, rci, rval, rrhs, ins_diag, err);
  return (int)cudaGetLastError();
}
// rp[0] = 0 and rp[1..n] = row lengths on entry; inclusive scan in place
int vk_scan_rowptr(int64_t *rp, int64_t n, void *tmp, size_t *tmp_bytes, cudaStream_t s) {
  return (int)cub::DeviceScan::InclusiveSum(tmp, *tmp_bytes, rp + 1, rp + 1, n, s);
}
int vk_she_normalise(const SheDev *P, int64_t n, const int64_t *rp, const int32_t *ci, double *val, double *rhs, const uint8_t *ins_diag,
                     int scale, double *s_vec, double *sf, int64_t *diag_pos, int64_t *cptr, int64_t *cursor, int64_t *cpos,
                     void *tmp, size_t tmp_bytes, cudaStream_t s) {
  cudaError_t e;
  const int g = blocks_for(n);
  vk_count_launches(1);
  k_diag_pos<<<g, 256, 0, s>>>(n, rp, ci, diag_pos);
  if (scale) {
    vk_count_launches(1);
    k_unknown_scaling<<<blocks_for(P->n_even_nodes), 256, 0, s>>>(*P, s_vec);
    vk_count_launches(1);
    k_rescale<<<g, 256, 0, s>>>(n, rp, ci, val, s_vec);
  }
  if ((e = cudaMemsetAsync(cptr, 0, sizeof(int64_t) * (size_t)(n + 1), s)) != cudaSuccess) return (int)e;
  if ((e = cudaMemsetAsync(cursor, 0, sizeof(int64_t) * (size_t)n, s)) != cudaSuccess) return (int)e;
  vk_count_launches(1);
  k_col_count<<<g, 256, 0, s>>>(n, rp, ci, cptr);
  size_t tb = tmp_bytes;
  if ((e = cub::DeviceScan::InclusiveSum(tmp, tb, cptr + 1, cptr + 1, n, s)) != cudaSuccess) return (int)e;
  vk_count_launches(1);
  k_col_fill<<<g, 256, 0, s>>>(n, rp, ci, cptr, cursor, cpos);
  vk_count_launches(1);
  k_col_sort<<<g, 256, 0, s>>>(n, cptr, cpos);
  vk_count_launches(1);
  k_col_normalise<<<g, 256, 0, s>>>(n, cptr, cpos, ci, rp, val, ins_diag, diag_pos, sf);
  vk_count_launches(1);
  k_row_normalise<<<g, 256, 0, s>>>(n, rp, ci, val, rhs, diag_pos);
  return (int)cudaGetLastError();
}
int vk_she_finish(const SheDev *P, const FullDev *A, const double *x_red, const double *s_vec, const double *sf, int scale,
                  double *xf, double *part, double *dens, int ncontacts, double *cur, cudaStream_t s) {
  const int64_t ne = P->n_even, nf = P->n_even + P->n_odd;
  vk_count_launches(1);
  k_unscale<<<blocks_for(ne), 256, 0, s>>>(ne, x_red, s_vec, sf, scale, xf);
  if (P->n_odd > 0) { vk_count_launches(1); k_recover_odd<<<blocks_for(P->n_odd), 256, 0, s>>>(*A, ne, nf, xf); }
  vk_count_launches(1);
  k_full_residual<<<blocks_for(nf), 256, 0, s>>>(*A, nf, xf, part);
  vk_count_launches(1);
  k_density<<<blocks_for(P->nc), 256, 0, s>>>(*P, xf, dens);
  if (ncontacts > 0) { vk_count_launches(1); k_terminal_currents<<<1, 32, 0, s>>>(*P, xf, ncontacts, cur); }
  return (int)cudaGetLastError();
}
int vk_she_residual_blocks(int64_t n_full) { return blocks_for(n_full); }

}  // extern "C"

// poisson.cpp -- the outer loop's Gummel update of the electrostatic potential on the device
// (vshe_poisson_*): pattern and unknown numbering on the host, assembly and the damped update in
// poisson_kernels.cu, the FP64 solve by the batch solver of host_solver.cpp.
//
// Reference: viennashe/simulator.hpp:1029-1052 (one spatial Gummel step: assemble, solve,
// ||dpsi||, ||b||, damped update), viennashe/assemble.hpp:165-345 (assemble_poisson with the
// Gummel term), viennashe/simulator.hpp:606-647 (update_quantity with damping).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>
#include <cuda_runtime.h>
#include "../../include/vshe_gpu.h"
#include "host_internal.h"
#include "poisson_kernels.h"

namespace vshe {

struct PoissonProblem {
  int32_t nc = 0, nf = 0, dim = 0, nu = 0;
  int64_t nnz = 0;
  std::vector<int64_t> rp;
  std::vector<int32_t> ci;
  DevArena arena;
  PoissonDev P{};
  double *d_psi = nullptr, *d_n = nullptr, *d_p = nullptr, *d_val = nullptr, *d_rhs = nullptr, *d_out = nullptr;
  int64_t *d_rp = nullptr;
  int32_t *d_ci = nullptr;
  std::unique_ptr<System> sys;
  std::unique_ptr<Batch> batch;
  bool assembled = false;
  size_t bytes() const {
    size_t t = arena.total;
    if (sys) t += sys->arena.total;
    if (batch) t += batch->arena.total + batch->tile_arena.total;
    return t;
  }
};

static std::mutex g_poi_mu;
static std::map<Ctx *, std::map<int64_t, std::unique_ptr<PoissonProblem>>> g_poi;

size_t poisson_bytes(Ctx *ctx) {
  std::lock_guard<std::mutex> lk(g_poi_mu);
  size_t t = 0;
  auto it = g_poi.find(ctx);
  if (it != g_poi.end())
    for (auto &kv : it->second) t += kv.second->bytes();
  return t;
}

void poisson_release_all(Ctx *ctx) {
  std::lock_guard<std::mutex> lk(g_poi_mu);
  g_poi.erase(ctx);
}

static PoissonProblem *find_poisson(Ctx *ctx, int64_t h) {
  std::lock_guard<std::mutex> lk(g_poi_mu);
  auto it = g_poi.find(ctx);
  if (it == g_poi.end()) return nullptr;
  auto f = it->second.find(h);
  return f == it->second.end() ? nullptr : f->second.get();
}

template <typename T>
static T *upload(Ctx &ctx, DevArena &ar, const T *src, size_t count, int &rc) {
  cudaError_t e;
  T *p = (T *)ar.alloc(sizeof(T) * std::max<size_t>(count, 1), e);
  if (!p) { rc = ctx.cuda_fail(e, "cudaMalloc poisson"); return nullptr; }
  if (src && count && (e = cudaMemcpyAsync(p, src, sizeof(T) * count, cudaMemcpyHostToDevice, ctx.stream)) != cudaSuccess) {
    rc = ctx.cuda_fail(e, "upload poisson");
    return nullptr;
  }
  rc = VSHE_OK;
  return p;
}

static bool has_permittivity(int32_t m) { return m >= VSHE_MATERIAL_SI && m <= VSHE_MATERIAL_GAS; }

}  // namespace vshe

using namespace vshe;

extern "C" {

int vshe_poisson_create(vshe_ctx *ctx, const vshe_device_desc *d, const double *facet_centroid, const vshe_solve_opts *opts,
                        int64_t *handle) {
  if (!ctx || !d || !facet_centroid || !handle) return VSHE_E_INVALID_ARGUMENT;
  if ((d->dim != 1 && d->dim != 2) || d->n_cells <= 0 || d->n_facets < 0 || !d->cell_material || !d->cell_volume ||
      !d->cell_centroid || !d->doping_n || !d->doping_p || !d->potential || !d->contact_id || !d->facet_cells ||
      !d->facet_volume || !d->facet_normal || !d->cell_facet_ptr || !d->cell_facet_idx || !(d->temperature > 0.0))
    return VSHE_E_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lk(ctx->mu);
  cudaSetDevice(ctx->device);
  const int32_t nc = d->n_cells, nf = d->n_facets, dim = d->dim;
  const int32_t *cfp = d->cell_facet_ptr, *cfi = d->cell_facet_idx, *fc = d->facet_cells;
  if (cfp[0] != 0) return ctx->fail(VSHE_E_INVALID_ARGUMENT, "cell_facet_ptr[0] != 0");
  for (int32_t c = 0; c < nc; ++c)
    if (cfp[c + 1] < cfp[c]) return ctx->fail(VSHE_E_INVALID_ARGUMENT, "cell_facet_ptr not monotone");
  for (int32_t k = 0; k < cfp[nc]; ++k)
    if (cfi[k] < 0 || cfi[k] >= nf) return ctx->fail(VSHE_E_INVALID_ARGUMENT, "cell_facet_idx out of range");
  for (int32_t f = 0; f < nf; ++f)
    for (int s = 0; s < 2; ++s)
      if (fc[2 * f + s] < -1 || fc[2 * f + s] >= nc) return ctx->fail(VSHE_E_INVALID_ARGUMENT, "facet_cells out of range");
  std::unique_ptr<PoissonProblem> Q(new PoissonProblem);
  Q->nc = nc; Q->nf = nf; Q->dim = dim;
  // unknowns: the non-contact cells, in cell order
  std::vector<int32_t> unk((size_t)nc, -1), row_cell;
  for (int32_t c = 0; c < nc; ++c) {
    if (d->contact_id[c] >= 0) continue;
    if (!has_permittivity(d->cell_material[c]))
      return ctx->fail(VSHE_E_INVALID_ARGUMENT, "cell " + std::to_string(c) + " is not a contact and has no permittivity");
    unk[(size_t)c] = int32_t(row_cell.size());
    row_cell.push_back(c);
  }
  const int32_t nu = int32_t(row_cell.size());
  Q->nu = nu;
  // pattern: per row its diagonal and its unknown neighbours, columns ascending
  std::vector<int64_t> diag_pos((size_t)std::max(nu, 1), 0), fpos((size_t)std::max(cfp[nc], 1), -1);
  Q->rp.assign((size_t)nu + 1, 0);
  std::vector<int32_t> cols;
  for (int32_t u = 0; u < nu; ++u) {
    const int32_t c = row_cell[(size_t)u];
    cols.assign(1, u);
    for (int32_t k = cfp[c]; k < cfp[c + 1]; ++k) {
      const int32_t f = cfi[k], o = fc[2 * f] == c ? fc[2 * f + 1] : fc[2 * f];
      if (o >= 0 && unk[(size_t)o] >= 0) cols.push_back(unk[(size_t)o]);
    }
    std::sort(cols.begin(), cols.end());
    cols.erase(std::unique(cols.begin(), cols.end()), cols.end());
    const int64_t r0 = int64_t(Q->ci.size());
    for (int32_t j : cols) Q->ci.push_back(j);
    Q->rp[(size_t)u + 1] = int64_t(Q->ci.size());
    auto pos = [&](int32_t j) { return r0 + int64_t(std::lower_bound(cols.begin(), cols.end(), j) - cols.begin()); };
    diag_pos[(size_t)u] = pos(u);
    for (int32_t k = cfp[c]; k < cfp[c + 1]; ++k) {
      const int32_t f = cfi[k], o = fc[2 * f] == c ? fc[2 * f + 1] : fc[2 * f];
      if (o >= 0 && unk[(size_t)o] >= 0) fpos[(size_t)k] = pos(unk[(size_t)o]);
    }
  }
  Q->nnz = int64_t(Q->ci.size());
  const int64_t nnz = Q->nnz;
  // admission against the context's budget (a bound of the tables below and of the solver)
  const size_t est = size_t(nc) * 128 + size_t(nf) * 64 + size_t(cfp[nc]) * 12 +
                     size_t(nnz) * (4 + 8 + 8 + 4 + 8 + 8 + 8 + 8) + size_t(nu) * (8 * 8 + 9 * 8 + 32) + (size_t(1) << 20);
  if (vshe_bytes_in_use(ctx) + est > ctx->budget) return ctx->fail(VSHE_E_BUDGET, std::to_string(est) + " bytes requested");
  int rc = VSHE_OK;
  DevArena &ar = Q->arena;
  PoissonDev &P = Q->P;
  P.n_cells = nc; P.n_facets = nf; P.dim = dim; P.n_unk = nu; P.temperature = d->temperature;
#define UP(dst, src, count) dst = upload(*ctx, ar, src, size_t(count), rc); if (rc) return rc;
  UP(P.row_cell, row_cell.data(), nu);
  UP(P.unk, unk.data(), nc);
  UP(P.material, d->cell_material, nc);
  UP(P.volume, d->cell_volume, nc);
  UP(P.centroid, d->cell_centroid, size_t(nc) * dim);
  UP(P.doping_n, d->doping_n, nc);
  UP(P.doping_p, d->doping_p, nc);
  UP(P.facet_cells, fc, size_t(nf) * 2);
  UP(P.facet_volume, d->facet_volume, nf);
  UP(P.facet_normal, d->facet_normal, size_t(nf) * dim);
  UP(P.facet_centroid, facet_centroid, size_t(nf) * dim);
  UP(P.cf_ptr, cfp, size_t(nc) + 1);
  UP(P.cf_idx, cfi, cfp[nc]);
  UP(P.diag_pos, diag_pos.data(), nu);
  UP(P.fpos, fpos.data(), cfp[nc]);
  UP(P.bval, d->potential, nc);
  UP(Q->d_rp, Q->rp.data(), size_t(nu) + 1);
  UP(Q->d_ci, Q->ci.data(), nnz);
  UP(Q->d_val, (const double *)nullptr, nnz);
  UP(Q->d_rhs, (const double *)nullptr, nu);
  UP(Q->d_psi, (const double *)nullptr, nc);
  UP(Q->d_n, (const double *)nullptr, nc);
  UP(Q->d_p, (const double *)nullptr, nc);
  UP(Q->d_out, (const double *)nullptr, nc);
#undef UP
  cudaError_t e = cudaMemsetAsync(Q->d_val, 0, sizeof(double) * size_t(std::max<int64_t>(nnz, 1)), ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) return ctx->cuda_fail(e, "poisson upload");
  if (nu > 0) {
    vshe_solve_opts o;
    if (opts) o = *opts;
    else {
      vshe_default_opts(&o);
      o.precond = VSHE_PRECOND_ILU0;
      o.ordering = VSHE_ORDER_NATURAL;
      o.tol = 1e-12;
      o.max_iters = 10000;
    }
    o.precision = VSHE_PRECISION_FP64;
    Q->sys.reset(new System);
    rc = Q->sys->create_borrowed(*ctx, nu, nnz, Q->rp.data(), Q->ci.data(), Q->d_rp, Q->d_ci, Q->d_val, Q->d_rhs, o, nullptr);
    if (rc) return rc;
    Q->sys->opts.block_ptr = nullptr;
    Q->sys->opts.perm = nullptr;
    Q->batch.reset(new Batch);
    std::vector<System *> mem{Q->sys.get()};
    if ((rc = Q->batch->build(*ctx, mem))) return rc;
  }
  const int64_t h = ++ctx->next_handle;
  std::lock_guard<std::mutex> lk2(g_poi_mu);
  g_poi[ctx][h] = std::move(Q);
  *handle = h;
  return VSHE_OK;
}

int vshe_poisson_update(vshe_ctx *ctx, int64_t h, const double *potential, const double *n, const double *p, double damping,
                        double *potential_out, vshe_poisson_stats *stats) {
  if (!ctx || !potential || !n || !p || !potential_out || !(damping > 0.0 && damping <= 1.0)) return VSHE_E_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lk(ctx->mu);
  cudaSetDevice(ctx->device);
  PoissonProblem *Q = find_poisson(ctx, h);
  if (!Q) return ctx->fail(VSHE_E_NOT_FOUND, "");
  const size_t nc = size_t(Q->nc);
  for (size_t c = 0; c < nc; ++c)
    if (!std::isfinite(potential[c]) || !std::isfinite(n[c]) || !std::isfinite(p[c])) return ctx->fail(VSHE_E_NAN, "cell " + std::to_string(c));
  cudaStream_t s = ctx->stream;
  cudaError_t e;
  if ((e = cudaMemcpyAsync(Q->d_psi, potential, sizeof(double) * nc, cudaMemcpyHostToDevice, s)) != cudaSuccess ||
      (e = cudaMemcpyAsync(Q->d_n, n, sizeof(double) * nc, cudaMemcpyHostToDevice, s)) != cudaSuccess ||
      (e = cudaMemcpyAsync(Q->d_p, p, sizeof(double) * nc, cudaMemcpyHostToDevice, s)) != cudaSuccess)
    return ctx->cuda_fail(e, "poisson upload");
  int rc = vk_poisson_assemble(&Q->P, Q->d_psi, Q->d_n, Q->d_p, Q->d_val, Q->d_rhs, s);
  if (rc) return ctx->cuda_fail(cudaError_t(rc), "poisson assemble");
  Q->assembled = true;
  vshe_poisson_stats st{};
  st.n_unknowns = Q->nu;
  const double *dpsi = nullptr;
  std::vector<double> b((size_t)Q->nu), x((size_t)Q->nu);
  if (Q->nu > 0) {
    std::vector<vshe_solve_stats> ss;
    if ((rc = Q->batch->solve(*ctx, ss))) return rc;
    st.status = ss[0].status;
    st.iterations = ss[0].iterations;
    st.rel_residual = ss[0].rel_residual;
    dpsi = Q->sys->d_x64;
    if ((e = cudaMemcpyAsync(b.data(), Q->d_rhs, sizeof(double) * b.size(), cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
        (e = cudaMemcpyAsync(x.data(), dpsi, sizeof(double) * x.size(), cudaMemcpyDeviceToHost, s)) != cudaSuccess)
      return ctx->cuda_fail(e, "poisson download");
  }
  rc = vk_poisson_update(&Q->P, Q->d_psi, dpsi ? dpsi : Q->d_rhs, damping, Q->d_out, s);
  if (rc) return ctx->cuda_fail(cudaError_t(rc), "poisson update");
  if ((e = cudaMemcpyAsync(potential_out, Q->d_out, sizeof(double) * nc, cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
      (e = cudaStreamSynchronize(s)) != cudaSuccess)
    return ctx->cuda_fail(e, "poisson download");
  double bn = 0.0, xn = 0.0;
  for (size_t i = 0; i < b.size(); ++i) { bn += b[i] * b[i]; xn += x[i] * x[i]; }
  st.rhs_norm = std::sqrt(bn);
  st.update_norm = std::sqrt(xn);
  if (stats) *stats = st;
  if (st.status) return ctx->fail(st.status, "poisson solve");
  return VSHE_OK;
}

int vshe_poisson_export(vshe_ctx *ctx, int64_t h, int64_t *row_ptr, int32_t *col, double *val, double *rhs, int64_t *nnz) {
  if (!ctx) return VSHE_E_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lk(ctx->mu);
  cudaSetDevice(ctx->device);
  PoissonProblem *Q = find_poisson(ctx, h);
  if (!Q) return ctx->fail(VSHE_E_NOT_FOUND, "");
  if (nnz) *nnz = Q->nnz;
  if (row_ptr) std::memcpy(row_ptr, Q->rp.data(), sizeof(int64_t) * Q->rp.size());
  if (col) std::memcpy(col, Q->ci.data(), sizeof(int32_t) * Q->ci.size());
  if ((val || rhs) && !Q->assembled) return ctx->fail(VSHE_E_INVALID_ARGUMENT, "not assembled yet");
  cudaError_t e = cudaSuccess;
  if (val && Q->nnz) e = cudaMemcpyAsync(val, Q->d_val, sizeof(double) * size_t(Q->nnz), cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess && rhs && Q->nu) e = cudaMemcpyAsync(rhs, Q->d_rhs, sizeof(double) * size_t(Q->nu), cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) return ctx->cuda_fail(e, "poisson export");
  return VSHE_OK;
}

int vshe_poisson_free(vshe_ctx *ctx, int64_t h) {
  if (!ctx) return VSHE_E_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lk(ctx->mu);
  cudaSetDevice(ctx->device);
  std::lock_guard<std::mutex> lk2(g_poi_mu);
  auto it = g_poi.find(ctx);
  if (it == g_poi.end() || !it->second.count(h)) return ctx->fail(VSHE_E_NOT_FOUND, "");
  it->second.erase(h);
  return VSHE_OK;
}

}  // extern "C"

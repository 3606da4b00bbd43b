// she_pipeline.cpp -- C++ host orchestration of the device-side SHE path:
// setup on the host (she_host.cpp), then on the GPU: assembly (K1/K2),
// odd elimination (K3), unknown scaling + row/column normalisation (K4),
// ILU(0)/BiCGStab solve of the reduced system (host_solver.cpp), and
// recovery + post-processing (K10).  Implements the vshe_she_* C ABI.
//
// Mirrors viennashe::she::assemble (viennashe/she/assemble_all.hpp:46-424) followed by
// viennashe::she::solve (viennashe/she/linear_solver.hpp:100-189).

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
#include "she_host.h"
#include "she_kernels.h"

namespace vshe {

struct SheProblem {
  SheSetup H;
  DevArena arena;
  SheDev P{};
  vshe_solve_opts opts{};
  int ncontacts = 0;
  // full (even + odd) system
  int64_t n_full = 0, nnz_full = 0;
  int64_t *d_frp = nullptr; int32_t *d_fci = nullptr; double *d_fval = nullptr, *d_frhs = nullptr;
  // reduced system
  int64_t n_red = 0, nnz_red = 0;
  int64_t *d_rrp = nullptr; int32_t *d_rci = nullptr; double *d_rval = nullptr, *d_rrhs = nullptr;
  uint8_t *d_ins = nullptr;
  double *d_s = nullptr, *d_sf = nullptr;
  int64_t *d_dpos = nullptr, *d_cptr = nullptr, *d_cursor = nullptr, *d_cpos = nullptr;
  void *d_tmp = nullptr; size_t tmp_bytes = 0;
  int32_t *d_err = nullptr;
  // outputs
  double *d_xf = nullptr, *d_dens = nullptr, *d_cur = nullptr, *d_part = nullptr;
  std::vector<int64_t> slab_ptr;
  std::unique_ptr<System> sys;
  std::unique_ptr<Batch> batch;
  // between create_device_pattern and create_device_finish: the solver options with the node
  // colouring and slab bounds they point at, the values ILUT's pattern needs, the layout
  vshe_solve_opts so_{};
  std::vector<int32_t> node_perm_;
  std::vector<double> hval_;
  std::unique_ptr<Layout> layout_;
  int layout_rc_ = 0;
  std::string layout_err_;
  double full_residual = -1.0;
  int stage = 0;

  int create(Ctx &ctx, const vshe_device_desc &d, const vshe_she_config &c, const vshe_coupling_tables &ct, const vshe_solve_opts &o);
  int setup_host(Ctx &ctx, const vshe_device_desc &d, const vshe_she_config &c, const vshe_coupling_tables &ct, const vshe_solve_opts &o);
  size_t estimate_bytes() const;
  int create_device(Ctx &ctx);  // = create_device_pattern, build_layout, create_device_finish
  int create_device_pattern(Ctx &ctx);
  void build_layout();
  int create_device_finish(Ctx &ctx);
  int symbolic_full(Ctx &ctx);
  int fill_full(Ctx &ctx);
  int assemble(Ctx &ctx, int upto);
  int finish(Ctx &ctx);
  int check(Ctx &ctx, const char *what);
};

template <typename T>
static T *upload(Ctx &ctx, DevArena &ar, const std::vector<T> &v, int &rc) {
  cudaError_t e;
  T *p = (T *)ar.alloc(sizeof(T) * std::max<size_t>(v.size(), 1), e);
  if (!p) { rc = ctx.cuda_fail(e, "cudaMalloc she table"); return nullptr; }
  if (!v.empty() && (e = cudaMemcpyAsync(p, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice, ctx.stream)) != cudaSuccess) {
    rc = ctx.cuda_fail(e, "upload she table");
    return nullptr;
  }
  rc = 0;
  return p;
}

int SheProblem::check(Ctx &ctx, const char *what) {
  int32_t err = 0;
  cudaError_t e = cudaMemcpyAsync(&err, d_err, sizeof(int32_t), cudaMemcpyDeviceToHost, ctx.stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx.stream);
  if (e != cudaSuccess) return ctx.cuda_fail(e, what);
  if (err) {
    cudaMemsetAsync(d_err, 0, sizeof(int32_t), ctx.stream);
    if (err == -100) return -100;
    if (err == -4) return ctx.fail(VSHE_E_ODD_DIAGONAL, what);
    return ctx.fail(VSHE_E_INVALID_ARGUMENT, std::string(what) + ": per-row capacity exceeded");
  }
  return VSHE_OK;
}

int SheProblem::create(Ctx &ctx, const vshe_device_desc &d, const vshe_she_config &c, const vshe_coupling_tables &ct, const vshe_solve_opts &o) {
  int rc = setup_host(ctx, d, c, ct, o);
  if (rc) return rc;
  return create_device(ctx);
}

// The host part of the set-up (energies, orders, mapping, boundary values): no device work.
int SheProblem::setup_host(Ctx &ctx, const vshe_device_desc &d, const vshe_she_config &c, const vshe_coupling_tables &ct, const vshe_solve_opts &o) {
  std::string msg = H.build(d, c, ct);
  if (!msg.empty()) return ctx.fail(VSHE_E_INVALID_ARGUMENT, msg);
  opts = o;
  for (int i = 0; i < H.nc; ++i) ncontacts = std::max(ncontacts, H.contact[i] + 1);
  return VSHE_OK;
}

// Upper bound of the device memory the problem will hold, from the host set-up alone, so that
// admission against an HBM budget happens before any allocation.  Row lengths are bounded by the
// mesh and the harmonics per node: a full-system even row holds its diagonal, two optical
// in-scattering entries and at most o(L) odd couplings per facet of its cell (at most f facets,
// the mesh's largest cell; 2 dim on the structured meshes); an odd row its diagonal and at most
// e(L) couplings to each of its two cells; a reduced row its diagonal, the in-scattering pair and
// at most e(L) columns for its cell and each neighbour.  The
// factor keeps at most (1 + k) times the reduced pattern for ILU(k), and 2 p + 1 entries per row
// more for ILUT(p).  Per entry and per row, the bytes of every buffer the pipeline, the solver
// (SELL copies of A, L and U, factorisation CSR and maps, Krylov vectors) and the batch hold.
size_t SheProblem::estimate_bytes() const {
  int64_t e = 0;
  for (int l = 0; l <= H.L; l += 2) e += 2 * l + 1;
  const int64_t o = int64_t(H.L + 1) * (H.L + 1) - e;
  const int64_t ne = H.n_even, no = H.n_odd, nfull = ne + no;
  int64_t f = 2 * H.dim;
  for (int c = 0; c < H.nc; ++c) f = std::max<int64_t>(f, H.cf_ptr[size_t(c) + 1] - H.cf_ptr[size_t(c)]);
  const int64_t nnz_full = ne * (3 + f * o) + no * (1 + 2 * e);
  const int64_t nnz_red = ne * (3 + (1 + f) * e);
  const int64_t nnz_f = opts.precond == VSHE_PRECOND_ILUT
                            ? nnz_red + ne * (2 * int64_t(opts.ilut_entries > 0 ? opts.ilut_entries : 60) + 1)
                            : nnz_red * (1 + std::max(0, int(opts.fill_level)));
  const int64_t tsz = opts.precision == VSHE_PRECISION_MIXED ? 4 : 8;
  const int64_t tables = (int64_t(H.nc) + H.nf) * H.NH * 48 + int64_t(H.nc + H.nf) * 256 + (int64_t(1) << 20);
  const int64_t pipeline = nnz_full * 12 + nfull * 40 + nnz_red * 20 + ne * 72;
  const int64_t solver = nnz_red * 24 + nnz_f * (32 + 2 * (4 + tsz)) + ne * (11 * 8 + 48 + tsz);
  const int64_t batch = (ne / 256 + 64) * 64 + (int64_t(1) << 20);
  return size_t(tables + pipeline + (solver * 11) / 10 + batch);
}

int SheProblem::create_device(Ctx &ctx) {
  int rc = create_device_pattern(ctx);
  if (rc) return rc;
  build_layout();
  return create_device_finish(ctx);
}

// Device set-up up to the reduced system's pattern on the host (the system's host copies).
int SheProblem::create_device_pattern(Ctx &ctx) {
  int rc = 0;
  cudaError_t e;
#define UP(dst, vec) dst = upload(ctx, arena, vec, rc); if (rc) return rc;
  P.dim = H.dim; P.nc = H.nc; P.nf = H.nf; P.NH = H.NH; P.D = H.D; P.L = H.L; P.T = H.T;
  const int32_t *i32; const double *f64; const int64_t *i64; const char *ch;
  UP(i32, H.mat); P.mat = i32;
  UP(i32, H.contact); P.contact = i32;
  UP(i32, H.cf_ptr); P.cf_ptr = i32;
  UP(i32, H.cf_idx); P.cf_idx = i32;
  UP(i32, H.inc_dir_even); P.inc_dir_even = i32;
  UP(f64, H.vol); P.vol = f64;
  UP(f64, H.cen); P.cen = f64;
  UP(f64, H.shift_c); P.shift_c = f64;
  UP(ch, H.mask_c); P.mask_c = ch;
  UP(i32, H.fcell); P.fcell = i32;
  UP(i32, H.inc_dir_odd); P.inc_dir_odd = i32;
  UP(f64, H.fvol); P.fvol = f64;
  UP(f64, H.fnorm); P.fnorm = f64;
  UP(f64, H.shift_f); P.shift_f = f64;
  UP(f64, H.Hval); P.Hval = f64;
  UP(f64, H.bnd_c); P.bnd_c = f64;
  UP(i32, H.ord_c); P.ord_c = i32;
  UP(i32, H.ord_f); P.ord_f = i32;
  UP(i64, H.idx_c); P.idx_c = i64;
  UP(i64, H.idx_f); P.idx_f = i64;
  UP(i32, H.even_nodes); P.even_nodes = i32;
  UP(i32, H.odd_nodes); P.odd_nodes = i32;
  UP(i32, H.even_harm); P.even_harm = i32;
  UP(i32, H.odd_harm); P.odd_harm = i32;
  UP(f64, H.cblocks); P.cblocks = f64;
#undef UP
  P.n_even_nodes = int64_t(H.even_nodes.size() / 2);
  P.n_odd_nodes = int64_t(H.odd_nodes.size() / 2);
  P.n_even = H.n_even; P.n_odd = H.n_odd;
  P.acoustic = H.cfg.acoustic_phonon; P.optical = H.cfg.optical_phonon;
  P.bnd_type = H.cfg.boundary_type == VSHE_BOUNDARY_DIRICHLET ? 1 : 0;
  P.scaling_type = H.cfg.scaling_type;
  P.tau = H.cfg.gr_tau;
  P.hbar_omega = H.hbar_omega;
  {
    // rates: acoustic_phonon_scattering.hpp:98-114, optical_phonon_scattering.hpp:162-179, physics.hpp:71-75
    const double PI = SheConst::PI, Q = SheConst::Q, KB = SheConst::KB;
    const double hbar = 6.62606896e-34 / (2.0 * 3.1415926535897932384626433832795);
    const double ul = 9040.0, rho = 2330.0, E1 = 8.9 * Q, DtK = 5e10 * Q;
    P.rate_ac = H.cfg.acoustic_fit_factor * (2.0 * PI * KB * H.T * E1 * E1 / (hbar * ul * ul * rho));
    P.rate_op = H.cfg.optical_fit_factor * (PI * DtK * DtK * hbar / (2.0 * rho * H.hbar_omega));
    P.n_op = 1.0 / (std::exp(H.hbar_omega / (KB * H.T)) - 1.0);
  }
  for (int j = 0; j < 3; ++j) { P.ax01[j] = H.a_x01[j]; P.ay01[j] = H.a_y01[j]; }
  n_full = H.n_even + H.n_odd;
  n_red = H.n_even;
  slab_ptr = H.slab_ptr;
#define ALLOC(ptr, type, count) \
  ptr = (type *)arena.alloc(sizeof(type) * size_t(count), e); if (!ptr) return ctx.cuda_fail(e, "cudaMalloc she " #ptr);
  ALLOC(d_err, int32_t, 1);
  ALLOC(d_frp, int64_t, n_full + 1);
  ALLOC(d_rrp, int64_t, n_red + 1);
  if ((e = cudaMemsetAsync(d_err, 0, sizeof(int32_t), ctx.stream)) != cudaSuccess) return ctx.cuda_fail(e, "memset");
  // scan scratch sized for the larger of the scans
  {
    size_t t1 = 0;
    vk_scan_rowptr(d_frp, n_full, nullptr, &t1, ctx.stream);
    tmp_bytes = std::max<size_t>(t1, 256) * 2;
    d_tmp = arena.alloc(tmp_bytes, e);
    if (!d_tmp) return ctx.cuda_fail(e, "cudaMalloc scan scratch");
  }
  rc = symbolic_full(ctx);
  if (rc) return rc;
  // reduced pattern: count pass of K3 needs the assembled full system
  rc = fill_full(ctx);
  if (rc) return rc;
  FullDev A{d_frp, d_fci, d_fval, d_frhs};
  if ((e = cudaMemsetAsync(d_rrp, 0, sizeof(int64_t), ctx.stream)) != cudaSuccess) return ctx.cuda_fail(e, "memset");
  if ((rc = vk_she_schur(&A, n_red, 0, d_rrp + 1, nullptr, nullptr, nullptr, nullptr, nullptr, d_err, ctx.stream))) return ctx.cuda_fail(cudaError_t(rc), "schur count");
  if ((rc = check(ctx, "eliminate_odd_unknowns (count)"))) return rc;
  {
    size_t tb = tmp_bytes;
    if ((rc = vk_scan_rowptr(d_rrp, n_red, d_tmp, &tb, ctx.stream))) return ctx.cuda_fail(cudaError_t(rc), "scan");
  }
  if ((e = cudaMemcpyAsync(&nnz_red, d_rrp + n_red, sizeof(int64_t), cudaMemcpyDeviceToHost, ctx.stream)) != cudaSuccess) return ctx.cuda_fail(e, "nnz");
  if ((e = cudaStreamSynchronize(ctx.stream)) != cudaSuccess) return ctx.cuda_fail(e, "nnz");
  if (nnz_red >= (int64_t(1) << 40)) return ctx.fail(VSHE_E_INVALID_ARGUMENT, "reduced system too large");
  ALLOC(d_rci, int32_t, nnz_red);
  ALLOC(d_rval, double, nnz_red);
  ALLOC(d_rrhs, double, n_red);
  ALLOC(d_ins, uint8_t, n_red);
  ALLOC(d_s, double, n_red);
  ALLOC(d_sf, double, n_red);
  ALLOC(d_dpos, int64_t, n_red);
  ALLOC(d_cptr, int64_t, n_red + 1);
  ALLOC(d_cursor, int64_t, n_red);
  ALLOC(d_cpos, int64_t, nnz_red);
  ALLOC(d_xf, double, n_full);
  ALLOC(d_dens, double, H.nc);
  ALLOC(d_cur, double, std::max(ncontacts, 1));
  ALLOC(d_part, double, 2 * size_t(vk_she_residual_blocks(n_full)));
#undef ALLOC
  {
    std::vector<double> ones((size_t)(n_red), 1.0);
    if ((e = cudaMemcpyAsync(d_s, ones.data(), sizeof(double) * ones.size(), cudaMemcpyHostToDevice, ctx.stream)) != cudaSuccess) return ctx.cuda_fail(e, "scaling");
    if ((e = cudaStreamSynchronize(ctx.stream)) != cudaSuccess) return ctx.cuda_fail(e, "scaling");
  }
  rc = assemble(ctx, 3);
  if (rc) return rc;
  // reduced pattern on the host for the preconditioner's schedules
  std::vector<int64_t> hrp((size_t)n_red + 1);
  std::vector<int32_t> hci((size_t)nnz_red);
  if ((e = cudaMemcpyAsync(hrp.data(), d_rrp, sizeof(int64_t) * hrp.size(), cudaMemcpyDeviceToHost, ctx.stream)) != cudaSuccess) return ctx.cuda_fail(e, "pattern");
  if ((e = cudaMemcpyAsync(hci.data(), d_rci, sizeof(int32_t) * hci.size(), cudaMemcpyDeviceToHost, ctx.stream)) != cudaSuccess) return ctx.cuda_fail(e, "pattern");
  if ((e = cudaStreamSynchronize(ctx.stream)) != cudaSuccess) return ctx.cuda_fail(e, "pattern");
  vshe_solve_opts &so = so_;
  so = opts;
  std::vector<int32_t> &node_perm = node_perm_;
  if (so.ordering == VSHE_ORDER_MULTICOLOR && !so.perm && so.precond != VSHE_PRECOND_NONE) {
    node_colour_order(H, so.fill_level, node_perm, nullptr);
    so.perm = node_perm.data();
  }
  if (so.precond == VSHE_PRECOND_BLOCK_ILU0 && (so.n_blocks <= 0 || !so.block_ptr)) {
    // energy slabs (fill_block_indices, linear_solver.hpp:44-83): one block per H with unknowns
    so.n_blocks = int64_t(slab_ptr.size()) - 1;
    so.block_ptr = slab_ptr.data();
  }
  std::vector<double> &hval = hval_;
  if (so.precond == VSHE_PRECOND_ILUT) {
    // the ILUT pattern is found from the values of this first assembly
    hval.resize((size_t)nnz_red);
    if ((e = cudaMemcpyAsync(hval.data(), d_rval, sizeof(double) * hval.size(), cudaMemcpyDeviceToHost, ctx.stream)) != cudaSuccess) return ctx.cuda_fail(e, "values");
    if ((e = cudaStreamSynchronize(ctx.stream)) != cudaSuccess) return ctx.cuda_fail(e, "values");
  }
  sys.reset(new System);
  return sys->init_borrowed(ctx, n_red, nnz_red, hrp.data(), hci.data(), d_rrp, d_rci, d_rval, d_rrhs, so);
}

// The solver layout of the reduced system (ordering, ILU(k) or ILUT pattern, level schedules,
// SELL tables) from its host pattern: host work only, no device or context call, so it may run
// on another thread while the context serves other work.
void SheProblem::build_layout() {
  layout_.reset(new Layout);
  layout_rc_ = layout_->build(sys->n, sys->nnz, sys->rp, sys->ci, sys->opts, hval_.empty() ? nullptr : hval_.data(), layout_err_);
}

// Device buffers of the reduced system from the layout, and the problem's own batch.
int SheProblem::create_device_finish(Ctx &ctx) {
  if (!layout_) return ctx.fail(VSHE_E_INVALID_ARGUMENT, "layout not built");
  int rc = layout_rc_ ? ctx.fail(layout_rc_, layout_err_) : sys->setup_from_layout(ctx, *layout_);
  layout_.reset();
  std::vector<double>().swap(hval_);
  if (rc) return rc;
  sys->opts.block_ptr = nullptr;  // the pointers above are only read during creation
  sys->opts.perm = nullptr;
  std::vector<int32_t>().swap(node_perm_);
  batch.reset(new Batch);
  std::vector<System *> mem{sys.get()};
  return batch->build(ctx, mem);
}

int SheProblem::symbolic_full(Ctx &ctx) {
  cudaError_t e;
  int rc;
  if ((e = cudaMemsetAsync(d_frp, 0, sizeof(int64_t), ctx.stream)) != cudaSuccess) return ctx.cuda_fail(e, "memset");
  if ((rc = vk_she_assemble_even(&P, 0, d_frp + 1, nullptr, nullptr, nullptr, nullptr, d_err, ctx.stream))) return ctx.cuda_fail(cudaError_t(rc), "assemble even (count)");
  if ((rc = vk_she_assemble_odd(&P, 0, d_frp + 1, nullptr, nullptr, nullptr, nullptr, d_err, ctx.stream))) return ctx.cuda_fail(cudaError_t(rc), "assemble odd (count)");
  size_t tb = tmp_bytes;
  if ((rc = vk_scan_rowptr(d_frp, n_full, d_tmp, &tb, ctx.stream))) return ctx.cuda_fail(cudaError_t(rc), "scan");
  if ((e = cudaMemcpyAsync(&nnz_full, d_frp + n_full, sizeof(int64_t), cudaMemcpyDeviceToHost, ctx.stream)) != cudaSuccess) return ctx.cuda_fail(e, "nnz");
  if ((rc = check(ctx, "assemble (count)"))) return rc;
  if (d_fci) return ctx.fail(VSHE_E_INVALID_ARGUMENT, "full pattern already allocated");
  d_fci = (int32_t *)arena.alloc(sizeof(int32_t) * size_t(nnz_full), e);
  if (!d_fci) return ctx.cuda_fail(e, "cudaMalloc full ci");
  d_fval = (double *)arena.alloc(sizeof(double) * size_t(nnz_full), e);
  if (!d_fval) return ctx.cuda_fail(e, "cudaMalloc full val");
  d_frhs = (double *)arena.alloc(sizeof(double) * size_t(n_full), e);
  if (!d_frhs) return ctx.cuda_fail(e, "cudaMalloc full rhs");
  return VSHE_OK;
}

int SheProblem::fill_full(Ctx &ctx) {
  int rc;
  if ((rc = vk_she_assemble_even(&P, 1, nullptr, d_frp, d_fci, d_fval, d_frhs, d_err, ctx.stream))) return ctx.cuda_fail(cudaError_t(rc), "assemble even");
  if ((rc = vk_she_assemble_odd(&P, 1, nullptr, d_frp, d_fci, d_fval, d_frhs, d_err, ctx.stream))) return ctx.cuda_fail(cudaError_t(rc), "assemble odd");
  rc = check(ctx, "assemble");
  if (rc == -100) return ctx.fail(VSHE_E_INVALID_ARGUMENT, "the assembled pattern changed (an entry cancelled to zero); recreate the problem");
  return rc;
}

// upto: 1 = assemble the full system, 2 = + eliminate odd unknowns, 3 = + scaling/normalisation
int SheProblem::assemble(Ctx &ctx, int upto) {
  int rc;
  if (stage > 0 || upto >= 1) {
    if ((rc = fill_full(ctx))) return rc;
  }
  stage = 1;
  if (upto < 2) return VSHE_OK;
  FullDev A{d_frp, d_fci, d_fval, d_frhs};
  if ((rc = vk_she_schur(&A, n_red, 1, nullptr, d_rrp, d_rci, d_rval, d_rrhs, d_ins, d_err, ctx.stream))) return ctx.cuda_fail(cudaError_t(rc), "schur");
  rc = check(ctx, "eliminate_odd_unknowns");
  if (rc == -100) return ctx.fail(VSHE_E_INVALID_ARGUMENT, "reduced pattern changed; recreate the problem");
  if (rc) return rc;
  stage = 2;
  if (upto < 3) return VSHE_OK;
  if ((rc = vk_she_normalise(&P, n_red, d_rrp, d_rci, d_rval, d_rrhs, d_ins, H.cfg.scale ? 1 : 0, d_s, d_sf, d_dpos, d_cptr, d_cursor, d_cpos, d_tmp, tmp_bytes, ctx.stream)))
    return ctx.cuda_fail(cudaError_t(rc), "normalise");
  stage = 3;
  return VSHE_OK;
}

int SheProblem::finish(Ctx &ctx) {
  FullDev A{d_frp, d_fci, d_fval, d_frhs};
  int rc = vk_she_finish(&P, &A, sys->d_x64, d_s, d_sf, H.cfg.scale ? 1 : 0, d_xf, d_part, d_dens, ncontacts, d_cur, ctx.stream);
  if (rc) return ctx.cuda_fail(cudaError_t(rc), "finish");
  const int nb = vk_she_residual_blocks(n_full);
  std::vector<double> part(2 * size_t(nb));
  cudaError_t e = cudaMemcpyAsync(part.data(), d_part, sizeof(double) * part.size(), cudaMemcpyDeviceToHost, ctx.stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx.stream);
  if (e != cudaSuccess) return ctx.cuda_fail(e, "finish");
  double r2 = 0, b2 = 0;
  for (int k = 0; k < nb; ++k) { r2 += part[2 * size_t(k)]; b2 += part[2 * size_t(k) + 1]; }
  full_residual = b2 > 0 ? std::sqrt(r2) / std::sqrt(b2) : 0.0;
  return VSHE_OK;
}

}  // namespace vshe

using namespace vshe;

static std::map<vshe::Ctx *, std::map<int64_t, std::unique_ptr<SheProblem>>> g_she;
// batch schedules of vshe_she_run_batch, per context and handle set
static std::map<vshe::Ctx *, std::map<std::vector<int64_t>, std::unique_ptr<Batch>>> g_she_batches;
static std::mutex g_she_mu;

static size_t problem_bytes(const SheProblem *S) {
  size_t b = S->arena.total;
  if (S->sys) b += S->sys->arena.total;
  if (S->batch) b += S->batch->arena.total + S->batch->tile_arena.total;
  return b;
}

size_t vshe::she_bytes(Ctx *ctx) {
  std::lock_guard<std::mutex> lk(g_she_mu);
  size_t t = 0;
  auto it = g_she.find(ctx);
  if (it != g_she.end())
    for (auto &kv : it->second) t += problem_bytes(kv.second.get());
  return t;
}

static SheProblem *find_she(vshe_ctx *ctx, int64_t h) {
  std::lock_guard<std::mutex> lk(g_she_mu);
  auto it = g_she.find(ctx);
  if (it == g_she.end()) return nullptr;
  auto jt = it->second.find(h);
  return jt == it->second.end() ? nullptr : jt->second.get();
}

namespace vshe {
void she_release_all(Ctx *ctx) {
  std::lock_guard<std::mutex> lk(g_she_mu);
  g_she_batches.erase(ctx);
  g_she.erase(ctx);
}
}  // namespace vshe

extern "C" {

int vshe_coupling_tables_compute(int32_t L, double *out) {
  if (L < 1 || L > 9 || !out) return VSHE_E_INVALID_ARGUMENT;
  vshe::coupling_quadrature(L, out);
  return VSHE_OK;
}

int vshe_she_create(vshe_ctx *ctx, const vshe_device_desc *d, const vshe_she_config *c, const vshe_coupling_tables *ct,
                    const vshe_solve_opts *opts, int64_t *handle) {
  if (!ctx || !d || !c || !ct || !handle) return VSHE_E_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lk(ctx->mu);
  cudaSetDevice(ctx->device);
  vshe_solve_opts o;
  if (opts) o = *opts; else vshe_default_opts(&o);
  std::unique_ptr<SheProblem> S(new SheProblem);
  int rc = S->setup_host(*ctx, *d, *c, *ct, o);
  if (rc) return rc;
  // admission against the context's HBM budget before any allocation
  const size_t est = S->estimate_bytes();
  if (vshe_bytes_in_use(ctx) + est > ctx->budget) return ctx->fail(VSHE_E_BUDGET, std::to_string(est) + " bytes (upper bound) requested");
  rc = S->create_device(*ctx);
  if (rc) return rc;
  int64_t h = ++ctx->next_handle;
  std::lock_guard<std::mutex> lk2(g_she_mu);
  g_she[ctx][h] = std::move(S);
  *handle = h;
  return VSHE_OK;
}

int vshe_she_plan(const vshe_device_desc *d, const vshe_she_config *c, const vshe_coupling_tables *ct,
                  const vshe_solve_opts *opts, vshe_she_info *info) {
  if (!d || !c || !ct || !info) return VSHE_E_INVALID_ARGUMENT;
  SheProblem S;
  if (opts) S.opts = *opts; else vshe_default_opts(&S.opts);
  if (!S.H.build(*d, *c, *ct).empty()) return VSHE_E_INVALID_ARGUMENT;
  std::memset(info, 0, sizeof(*info));
  int ncont = 0;
  for (int i = 0; i < S.H.nc; ++i) ncont = std::max(ncont, S.H.contact[i] + 1);
  info->n_energies = S.H.NH;
  info->n_even = S.H.n_even;
  info->n_odd = S.H.n_odd;
  info->n_cells = S.H.nc;
  info->n_facets = S.H.nf;
  info->n_contacts = ncont;
  info->hbar_omega = S.H.hbar_omega;
  info->bytes_estimate = int64_t(S.estimate_bytes());
  return VSHE_OK;
}

int vshe_she_space(const vshe_device_desc *d, const vshe_she_config *c, const vshe_coupling_tables *ct, double *energies,
                   int64_t *even_index, int32_t *even_order, double *kinetic_energy, double *density_of_states,
                   int64_t *odd_index, int32_t *odd_order) {
  if (!d || !c || !ct) return VSHE_E_INVALID_ARGUMENT;
  SheSetup H;
  if (!H.build(*d, *c, *ct).empty()) return VSHE_E_INVALID_ARGUMENT;
  const size_t nh = size_t(H.NH), cells = size_t(H.nc) * nh, facets = size_t(H.nf) * nh;
  if (energies) std::copy(H.Hval.begin(), H.Hval.end(), energies);
  if (even_index) std::copy(H.idx_c.begin(), H.idx_c.begin() + cells, even_index);
  if (even_order) std::copy(H.ord_c.begin(), H.ord_c.begin() + cells, even_order);
  if (odd_index) std::copy(H.idx_f.begin(), H.idx_f.begin() + facets, odd_index);
  if (odd_order) std::copy(H.ord_f.begin(), H.ord_f.begin() + facets, odd_order);
  for (int i = 0; i < H.nc; ++i)
    for (int h = 0; h < H.NH; ++h) {
      const double eps = H.ekin_c(i, h);
      if (kinetic_energy) kinetic_energy[size_t(i) * nh + size_t(h)] = eps;
      if (density_of_states) density_of_states[size_t(i) * nh + size_t(h)] = vshe::density_of_states(eps);
    }
  return VSHE_OK;
}

int vshe_she_node_order(const vshe_device_desc *d, const vshe_she_config *c, const vshe_coupling_tables *ct, int32_t fill_level,
                        int32_t *perm, int32_t *colour) {
  if (!d || !c || !ct || fill_level < 0) return VSHE_E_INVALID_ARGUMENT;
  SheSetup H;
  if (!H.build(*d, *c, *ct).empty()) return VSHE_E_INVALID_ARGUMENT;
  std::vector<int32_t> p, col;
  node_colour_order(H, fill_level, p, &col);
  if (perm) std::copy(p.begin(), p.end(), perm);
  if (colour) std::copy(col.begin(), col.end(), colour);
  return VSHE_OK;
}

int vshe_she_info_get(vshe_ctx *ctx, int64_t h, vshe_she_info *info) {
  if (!ctx || !info) return VSHE_E_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lk(ctx->mu);
  SheProblem *S = find_she(ctx, h);
  if (!S) return ctx->fail(VSHE_E_NOT_FOUND, "");
  info->n_energies = S->H.NH;
  info->n_even = S->H.n_even;
  info->n_odd = S->H.n_odd;
  info->nnz_full = S->nnz_full;
  info->nnz_reduced = S->nnz_red;
  info->n_cells = S->H.nc;
  info->n_facets = S->H.nf;
  info->n_contacts = S->ncontacts;
  info->hbar_omega = S->H.hbar_omega;
  info->bytes_device = int64_t(S->arena.total + (S->sys ? S->sys->arena.total : 0) + (S->batch ? S->batch->arena.total + S->batch->tile_arena.total : 0));
  info->levels_L = S->sys ? S->sys->nlevL : 0;
  info->levels_U = S->sys ? S->sys->nlevU : 0;
  info->nnz_factor = S->sys ? S->sys->nnzL + S->sys->nnzU : 0;
  info->bytes_estimate = int64_t(S->estimate_bytes());
  return VSHE_OK;
}

int vshe_she_assemble(vshe_ctx *ctx, int64_t h, int32_t upto) {
  if (!ctx) return VSHE_E_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lk(ctx->mu);
  cudaSetDevice(ctx->device);
  SheProblem *S = find_she(ctx, h);
  if (!S) return ctx->fail(VSHE_E_NOT_FOUND, "");
  if (upto < 1 || upto > 3) return ctx->fail(VSHE_E_INVALID_ARGUMENT, "upto must be 1, 2 or 3");
  return S->assemble(*ctx, upto);
}

int vshe_she_solve(vshe_ctx *ctx, int64_t h, vshe_solve_stats *stats) {
  if (!ctx) return VSHE_E_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lk(ctx->mu);
  cudaSetDevice(ctx->device);
  SheProblem *S = find_she(ctx, h);
  if (!S) return ctx->fail(VSHE_E_NOT_FOUND, "");
  if (S->stage < 3) return ctx->fail(VSHE_E_INVALID_ARGUMENT, "assemble the system first");
  std::vector<vshe_solve_stats> st;
  int rc = S->batch->solve(*ctx, st);
  if (rc) return rc;
  if (stats) *stats = st[0];
  if (st[0].status) return ctx->fail(st[0].status, "");
  return VSHE_OK;
}

int vshe_she_finish(vshe_ctx *ctx, int64_t h, double *full_residual) {
  if (!ctx) return VSHE_E_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lk(ctx->mu);
  cudaSetDevice(ctx->device);
  SheProblem *S = find_she(ctx, h);
  if (!S) return ctx->fail(VSHE_E_NOT_FOUND, "");
  int rc = S->finish(*ctx);
  if (rc) return rc;
  if (full_residual) *full_residual = S->full_residual;
  return VSHE_OK;
}

int vshe_she_run(vshe_ctx *ctx, int64_t h, vshe_solve_stats *stats, double *full_residual) {
  int rc = vshe_she_assemble(ctx, h, 3);
  if (rc) return rc;
  rc = vshe_she_solve(ctx, h, stats);
  if (rc && rc != VSHE_E_NOT_CONVERGED) return rc;
  int rc2 = vshe_she_finish(ctx, h, full_residual);
  return rc ? rc : rc2;
}

int vshe_she_bench(vshe_ctx *ctx, int64_t h, int32_t warmup, int32_t steps, double *step_ms, vshe_solve_stats *last) {
  if (!ctx || steps <= 0 || !step_ms) return VSHE_E_INVALID_ARGUMENT;
  cudaSetDevice(ctx->device);
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  int rc = VSHE_OK;
  for (int k = 0; k < warmup + steps && rc == VSHE_OK; ++k) {
    cudaDeviceSynchronize();
    cudaEventRecord(a, ctx->stream);
    vshe_solve_stats st;
    double fr = 0;
    rc = vshe_she_run(ctx, h, &st, &fr);
    cudaEventRecord(b, ctx->stream);
    cudaEventSynchronize(b);
    cudaDeviceSynchronize();
    float ms = 0;
    cudaEventElapsedTime(&ms, a, b);
    if (k >= warmup) step_ms[k - warmup] = ms;
    if (last) *last = st;
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  return rc;
}

int vshe_she_results(vshe_ctx *ctx, int64_t h, double *x_full, double *density, double *currents) {
  if (!ctx) return VSHE_E_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lk(ctx->mu);
  cudaSetDevice(ctx->device);
  SheProblem *S = find_she(ctx, h);
  if (!S) return ctx->fail(VSHE_E_NOT_FOUND, "");
  cudaError_t e = cudaSuccess;
  if (x_full) e = cudaMemcpyAsync(x_full, S->d_xf, sizeof(double) * size_t(S->n_full), cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess && density) e = cudaMemcpyAsync(density, S->d_dens, sizeof(double) * size_t(S->H.nc), cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess && currents && S->ncontacts > 0) e = cudaMemcpyAsync(currents, S->d_cur, sizeof(double) * size_t(S->ncontacts), cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) return ctx->cuda_fail(e, "download results");
  return VSHE_OK;
}

int vshe_she_export(vshe_ctx *ctx, int64_t h, int32_t which, int64_t *rp, int32_t *ci, double *val, double *rhs) {
  if (!ctx) return VSHE_E_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lk(ctx->mu);
  cudaSetDevice(ctx->device);
  SheProblem *S = find_she(ctx, h);
  if (!S) return ctx->fail(VSHE_E_NOT_FOUND, "");
  const bool full = which == 0;
  const int64_t n = full ? S->n_full : S->n_red, nnz = full ? S->nnz_full : S->nnz_red;
  const int64_t *drp = full ? S->d_frp : S->d_rrp;
  const int32_t *dci = full ? S->d_fci : S->d_rci;
  const double *dv = full ? S->d_fval : S->d_rval, *db = full ? S->d_frhs : S->d_rrhs;
  cudaError_t e = cudaSuccess;
  if (rp) e = cudaMemcpyAsync(rp, drp, sizeof(int64_t) * size_t(n + 1), cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess && ci) e = cudaMemcpyAsync(ci, dci, sizeof(int32_t) * size_t(nnz), cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess && val) e = cudaMemcpyAsync(val, dv, sizeof(double) * size_t(nnz), cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess && rhs) e = cudaMemcpyAsync(rhs, db, sizeof(double) * size_t(n), cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) return ctx->cuda_fail(e, "export");
  return VSHE_OK;
}

int vshe_she_scaling(vshe_ctx *ctx, int64_t h, double *scaling, double *scale_factors) {
  if (!ctx) return VSHE_E_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lk(ctx->mu);
  SheProblem *S = find_she(ctx, h);
  if (!S) return ctx->fail(VSHE_E_NOT_FOUND, "");
  cudaError_t e = cudaSuccess;
  if (scaling) e = cudaMemcpyAsync(scaling, S->d_s, sizeof(double) * size_t(S->n_red), cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess && scale_factors) e = cudaMemcpyAsync(scale_factors, S->d_sf, sizeof(double) * size_t(S->n_red), cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) return ctx->cuda_fail(e, "download scaling");
  return VSHE_OK;
}

int vshe_she_blocks(vshe_ctx *ctx, int64_t h, int64_t *block_ptr) {
  if (!ctx || !block_ptr) return VSHE_E_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lk(ctx->mu);
  SheProblem *S = find_she(ctx, h);
  if (!S) return ctx->fail(VSHE_E_NOT_FOUND, "");
  std::copy(S->slab_ptr.begin(), S->slab_ptr.end(), block_ptr);
  return VSHE_OK;
}

int vshe_she_free(vshe_ctx *ctx, int64_t h) {
  if (!ctx) return VSHE_E_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lk(ctx->mu);
  cudaSetDevice(ctx->device);
  cudaStreamSynchronize(ctx->stream);
  std::unique_ptr<SheProblem> dead;
  {
    std::lock_guard<std::mutex> lk2(g_she_mu);
    auto it = g_she.find(ctx);
    if (it == g_she.end() || !it->second.count(h)) return ctx->fail(VSHE_E_NOT_FOUND, "");
    dead = std::move(it->second[h]);
    it->second.erase(h);
    // batch schedules that include this problem point at its system: drop them
    auto bt = g_she_batches.find(ctx);
    if (bt != g_she_batches.end())
      for (auto b = bt->second.begin(); b != bt->second.end();) {
        if (std::find(b->first.begin(), b->first.end(), h) != b->first.end()) b = bt->second.erase(b);
        else ++b;
      }
  }
  return VSHE_OK;
}

int vshe_she_run_batch(vshe_ctx *ctx, int32_t count, const int64_t *handles, vshe_solve_stats *stats,
                       double *full_residuals, double *device_ms) {
  if (!ctx || count <= 0 || !handles) return VSHE_E_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lk(ctx->mu);
  cudaSetDevice(ctx->device);
  std::vector<int64_t> key(handles, handles + count);
  std::vector<SheProblem *> probs;
  for (int64_t h : key) {
    SheProblem *S = find_she(ctx, h);
    if (!S) return ctx->fail(VSHE_E_NOT_FOUND, "handle " + std::to_string(h));
    if (std::find(probs.begin(), probs.end(), S) != probs.end()) return ctx->fail(VSHE_E_INVALID_ARGUMENT, "handle listed twice");
    probs.push_back(S);
  }
  Batch *B = nullptr;
  {
    std::lock_guard<std::mutex> lk2(g_she_mu);
    auto &m = g_she_batches[ctx];
    auto it = m.find(key);
    if (it != m.end()) B = it->second.get();
  }
  if (!B) {
    std::vector<System *> mem;
    for (SheProblem *S : probs) mem.push_back(S->sys.get());
    std::unique_ptr<Batch> nb(new Batch);
    int rc = nb->build(*ctx, mem);
    if (rc) return rc;
    B = nb.get();
    std::lock_guard<std::mutex> lk2(g_she_mu);
    g_she_batches[ctx][key] = std::move(nb);
  }
  cudaEvent_t a = nullptr, b = nullptr;
  if (device_ms) {
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    cudaEventRecord(a, ctx->stream);
  }
  int rc = VSHE_OK;
  for (SheProblem *S : probs)
    if ((rc = S->assemble(*ctx, 3))) break;
  std::vector<vshe_solve_stats> st;
  if (!rc) rc = B->solve(*ctx, st);
  for (size_t k = 0; !rc && k < probs.size(); ++k) rc = probs[k]->finish(*ctx);
  if (device_ms) {
    cudaEventRecord(b, ctx->stream);
    cudaEventSynchronize(b);
    float ms = 0;
    cudaEventElapsedTime(&ms, a, b);
    *device_ms = ms;
    cudaEventDestroy(a);
    cudaEventDestroy(b);
  }
  if (rc) return rc;
  int worst = VSHE_OK;
  for (size_t k = 0; k < probs.size(); ++k) {
    if (stats) stats[k] = st[k];
    if (full_residuals) full_residuals[k] = probs[k]->full_residual;
    if (st[k].status && !worst) worst = st[k].status;
  }
  if (worst) return ctx->fail(worst, "one or more systems of the batch");
  return VSHE_OK;
}

}  // extern "C"

// =======================================================================
// Served stream: continuous batching of SHE solves (vshe_server_*).
//
// A request is a device description + SHE configuration (+ solver options).  Its arrays are
// copied at submission.  One worker thread per server admits queued requests in arrival
// order while the HBM the resident problems hold stays within the budget (and at most
// max_active are resident), a quarter second of set-up per scheduling step at most while
// others are resident (the host layout of a large request on a thread of its own), sets each
// one up on the device (host set-up of the (x, H) space,
// device assembly, odd elimination, normalisation, ILU(0) factorisation) and then iterates all
// resident systems together, chunk by chunk, in one batch (shared launches of the SELL SpMV,
// the sweeps and the vector kernels).  After every chunk a converged member leaves the batch:
// its true FP64 residual is checked (a residual replacement restarts it if needed), its
// solution is recovered and post-processed, its results are copied to the host and its
// device memory is released, and queued requests take its place.  Each member's iterates do
// not depend on the batch (per-system reductions in a fixed order, per-system tiles), so a
// result in the mix equals the same request served alone.
// =======================================================================
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <thread>

namespace vshe {

struct ServeRequest {
  int64_t ticket = 0;
  // owned copies of the caller's description
  std::vector<int32_t> mat, contact, fcells, cfp, cfi;
  std::vector<double> vol, cen, nd, na, phi, fvol, fn, cpl;
  vshe_device_desc d{};
  vshe_she_config c{};
  vshe_coupling_tables t{};
  vshe_solve_opts o{};
  std::chrono::steady_clock::time_point t_submit, t_admit, t_done;
  vshe_server_result res{};
  std::vector<double> density, currents;
  std::unique_ptr<SheProblem> prob;
  std::vector<char> state;  // BiState between batch rebuilds
  int phase = 0;            // 0 queued, 1 resident, 2 done
  bool collected = false;   // the caller has its result: the worker may free the record
  int replacements = 0;
  bool needs_start = true;
  size_t need = 0;                       // the footprint bound it was admitted with
  std::thread layout_thread;             // host layout of a large request, off the worker thread
  std::atomic<bool> layout_done{false};
  // stagnation watch: the best recursive residual so far and the iteration it was reached at
  double best_res = 1e300;
  int best_iter = 0;
  bool stagnated = false;
};

struct Server {
  vshe_ctx *ctx = nullptr;
  vshe_server_opts opts{};
  std::mutex mu;
  std::condition_variable cv;
  bool stop = false;
  std::deque<ServeRequest *> pending;
  std::map<int64_t, std::unique_ptr<ServeRequest>> all;
  std::vector<ServeRequest *> active;
  std::vector<ServeRequest *> setting_up;  // admitted, host layout running on its own thread
  std::unique_ptr<Batch> batch;
  int64_t next_ticket = 0;
  std::thread worker;
  std::string error;

  void run();
  int admit(std::vector<ServeRequest *> &fresh);
  int finish_setup(ServeRequest *r);
  void end_setting_up(int status);
  int step();
  void complete(ServeRequest *r, int status);
};


void Server::complete(ServeRequest *r, int status) {
  r->t_done = std::chrono::steady_clock::now();
  r->res.status = status;
  r->res.queue_ms = std::chrono::duration<double, std::milli>(r->t_admit - r->t_submit).count();
  r->res.latency_ms = std::chrono::duration<double, std::milli>(r->t_done - r->t_submit).count();
  r->prob.reset();  // releases the problem's device memory
  std::lock_guard<std::mutex> lk(mu);
  r->phase = 2;
  cv.notify_all();
}

// Admits queued requests while memory and slots allow, for at most kAdmitSliceMs of set-up per
// step once a request is resident, admitted in this step or being set up (then the residents
// iterate and the rest of the queue is admitted in later steps, so that a long set-up at the
// back of the queue does not hold up the requests in front of it); returns the first error of
// a set-up.  The host layout of a request with at least kAsyncLayoutRows reduced unknowns (its
// ordering, ILU(k) or ILUT pattern and level schedules: seconds of host work for millions of
// rows) runs on a thread of its own; the request joins the batch in the first step after it.
constexpr double kAdmitSliceMs = 250.0;
constexpr int64_t kAsyncLayoutRows = int64_t(1) << 18;

// Device set-up after the layout: device buffers, assembly, factorisation.
int Server::finish_setup(ServeRequest *r) {
  Ctx &c = *ctx;
  SheProblem *S = r->prob.get();
  int rc = S->create_device_finish(c);
  if (!rc) rc = S->assemble(c, 3);
  if (!rc) {
    S->sys->prepare(c);
    rc = S->batch->autotune_tiles(c);
  }
  if (!rc) rc = S->batch->factor(c);
  if (rc) { r->res.status = rc; return rc; }
  r->res.n_unknowns = S->n_red;
  r->phase = 1;
  r->needs_start = true;
  return VSHE_OK;
}

// Waits for every running layout thread and ends its request with `status`.
void Server::end_setting_up(int status) {
  for (ServeRequest *r : setting_up) {
    if (r->layout_thread.joinable()) r->layout_thread.join();
    r->res.status = status;
    complete(r, status);
  }
  setting_up.clear();
}

int Server::admit(std::vector<ServeRequest *> &fresh) {
  Ctx &c = *ctx;
  size_t held = 0;
  for (ServeRequest *r : active) held += problem_bytes(r->prob.get());
  for (ServeRequest *r : setting_up) held += r->need;
  // requests whose layout has finished
  for (auto it = setting_up.begin(); it != setting_up.end();) {
    ServeRequest *r = *it;
    if (!r->layout_done.load()) { ++it; continue; }
    r->layout_thread.join();
    it = setting_up.erase(it);
    const int rc = finish_setup(r);
    if (rc) { held -= r->need; complete(r, rc); continue; }
    fresh.push_back(r);
  }
  const auto t0 = std::chrono::steady_clock::now();
  while (true) {
    if ((!active.empty() || !fresh.empty() || !setting_up.empty()) &&
        std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count() > kAdmitSliceMs)
      break;
    ServeRequest *r = nullptr;
    {
      std::lock_guard<std::mutex> lk(mu);
      if (pending.empty() || int(active.size() + fresh.size() + setting_up.size()) >= opts.max_active) break;
      r = pending.front();
    }
    // the host set-up and the footprint bound first: nothing is allocated on the device for a
    // request that has to wait or is refused
    std::unique_ptr<SheProblem> S(new SheProblem);
    int rc = S->setup_host(c, r->d, r->c, r->t, r->o);
    const size_t need = rc ? 0 : S->estimate_bytes();
    if (!rc && held + need > opts.hbm_budget && !(active.empty() && fresh.empty() && setting_up.empty())) {
      break;  // wait for resident problems to finish
    }
    {
      std::lock_guard<std::mutex> lk(mu);
      pending.pop_front();
    }
    r->t_admit = std::chrono::steady_clock::now();
    if (!rc && held + need > opts.hbm_budget) rc = c.fail(VSHE_E_BUDGET, "request alone exceeds the server's HBM budget");
    if (!rc) rc = S->create_device_pattern(c);
    if (rc) { r->res.status = rc; complete(r, rc); continue; }
    r->prob = std::move(S);
    r->need = need;
    held += need;
    if (r->prob->n_red >= kAsyncLayoutRows) {
      r->layout_done.store(false);
      r->layout_thread = std::thread([this, r] {
        r->prob->build_layout();
        r->layout_done.store(true);
        std::lock_guard<std::mutex> lk(mu);
        cv.notify_all();
      });
      setting_up.push_back(r);
      continue;
    }
    r->prob->build_layout();
    rc = finish_setup(r);
    if (rc) { held -= need; complete(r, rc); continue; }
    fresh.push_back(r);
  }
  return VSHE_OK;
}

// One scheduling step: admission, batch rebuild, one iteration chunk, completions.
int Server::step() {
  Ctx &c = *ctx;
  {
    // free the records whose results were collected (none of them is resident)
    std::lock_guard<std::mutex> lk(mu);
    for (auto it = all.begin(); it != all.end();) {
      if (it->second->collected && it->second->phase == 2) it = all.erase(it);
      else ++it;
    }
  }
  std::lock_guard<std::mutex> lk(c.mu);
  cudaSetDevice(c.device);
  std::vector<ServeRequest *> fresh;
  int rc = admit(fresh);
  if (rc) return rc;
  if (!fresh.empty() || !batch) {
    for (ServeRequest *r : fresh) active.push_back(r);
    if (active.empty()) return VSHE_OK;
    std::vector<System *> mem;
    for (ServeRequest *r : active) mem.push_back(r->prob->sys.get());
    std::unique_ptr<Batch> nb(new Batch);
    if ((rc = nb->build(c, mem))) return rc;
    batch = std::move(nb);
    // carry the running members' states over; start the newcomers
    const size_t bsz = vk_bistate_size();
    std::vector<char> st(bsz * active.size(), 0);
    std::vector<int32_t> act(active.size(), 0);
    for (size_t k = 0; k < active.size(); ++k) {
      if (active[k]->needs_start) act[k] = 1;
      else std::memcpy(st.data() + bsz * k, active[k]->state.data(), bsz);
    }
    if ((rc = batch->write_states(c, st))) return rc;
    if ((rc = batch->set_active(c, act))) return rc;
    const vshe_solve_opts &o = active.front()->o;
    if ((rc = batch->start(c, o.tol, o.max_iters, false))) return rc;
    for (ServeRequest *r : active) r->needs_start = false;
    std::fill(act.begin(), act.end(), 1);
    if ((rc = batch->set_active(c, act))) return rc;
  }
  const vshe_solve_opts &o = active.front()->o;
  const int every = o.check_every > 0 ? o.check_every : 8;
  if ((rc = batch->run_chunk(c, every))) return rc;
  std::vector<char> st;
  if ((rc = batch->read_states(c, st))) return rc;
  if ((rc = batch->check_err(c, "served chunk"))) return rc;
  const size_t bsz = vk_bistate_size();
  std::vector<int32_t> fin(active.size(), 0);
  bool any = false;
  for (size_t k = 0; k < active.size(); ++k) {
    ServeRequest *r = active[k];
    r->state.assign(st.begin() + bsz * k, st.begin() + bsz * (k + 1));
    const BiState *b = (const BiState *)r->state.data();
    if (b->done) { fin[k] = 1; any = true; continue; }
    // stagnation stop: no halving of the recursive residual within stagnation_iters iterations
    if (b->res < 0.5 * r->best_res) {
      r->best_res = b->res;
      r->best_iter = b->iter;
    } else if (opts.stagnation_iters > 0 && b->iter - r->best_iter >= opts.stagnation_iters) {
      r->stagnated = true;
      fin[k] = 1;
      any = true;
    }
  }
  if (!any) return VSHE_OK;
  // true FP64 residual of the members that stopped
  if ((rc = batch->set_active(c, fin))) return rc;
  std::vector<double> rel;
  if ((rc = batch->residual(c, rel))) return rc;
  std::vector<int32_t> resume(active.size(), 0);
  bool any_resume = false;
  std::vector<ServeRequest *> keep;
  for (size_t k = 0; k < active.size(); ++k) {
    ServeRequest *r = active[k];
    if (!fin[k]) { keep.push_back(r); continue; }
    const BiState *b = (const BiState *)r->state.data();
    if (!r->stagnated && b->status == 0 && rel[k] >= o.tol && b->iter < o.max_iters && r->replacements < 3) {
      r->replacements++;
      resume[k] = 1;
      any_resume = true;
      keep.push_back(r);
      continue;
    }
    SheProblem *S = r->prob.get();
    vk_permute(S->sys->n, S->sys->d_perm, (const double *)S->sys->kv[0], S->sys->d_x64, 0, c.stream);
    int status = b->status;
    if (r->stagnated && status == 0) status = VSHE_E_NOT_CONVERGED;
    if (status == 0 && rel[k] >= o.tol) status = VSHE_E_NOT_CONVERGED;
    if (status != 0 && rel[k] < o.tol) status = 0;
    int frc = S->finish(c);
    r->res.iterations = b->iter;
    r->res.refinements = r->replacements;
    r->res.rel_residual = rel[k];
    r->res.full_residual = S->full_residual;
    r->density.assign(size_t(S->H.nc), 0.0);
    r->currents.assign(size_t(std::max(S->ncontacts, 0)), 0.0);
    cudaError_t e = cudaMemcpyAsync(r->density.data(), S->d_dens, sizeof(double) * r->density.size(), cudaMemcpyDeviceToHost, c.stream);
    if (e == cudaSuccess && !r->currents.empty())
      e = cudaMemcpyAsync(r->currents.data(), S->d_cur, sizeof(double) * r->currents.size(), cudaMemcpyDeviceToHost, c.stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c.stream);
    if (frc == 0 && e != cudaSuccess) frc = c.cuda_fail(e, "served results");
    complete(r, frc ? frc : status);
  }
  if (any_resume) {
    if ((rc = batch->set_active(c, resume))) return rc;
    if ((rc = batch->start(c, o.tol, o.max_iters, true))) return rc;
    std::vector<char> st2;
    if ((rc = batch->read_states(c, st2))) return rc;
    for (size_t k = 0; k < active.size(); ++k)
      if (resume[k]) active[k]->state.assign(st2.begin() + bsz * k, st2.begin() + bsz * (k + 1));
  }
  if (keep.size() != active.size()) {
    active = keep;
    batch.reset();  // rebuilt over the remaining members next step
    for (ServeRequest *r : active) r->needs_start = false;
  } else {
    std::vector<int32_t> act(active.size(), 1);
    if ((rc = batch->set_active(c, act))) return rc;
  }
  return VSHE_OK;
}

void Server::run() {
  while (true) {
    {
      std::unique_lock<std::mutex> lk(mu);
      if (active.empty() && !setting_up.empty()) {
        // nothing to iterate: wait for a layout (polled, its thread notifies too)
        cv.wait_for(lk, std::chrono::milliseconds(2), [&] {
          for (ServeRequest *r : setting_up)
            if (r->layout_done.load()) return true;
          return false;
        });
      } else {
        cv.wait(lk, [&] { return stop || !pending.empty() || !active.empty(); });
      }
      if (stop && active.empty() && setting_up.empty()) {
        // drop what is still queued
        for (ServeRequest *r : pending) { r->res.status = VSHE_E_NOT_FOUND; r->phase = 2; }
        pending.clear();
        cv.notify_all();
        return;
      }
    }
    int rc = step();
    if (rc) {
      // a device error ends every resident request, and every one being set up, with that error
      std::vector<ServeRequest *> act = active;
      active.clear();
      batch.reset();
      for (ServeRequest *r : act)
        if (r->phase != 2) complete(r, rc);
      end_setting_up(rc);
      std::lock_guard<std::mutex> lk(mu);
      error = ctx->last_error;
    }
  }
}

}  // namespace vshe

struct vshe_server : public vshe::Server {};

extern "C" {

int vshe_server_create(vshe_ctx *ctx, const vshe_server_opts *opts, vshe_server **out) {
  if (!ctx || !out) return VSHE_E_INVALID_ARGUMENT;
  std::unique_ptr<vshe_server> s(new vshe_server);
  s->ctx = ctx;
  if (opts) s->opts = *opts;
  else { std::memset(&s->opts, 0, sizeof(s->opts)); vshe_default_opts(&s->opts.solve); }
  if (s->opts.hbm_budget == 0) s->opts.hbm_budget = ctx->budget;
  if (s->opts.max_active <= 0) s->opts.max_active = 256;
  if (s->opts.stagnation_iters == 0) s->opts.stagnation_iters = 400;
  vshe_server *p = s.get();
  p->worker = std::thread([p] { p->run(); });
  *out = s.release();
  return VSHE_OK;
}

int vshe_server_submit(vshe_server *srv, const vshe_device_desc *d, const vshe_she_config *c, const vshe_coupling_tables *ct,
                       const vshe_solve_opts *opts, int64_t *ticket) {
  if (!srv || !d || !c || !ct || !ticket || d->n_cells <= 0 || d->n_facets < 0 || (d->dim != 1 && d->dim != 2) || !ct->data)
    return VSHE_E_INVALID_ARGUMENT;
  std::unique_ptr<vshe::ServeRequest> r(new vshe::ServeRequest);
  const size_t nc = size_t(d->n_cells), nf = size_t(d->n_facets), dim = size_t(d->dim);
  r->mat.assign(d->cell_material, d->cell_material + nc);
  r->vol.assign(d->cell_volume, d->cell_volume + nc);
  r->cen.assign(d->cell_centroid, d->cell_centroid + nc * dim);
  r->nd.assign(d->doping_n, d->doping_n + nc);
  r->na.assign(d->doping_p, d->doping_p + nc);
  r->phi.assign(d->potential, d->potential + nc);
  r->contact.assign(d->contact_id, d->contact_id + nc);
  r->fcells.assign(d->facet_cells, d->facet_cells + 2 * nf);
  r->fvol.assign(d->facet_volume, d->facet_volume + nf);
  r->fn.assign(d->facet_normal, d->facet_normal + nf * dim);
  r->cfp.assign(d->cell_facet_ptr, d->cell_facet_ptr + nc + 1);
  r->cfi.assign(d->cell_facet_idx, d->cell_facet_idx + size_t(d->cell_facet_ptr[nc]));
  const size_t D = size_t((ct->L + 1) * (ct->L + 1));
  r->cpl.assign(ct->data, ct->data + 6 * D * D);
  r->d = *d;
  r->d.cell_material = r->mat.data(); r->d.cell_volume = r->vol.data(); r->d.cell_centroid = r->cen.data();
  r->d.doping_n = r->nd.data(); r->d.doping_p = r->na.data(); r->d.potential = r->phi.data();
  r->d.contact_id = r->contact.data(); r->d.facet_cells = r->fcells.data(); r->d.facet_volume = r->fvol.data();
  r->d.facet_normal = r->fn.data(); r->d.cell_facet_ptr = r->cfp.data(); r->d.cell_facet_idx = r->cfi.data();
  r->c = *c;
  r->t.L = ct->L; r->t.data = r->cpl.data();
  r->o = opts ? *opts : srv->opts.solve;
  r->o.block_ptr = nullptr; r->o.n_blocks = 0; r->o.perm = nullptr;  // per-request arrays are not carried
  if (r->o.precision != srv->opts.solve.precision || (r->o.precond == VSHE_PRECOND_NONE) != (srv->opts.solve.precond == VSHE_PRECOND_NONE))
    return VSHE_E_INVALID_ARGUMENT;  // one batch: same precision and preconditioner kind
  r->o.tol = srv->opts.solve.tol; r->o.max_iters = srv->opts.solve.max_iters; r->o.check_every = srv->opts.solve.check_every;
  r->t_submit = std::chrono::steady_clock::now();
  std::lock_guard<std::mutex> lk(srv->mu);
  r->ticket = ++srv->next_ticket;
  *ticket = r->ticket;
  srv->pending.push_back(r.get());
  srv->all[r->ticket] = std::move(r);
  srv->cv.notify_all();
  return VSHE_OK;
}

int vshe_server_wait(vshe_server *srv, int64_t ticket, double timeout_ms, vshe_server_result *res, double *density, double *currents) {
  if (!srv) return VSHE_E_INVALID_ARGUMENT;
  std::unique_lock<std::mutex> lk(srv->mu);
  auto it = srv->all.find(ticket);
  if (it == srv->all.end() || it->second->collected) return VSHE_E_NOT_FOUND;
  vshe::ServeRequest *r = it->second.get();
  auto ready = [&] { return r->phase == 2; };
  if (timeout_ms < 0) srv->cv.wait(lk, ready);
  else if (!srv->cv.wait_for(lk, std::chrono::duration<double, std::milli>(timeout_ms), ready)) return VSHE_E_TIMEOUT;
  if (res) *res = r->res;
  if (density) std::copy(r->density.begin(), r->density.end(), density);
  if (currents) std::copy(r->currents.begin(), r->currents.end(), currents);
  const int status = r->res.status;
  r->collected = true;  // freed by the worker once it no longer refers to it
  return status;
}

int vshe_server_destroy(vshe_server *srv) {
  if (!srv) return VSHE_E_INVALID_ARGUMENT;
  {
    std::lock_guard<std::mutex> lk(srv->mu);
    srv->stop = true;
    srv->cv.notify_all();
  }
  if (srv->worker.joinable()) srv->worker.join();
  delete srv;
  return VSHE_OK;
}

}  // extern "C"

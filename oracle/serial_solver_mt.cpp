// serial_solver_mt.cpp -- TEST INFRASTRUCTURE, not product code.
//
// The reference's native SHE linear solve on the host's cores, for bench.py's reference arm and
// CPU baseline: src/solvers/viennacl/serial_linear_solver.hpp:101-156 runs ILU(0) on the whole
// reduced system in the caller's row order (ilu0_tag, :125-126) and BiCGStab with the initial
// residual as shadow vector (bicgstab_tag, :129-136) to the config's relative tolerance.  The
// arithmetic restates she_oracle.cpp's single-threaded ILU(0) (Saad Alg. 10.4, IKJ) and BiCGStab
// (van der Vorst 1992) row for row; only the schedule is parallel:
//   * the factorisation and both triangular solves run level by level (a row's level is one
//     more than the highest level of the earlier rows it reads), the rows of a level split over
//     the threads, so every row performs the same operations in the same order as serially; the
//     factor is copied into sweep order (a level's rows contiguous) so each thread streams its
//     part of a level;
//   * SpMV and vector updates split rows over the threads (same per-row arithmetic);
//   * inner products sum per-thread partials in thread order (deterministic for a fixed thread
//     count; with one thread, the serial oracle's order).
// ViennaCL itself is absent from the reference tree, so, as in she_oracle.cpp, the solver follows
// the published algorithms, not ViennaCL's source.
//
// Build: oracle/build.sh (g++ -O2 -ffp-contract=off -fopenmp).

#include <omp.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <vector>

namespace {

using clk = std::chrono::steady_clock;

struct Levels {
  std::vector<int64_t> ptr;  // level k = rows[ptr[k] .. ptr[k+1])
  std::vector<int32_t> rows;
};

// forward (L: columns < row) or backward (U: columns > row) levels of the pattern
Levels make_levels(int64_t n, const int64_t *rp, const int32_t *ci, bool forward) {
  std::vector<int32_t> lev((size_t)n, 0);
  int32_t nlev = 0;
  if (forward) {
    for (int64_t i = 0; i < n; ++i) {
      int32_t m = -1;
      for (int64_t k = rp[i]; k < rp[i + 1] && ci[k] < i; ++k) m = std::max(m, lev[size_t(ci[k])]);
      lev[size_t(i)] = m + 1;
      nlev = std::max(nlev, m + 2);
    }
  } else {
    for (int64_t i = n - 1; i >= 0; --i) {
      int32_t m = -1;
      for (int64_t k = rp[i + 1] - 1; k >= rp[i] && ci[k] > i; --k) m = std::max(m, lev[size_t(ci[k])]);
      lev[size_t(i)] = m + 1;
      nlev = std::max(nlev, m + 2);
    }
  }
  Levels L;
  L.ptr.assign(size_t(nlev) + 1, 0);
  for (int64_t i = 0; i < n; ++i) L.ptr[size_t(lev[size_t(i)]) + 1]++;
  for (size_t k = 1; k < L.ptr.size(); ++k) L.ptr[k] += L.ptr[k - 1];
  L.rows.resize((size_t)n);
  std::vector<int64_t> cur(L.ptr.begin(), L.ptr.end() - 1);
  for (int64_t i = 0; i < n; ++i) L.rows[size_t(cur[size_t(lev[size_t(i)])]++)] = int32_t(i);
  return L;
}

// rows of one level split into contiguous parts, one per thread
inline void level_part(const Levels &L, size_t k, int t, int nt, int64_t &a, int64_t &b) {
  const int64_t lo = L.ptr[k], m = L.ptr[k + 1] - lo;
  a = lo + m * t / nt;
  b = lo + m * (t + 1) / nt;
}

inline void row_part(int64_t n, int t, int nt, int64_t &a, int64_t &b) {
  a = n * t / nt;
  b = n * (t + 1) / nt;
}

struct Solver {
  int64_t n = 0;
  const int64_t *rp = nullptr;
  const int32_t *ci = nullptr;
  const double *v = nullptr;
  int nt = 1;
  std::vector<int64_t> diag;
  std::vector<double> lu;
  Levels fw, bw;
  std::vector<double> part;  // per-thread partial sums (padded to a cache line)
  // the factor copied into sweep order (the rows of a level contiguous, so every thread streams
  // its part of a level): forward row q = fw.rows[q] holds its L entries [fp[q], fp[q+1]);
  // backward row q = bw.rows[q] its U entries without the diagonal [bp[q], bp[q+1]) and the
  // diagonal bd[q]
  std::vector<int64_t> fp, bp;
  std::vector<int32_t> fc, bc;
  std::vector<double> fv, bv, bd;

  // ILU(0) in the pattern of A, in the caller's order: she_oracle.cpp ilu0_values without blocks
  // (pos map replaced by a merge of the two sorted rows; same updates in the same order)
  void factor() {
    lu.assign(v, v + rp[n]);
#pragma omp parallel num_threads(nt)
    {
      const int t = omp_get_thread_num();
      for (size_t lv = 0; lv + 1 < fw.ptr.size(); ++lv) {
        int64_t a, b;
        level_part(fw, lv, t, nt, a, b);
        for (int64_t q = a; q < b; ++q) {
          const int64_t i = fw.rows[size_t(q)];
          const int64_t e = rp[i + 1];
          for (int64_t k = rp[i]; k < e; ++k) {
            const int64_t c = ci[k];
            if (c >= i) break;
            const double piv = lu[size_t(diag[size_t(c)])];
            lu[size_t(k)] /= piv;
            const double lik = lu[size_t(k)];
            int64_t p = k + 1;
            for (int64_t kk = diag[size_t(c)] + 1; kk < rp[c + 1]; ++kk) {
              const int32_t j = ci[kk];
              while (p < e && ci[p] < j) ++p;
              if (p < e && ci[p] == j) lu[size_t(p)] -= lik * lu[size_t(kk)];
            }
          }
        }
#pragma omp barrier
      }
    }
  }

  void stream_factor() {
    fp.assign(size_t(n) + 1, 0);
    bp.assign(size_t(n) + 1, 0);
    for (int64_t q = 0; q < n; ++q) {
      const int64_t i = fw.rows[size_t(q)], j = bw.rows[size_t(q)];
      fp[size_t(q) + 1] = fp[size_t(q)] + (diag[size_t(i)] - rp[i]);
      bp[size_t(q) + 1] = bp[size_t(q)] + (rp[j + 1] - diag[size_t(j)] - 1);
    }
    fc.resize(size_t(fp[size_t(n)])); fv.resize(fc.size());
    bc.resize(size_t(bp[size_t(n)])); bv.resize(bc.size()); bd.resize(size_t(n));
#pragma omp parallel for num_threads(nt) schedule(static)
    for (int64_t q = 0; q < n; ++q) {
      const int64_t i = fw.rows[size_t(q)], j = bw.rows[size_t(q)];
      for (int64_t k = rp[i], o = fp[size_t(q)]; k < diag[size_t(i)]; ++k, ++o) { fc[size_t(o)] = ci[k]; fv[size_t(o)] = lu[size_t(k)]; }
      for (int64_t k = diag[size_t(j)] + 1, o = bp[size_t(q)]; k < rp[j + 1]; ++k, ++o) { bc[size_t(o)] = ci[k]; bv[size_t(o)] = lu[size_t(k)]; }
      bd[size_t(q)] = lu[size_t(diag[size_t(j)])];
    }
  }

  // x = (L U)^{-1} b: she_oracle.cpp ILU::apply
  void apply(const double *b, double *x) {
#pragma omp parallel num_threads(nt)
    {
      const int t = omp_get_thread_num();
      for (size_t lv = 0; lv + 1 < fw.ptr.size(); ++lv) {
        int64_t a, e;
        level_part(fw, lv, t, nt, a, e);
        for (int64_t q = a; q < e; ++q) {
          const int64_t i = fw.rows[size_t(q)];
          double s = b[i];
          for (int64_t k = fp[size_t(q)]; k < fp[size_t(q) + 1]; ++k) s -= fv[size_t(k)] * x[fc[size_t(k)]];
          x[i] = s;
        }
#pragma omp barrier
      }
      for (size_t lv = 0; lv + 1 < bw.ptr.size(); ++lv) {
        int64_t a, e;
        level_part(bw, lv, t, nt, a, e);
        for (int64_t q = a; q < e; ++q) {
          const int64_t i = bw.rows[size_t(q)];
          double s = x[i];
          for (int64_t k = bp[size_t(q)]; k < bp[size_t(q) + 1]; ++k) s -= bv[size_t(k)] * x[bc[size_t(k)]];
          x[i] = s / bd[size_t(q)];
        }
#pragma omp barrier
      }
    }
  }

  void spmv(const double *x, double *y) {
#pragma omp parallel for num_threads(nt) schedule(static)
    for (int64_t i = 0; i < n; ++i) {
      double s = 0.0;
      for (int64_t k = rp[i]; k < rp[i + 1]; ++k) s += v[k] * x[ci[k]];
      y[i] = s;
    }
  }

  double dot(const double *a, const double *b) {
#pragma omp parallel num_threads(nt)
    {
      const int t = omp_get_thread_num();
      int64_t lo, hi;
      row_part(n, t, nt, lo, hi);
      double s = 0.0;
      for (int64_t i = lo; i < hi; ++i) s += a[i] * b[i];
      part[size_t(t) * 8] = s;
    }
    double s = 0.0;
    for (int t = 0; t < nt; ++t) s += part[size_t(t) * 8];
    return s;
  }
};

}  // namespace

extern "C" {

// ILU(0) + BiCGStab (r^ = r_0) to `tol` on `threads` host threads (0: all), x0 = 0.  Returns
// 0 converged, 1 iteration limit, -1 breakdown, -2 a row without diagonal entry.  out[0] =
// iterations, out[1] = final recursive relative residual, out[2] = factorisation seconds (with
// the level analysis), out[3] = iteration seconds, out[4] = threads used; iter_s (may be NULL,
// maxit + 1 entries) receives the elapsed seconds after the factorisation and after every
// iteration.
int vsheo_serial_solve_mt(int64_t n, const int64_t *rp, const int32_t *ci, const double *v, const double *b, double *x,
                          double tol, int32_t maxit, int32_t threads, double *out, double *iter_s) {
  const auto t0 = clk::now();
  Solver S;
  S.n = n; S.rp = rp; S.ci = ci; S.v = v;
  S.nt = threads > 0 ? threads : omp_get_max_threads();
  S.part.assign(size_t(S.nt) * 8, 0.0);
  S.diag.assign(size_t(n), -1);
  for (int64_t i = 0; i < n; ++i) {
    for (int64_t k = rp[i]; k < rp[i + 1]; ++k)
      if (ci[k] == i) S.diag[size_t(i)] = k;
    if (S.diag[size_t(i)] < 0) return -2;  // ILU(0) needs every diagonal entry
  }
  S.fw = make_levels(n, rp, ci, true);
  S.bw = make_levels(n, rp, ci, false);
  S.factor();
  S.stream_factor();
  const auto t1 = clk::now();
  const size_t N = size_t(n);
  std::vector<double> r(b, b + n), rh, p(N, 0.0), vv(N, 0.0), s(N), t(N), ph(N, 0.0), sh(N, 0.0), xv(N, 0.0);
  rh = r;
  auto finish = [&](int rc, int it, double res) {
    std::copy(xv.begin(), xv.end(), x);
    out[0] = it; out[1] = res;
    out[2] = std::chrono::duration<double>(t1 - t0).count();
    out[3] = std::chrono::duration<double>(clk::now() - t1).count();
    out[4] = S.nt;
    return rc;
  };
  if (iter_s) iter_s[0] = 0.0;
  const double nb = std::sqrt(S.dot(b, b));
  if (nb == 0.0) return finish(0, 0, 0.0);
  double rho_old = 1, alpha = 1, omega = 1;
  double res = std::sqrt(S.dot(r.data(), r.data())) / nb;
  if (res < tol) return finish(0, 0, res);
  for (int it = 1; it <= maxit; ++it) {
    const double rho = S.dot(rh.data(), r.data());
    if (rho == 0.0) return finish(-1, it, res);
    if (it == 1) {
      p = r;
    } else {
      const double beta = (rho / rho_old) * (alpha / omega);
#pragma omp parallel for num_threads(S.nt) schedule(static)
      for (int64_t i = 0; i < n; ++i) p[size_t(i)] = r[size_t(i)] + beta * (p[size_t(i)] - omega * vv[size_t(i)]);
    }
    S.apply(p.data(), ph.data());
    S.spmv(ph.data(), vv.data());
    const double rv = S.dot(rh.data(), vv.data());
    if (rv == 0.0) return finish(-1, it, res);
    alpha = rho / rv;
#pragma omp parallel for num_threads(S.nt) schedule(static)
    for (int64_t i = 0; i < n; ++i) s[size_t(i)] = r[size_t(i)] - alpha * vv[size_t(i)];
    const double sn = std::sqrt(S.dot(s.data(), s.data())) / nb;
    if (sn < tol) {
#pragma omp parallel for num_threads(S.nt) schedule(static)
      for (int64_t i = 0; i < n; ++i) xv[size_t(i)] += alpha * ph[size_t(i)];
      if (iter_s) iter_s[it] = std::chrono::duration<double>(clk::now() - t1).count();
      return finish(0, it, sn);
    }
    S.apply(s.data(), sh.data());
    S.spmv(sh.data(), t.data());
    const double tt = S.dot(t.data(), t.data());
    omega = tt == 0.0 ? 0.0 : S.dot(t.data(), s.data()) / tt;
#pragma omp parallel for num_threads(S.nt) schedule(static)
    for (int64_t i = 0; i < n; ++i) {
      xv[size_t(i)] += alpha * ph[size_t(i)] + omega * sh[size_t(i)];
      r[size_t(i)] = s[size_t(i)] - omega * t[size_t(i)];
    }
    res = std::sqrt(S.dot(r.data(), r.data())) / nb;
    if (iter_s) iter_s[it] = std::chrono::duration<double>(clk::now() - t1).count();
    if (res < tol) return finish(0, it, res);
    if (omega == 0.0) return finish(-1, it, res);
    rho_old = rho;
  }
  return finish(1, maxit, res);
}

}  // extern "C"

"""Python view of libvshe_b200.so (ctypes over include/vshe_gpu.h).

The product is the C++/CUDA library; this module marshals numpy arrays into
its C ABI for tests and benchmarks.  There is no CPU fallback: if the
library or a GPU is missing, every call raises.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from .abi import LIB_PATH, SolveOptsC, SolveStatsC, ptr

VSHE_OK = 0
ERRORS = {
    -1: "INVALID_ARGUMENT", -2: "EMPTY_ROW", -3: "NAN", -4: "ODD_DIAGONAL", -5: "BREAKDOWN",
    -6: "NOT_CONVERGED", -7: "OUT_OF_MEMORY", -8: "BUDGET", -9: "CUDA", -10: "TIMEOUT",
    -11: "ZERO_PIVOT", -12: "NOT_FOUND", -13: "UNSUPPORTED",
}
PRECISION = {"fp64": 0, "mixed": 1}
PRECOND = {"none": 0, "ilu0": 1, "block_ilu0": 2}
TRSV = {"auto": 0, "persistent": 1, "per_level": 2}

_lib = None


class VsheError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("%s (%d): %s" % (ERRORS.get(code, "?"), code, msg))
        self.code = code


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise VsheError(-13, "library not built: %s (run __graft_entry__.build())" % LIB_PATH)
        L = C.CDLL(LIB_PATH)
        i64p = C.POINTER(C.c_int64)
        i32p = C.POINTER(C.c_int32)
        f64p = C.POINTER(C.c_double)
        vp = C.c_void_p
        L.vshe_default_opts.argtypes = [C.POINTER(SolveOptsC)]
        L.vshe_errstr.restype = C.c_char_p
        L.vshe_errstr.argtypes = [C.c_int]
        L.vshe_create.argtypes = [C.POINTER(vp), C.c_int, C.c_size_t]
        L.vshe_destroy.argtypes = [vp]
        L.vshe_last_error.restype = C.c_char_p
        L.vshe_last_error.argtypes = [vp]
        L.vshe_bytes_in_use.restype = C.c_size_t
        L.vshe_bytes_in_use.argtypes = [vp]
        L.vshe_solve_csr.argtypes = [vp, C.c_int64, C.c_int64, i64p, i32p, f64p, f64p, C.POINTER(SolveOptsC), f64p, C.POINTER(SolveStatsC)]
        L.vshe_system_create.argtypes = [vp, C.c_int64, C.c_int64, i64p, i32p, f64p, f64p, C.POINTER(SolveOptsC), i64p]
        L.vshe_system_set_values.argtypes = [vp, C.c_int64, f64p, f64p]
        L.vshe_system_solve.argtypes = [vp, C.c_int64, f64p, C.POINTER(SolveStatsC)]
        L.vshe_batch_solve.argtypes = [vp, C.c_int32, i64p, C.POINTER(SolveStatsC)]
        L.vshe_system_get_x.argtypes = [vp, C.c_int64, f64p]
        L.vshe_system_free.argtypes = [vp, C.c_int64]
        L.vshe_system_spmv.argtypes = [vp, C.c_int64, C.c_int32, f64p, f64p]
        L.vshe_system_factor_values.argtypes = [vp, C.c_int64, f64p]
        L.vshe_system_time_spmv.argtypes = [vp, C.c_int64, C.c_int32, C.c_int32, f64p]
        _lib = L
    return _lib


def make_opts(precision="mixed", precond="ilu0", tol=1e-10, max_iters=1000, inner_tol=1e-5,
              max_refinements=10, blocks=None, trsv="auto", check_every=8):
    o = SolveOptsC()
    lib().vshe_default_opts(C.byref(o))
    o.precision = PRECISION[precision]
    o.precond = PRECOND[precond]
    o.tol = tol
    o.max_iters = max_iters
    o.inner_tol = inner_tol
    o.max_refinements = max_refinements
    o.trsv_mode = TRSV[trsv]
    o.check_every = check_every
    keep = None
    if blocks is not None:
        keep = np.ascontiguousarray(blocks, np.int64)
        o.n_blocks = len(keep) - 1
        o.block_ptr = ptr(keep, C.c_int64)
    return o, keep


def stats_dict(st: SolveStatsC):
    return {k: getattr(st, k) for k, _ in SolveStatsC._fields_}


class Context:
    """A vshe_ctx on one GPU."""

    def __init__(self, device=0, hbm_budget=0):
        h = C.c_void_p()
        rc = lib().vshe_create(C.byref(h), device, hbm_budget)
        if rc:
            raise VsheError(rc, "vshe_create failed (no usable CUDA device?)")
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            lib().vshe_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc):
        if rc:
            raise VsheError(rc, lib().vshe_last_error(self.h).decode())

    def bytes_in_use(self):
        return int(lib().vshe_bytes_in_use(self.h))

    def solve_csr(self, rp, ci, v, b, **kw):
        """The drop-in call: host CSR + rhs in, host x out (copies inside)."""
        rp = np.ascontiguousarray(rp, np.int64)
        ci = np.ascontiguousarray(ci, np.int32)
        v = np.ascontiguousarray(v, np.float64)
        b = np.ascontiguousarray(b, np.float64)
        n = len(rp) - 1
        x = np.zeros(n)
        o, keep = make_opts(**kw)
        st = SolveStatsC()
        rc = lib().vshe_solve_csr(self.h, n, int(rp[-1]), ptr(rp, C.c_int64), ptr(ci, C.c_int32), ptr(v, C.c_double),
                                  ptr(b, C.c_double), C.byref(o), ptr(x, C.c_double), C.byref(st))
        if rc and rc != -6:
            self._check(rc)
        return x, stats_dict(st)

    def system(self, rp, ci, v, b, **kw):
        return System(self, rp, ci, v, b, **kw)

    def batch_solve(self, systems):
        hs = np.array([s.h for s in systems], np.int64)
        st = (SolveStatsC * len(systems))()
        rc = lib().vshe_batch_solve(self.h, len(systems), ptr(hs, C.c_int64), st)
        if rc and rc != -6:
            self._check(rc)
        return [stats_dict(s) for s in st]


class System:
    """A resident system (vshe_system_*)."""

    def __init__(self, ctx: Context, rp, ci, v, b, **kw):
        self.ctx = ctx
        self.rp = np.ascontiguousarray(rp, np.int64)
        self.ci = np.ascontiguousarray(ci, np.int32)
        v = np.ascontiguousarray(v, np.float64)
        b = np.ascontiguousarray(b, np.float64)
        self.n = len(self.rp) - 1
        self.nnz = int(self.rp[-1])
        o, self._keep = make_opts(**kw)
        h = C.c_int64()
        rc = lib().vshe_system_create(ctx.h, self.n, self.nnz, ptr(self.rp, C.c_int64), ptr(self.ci, C.c_int32),
                                      ptr(v, C.c_double), ptr(b, C.c_double), C.byref(o), C.byref(h))
        ctx._check(rc)
        self.h = h.value

    def free(self):
        if self.h:
            lib().vshe_system_free(self.ctx.h, self.h)
            self.h = 0

    def set_values(self, v, b):
        v = np.ascontiguousarray(v, np.float64)
        b = np.ascontiguousarray(b, np.float64)
        self.ctx._check(lib().vshe_system_set_values(self.ctx.h, self.h, ptr(v, C.c_double), ptr(b, C.c_double)))

    def solve(self, want_x=True):
        x = np.zeros(self.n) if want_x else None
        st = SolveStatsC()
        rc = lib().vshe_system_solve(self.ctx.h, self.h, ptr(x, C.c_double) if want_x else None, C.byref(st))
        if rc and rc != -6:
            self.ctx._check(rc)
        return x, stats_dict(st)

    def x(self):
        x = np.zeros(self.n)
        self.ctx._check(lib().vshe_system_get_x(self.ctx.h, self.h, ptr(x, C.c_double)))
        return x

    def spmv(self, x, precision="fp64"):
        x = np.ascontiguousarray(x, np.float64)
        y = np.zeros(self.n)
        self.ctx._check(lib().vshe_system_spmv(self.ctx.h, self.h, PRECISION[precision], ptr(x, C.c_double), ptr(y, C.c_double)))
        return y

    def factor_values(self):
        lu = np.zeros(self.nnz)
        self.ctx._check(lib().vshe_system_factor_values(self.ctx.h, self.h, ptr(lu, C.c_double)))
        return lu

    def time_spmv(self, precision="fp64", reps=20):
        ms = C.c_double()
        self.ctx._check(lib().vshe_system_time_spmv(self.ctx.h, self.h, PRECISION[precision], reps, C.byref(ms)))
        return ms.value

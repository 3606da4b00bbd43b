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
    -11: "ZERO_PIVOT", -12: "NOT_FOUND", -13: "UNSUPPORTED", -14: "CAPACITY",
}
PRECISION = {"fp64": 0, "mixed": 1}
PRECOND = {"none": 0, "ilu0": 1, "block_ilu0": 2, "ilut": 3}
ORDERING = {"natural": 0, "multicolor": 1}
TRSV = {"auto": 0, "persistent": 1, "per_level": 2, "per_system": 3, "flow": 4, "per_block": 5}

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
        L.vshe_set_profiling.argtypes = [vp, C.c_int32]
        L.vshe_set_spin_limit.argtypes = [vp, C.c_uint64]
        L.vshe_set_task_sweep.argtypes = [vp, C.c_int32]
        L.vshe_solve_csr_release.argtypes = [vp]
        L.vshe_get_profile.argtypes = [vp, f64p, i64p]
        L.vshe_kernel_launches.restype = C.c_int64
        L.vshe_kernel_launches.argtypes = []
        _lib = L
    return _lib


def layout(rp, ci, values=None, **kw):
    """The solver order and SELL-32 tables the library builds for this pattern and these
    options (host only, no GPU): dict of numpy arrays, see vshe_layout_export."""
    L = lib()
    i64p = C.POINTER(C.c_int64)
    i32p = C.POINTER(C.c_int32)
    rp = np.ascontiguousarray(rp, np.int64)
    ci = np.ascontiguousarray(ci, np.int32)
    n = len(rp) - 1
    nnz = int(rp[-1])
    o, keep = make_opts(**kw)
    sz = np.zeros(10, np.int64)
    vals = None if values is None else np.ascontiguousarray(values, np.float64)
    vp = None if vals is None else ptr(vals, C.c_double)
    L.vshe_layout_sizes.argtypes = [C.c_int64, C.c_int64, i64p, i32p, C.POINTER(C.c_double), C.POINTER(SolveOptsC), i64p]
    rc = L.vshe_layout_sizes(n, nnz, ptr(rp, C.c_int64), ptr(ci, C.c_int32), vp, C.byref(o), ptr(sz, C.c_int64))
    if rc:
        raise VsheError(rc, "vshe_layout_sizes")
    nslA, padA, nslL, padL, nslU, padU, nlevL, nlevU, nnzL, nnzU = [int(v) for v in sz]
    out = dict(perm=np.zeros(n, np.int32), lvr=np.zeros(nlevL + 1, np.int64), aoff=np.zeros(nslA + 1, np.int64),
               acol=np.zeros(padA, np.int32), amap=np.zeros(padA, np.int64), lrow0=np.zeros(nslL + 1, np.int32),
               loff=np.zeros(nslL + 1, np.int64), lcol=np.zeros(padL, np.int32), lmap=np.zeros(padL, np.int64),
               uslot0=np.zeros(nslU + 1, np.int32), uoff=np.zeros(nslU + 1, np.int64), ucol=np.zeros(padU, np.int32),
               umap=np.zeros(padU, np.int64), urow=np.zeros(n, np.int32))
    order = ["perm", "lvr", "aoff", "acol", "amap", "lrow0", "loff", "lcol", "lmap", "uslot0", "uoff", "ucol", "umap", "urow"]
    ct = {np.dtype(np.int32): C.c_int32, np.dtype(np.int64): C.c_int64}
    L.vshe_layout_export.argtypes = [C.c_int64, C.c_int64, i64p, i32p, C.POINTER(C.c_double), C.POINTER(SolveOptsC)] + \
        [C.POINTER(ct[out[k].dtype]) for k in order]
    rc = L.vshe_layout_export(n, nnz, ptr(rp, C.c_int64), ptr(ci, C.c_int32), vp, C.byref(o),
                              *[ptr(out[k], ct[out[k].dtype]) for k in order])
    if rc:
        raise VsheError(rc, "vshe_layout_export")
    out.update(n=n, nlevL=nlevL, nlevU=nlevU, nnzL=nnzL, nnzU=nnzU)
    return out


def sweep_plan(rp, ci, values=None, num_sms=148, **kw):
    """vshe_layout_sweep_plan: the task sweep plan of one system (host only) -> dict with "kind"
    (0 grid-wide, 1 one task, 2 block tasks), "tasks" (t, 6), "chunks" (c, 10), "sdesc" (d, 4)."""
    L = lib()
    rp = np.ascontiguousarray(rp, np.int64)
    ci = np.ascontiguousarray(ci, np.int32)
    n = len(rp) - 1
    o, keep = make_opts(**kw)
    vals = None if values is None else np.ascontiguousarray(values, np.float64)
    L.vshe_layout_sweep_plan.argtypes = [C.c_int64, C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(SolveOptsC),
                                         C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    cnt = np.zeros(4, np.int64)
    vp = None if vals is None else vals.ctypes.data
    args = (n, int(rp[-1]), rp.ctypes.data, ci.ctypes.data, vp, C.byref(o), int(num_sms))
    rc = L.vshe_layout_sweep_plan(*args, cnt.ctypes.data, None, None, None)
    if rc:
        raise VsheError(rc, "vshe_layout_sweep_plan")
    tasks = np.zeros((int(cnt[0]), 6), np.int32)
    chunks = np.zeros((int(cnt[1]), 10), np.int64)
    sdesc = np.zeros((int(cnt[2]), 4), np.int32)
    rc = L.vshe_layout_sweep_plan(*args, cnt.ctypes.data, tasks.ctypes.data, chunks.ctypes.data, sdesc.ctypes.data)
    if rc:
        raise VsheError(rc, "vshe_layout_sweep_plan")
    return {"kind": int(cnt[3]), "tasks": tasks, "chunks": chunks, "sdesc": sdesc}


def kernel_launches():
    """This library's own kernel launches in the process so far."""
    return int(lib().vshe_kernel_launches())


def set_host_threads(threads=0):
    """vshe_set_host_threads: host threads of the library's host work (0: up to 16)."""
    L = lib()
    L.vshe_set_host_threads.argtypes = [C.c_int32]
    rc = L.vshe_set_host_threads(int(threads))
    if rc:
        raise VsheError(rc, "vshe_set_host_threads")


def make_opts(precision="mixed", precond="ilu0", tol=1e-10, max_iters=1000, inner_tol=1e-5,
              max_refinements=10, blocks=None, trsv="auto", check_every=8, ordering="natural", perm=None,
              shadow="dense", fill_level=0, ilut_entries=20, ilut_drop=1e-3):
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
    o.ordering = ORDERING[ordering]
    o.shadow = {"dense": 0, "r0": 1}[shadow]
    o.fill_level = int(fill_level)
    o.ilut_entries = int(ilut_entries)
    o.ilut_drop = float(ilut_drop)
    keep = []
    if blocks is not None:
        kb = np.ascontiguousarray(blocks, np.int64)
        keep.append(kb)
        o.n_blocks = len(kb) - 1
        o.block_ptr = ptr(kb, C.c_int64)
    if perm is not None:
        kp = np.ascontiguousarray(perm, np.int32)
        keep.append(kp)
        o.perm = ptr(kp, C.c_int32)
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

    def set_profiling(self, on=True):
        self._check(lib().vshe_set_profiling(self.h, 1 if on else 0))

    def release_csr_cache(self):
        """Frees the system vshe_solve_csr keeps resident for its last pattern."""
        self._check(lib().vshe_solve_csr_release(self.h))

    def set_task_sweep(self, kernel=-1):
        """Task sweep kernel: -1 autotuned, 0 staged single CTA, 2 / 4 / 8 CTAs per cluster."""
        self._check(lib().vshe_set_task_sweep(self.h, int(kernel)))

    def set_spin_limit(self, polls=0):
        """Polls of every bounded device-side wait before VSHE_E_TIMEOUT (0: the default)."""
        self._check(lib().vshe_set_spin_limit(self.h, int(polls)))

    def profile(self):
        """Device ms of the last solve per kernel class and launch counts."""
        ms = np.zeros(5)
        cnt = np.zeros(2, np.int64)
        self._check(lib().vshe_get_profile(self.h, ptr(ms, C.c_double), ptr(cnt, C.c_int64)))
        return dict(spmv_ms=ms[0], trsv_ms=ms[1], vector_ms=ms[2], reliable_ms=ms[3], factor_ms=ms[4],
                    spmv_launches=int(cnt[0]), trsv_launches=int(cnt[1]))

    def autotune_info(self, n):
        """(rows per reduction tile chosen for n's size class, ms per SpMV for 512/1024/2048/4096)."""
        L = lib()
        L.vshe_autotune_info.argtypes = [C.c_void_p, C.c_int64, C.POINTER(C.c_int64), C.POINTER(C.c_double)]
        rows = C.c_int64()
        ms = np.zeros(4)
        self._check(L.vshe_autotune_info(self.h, int(n), C.byref(rows), ptr(ms, C.c_double)))
        return int(rows.value), ms

    def solve_csr(self, rp, ci, v, b, out=None, **kw):
        """The drop-in call: host CSR + rhs in, host x out (copies inside); `out` (n float64,
        contiguous) receives x when given."""
        rp = np.ascontiguousarray(rp, np.int64)
        ci = np.ascontiguousarray(ci, np.int32)
        v = np.ascontiguousarray(v, np.float64)
        b = np.ascontiguousarray(b, np.float64)
        n = len(rp) - 1
        x = np.zeros(n) if out is None else out
        assert x.dtype == np.float64 and x.flags["C_CONTIGUOUS"] and x.shape == (n,)
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


# ---------------------------------------------------------------- SHE path
class SheInfoC(C.Structure):
    _fields_ = [
        ("n_energies", C.c_int32), ("n_even", C.c_int64), ("n_odd", C.c_int64),
        ("nnz_full", C.c_int64), ("nnz_reduced", C.c_int64),
        ("n_cells", C.c_int32), ("n_facets", C.c_int32), ("n_contacts", C.c_int32),
        ("hbar_omega", C.c_double), ("bytes_device", C.c_int64),
        ("levels_L", C.c_int32), ("levels_U", C.c_int32), ("nnz_factor", C.c_int64), ("bytes_estimate", C.c_int64),
    ]


def _she_lib():
    L = lib()
    if not getattr(L, "_she_ready", False):
        i64p = C.POINTER(C.c_int64)
        i32p = C.POINTER(C.c_int32)
        f64p = C.POINTER(C.c_double)
        vp = C.c_void_p
        L.vshe_coupling_tables_compute.argtypes = [C.c_int32, f64p]
        L.vshe_she_create.argtypes = [vp, vp, vp, vp, C.POINTER(SolveOptsC), i64p]
        L.vshe_she_info_get.argtypes = [vp, C.c_int64, C.POINTER(SheInfoC)]
        L.vshe_she_assemble.argtypes = [vp, C.c_int64, C.c_int32]
        L.vshe_she_solve.argtypes = [vp, C.c_int64, C.POINTER(SolveStatsC)]
        L.vshe_she_finish.argtypes = [vp, C.c_int64, f64p]
        L.vshe_she_run.argtypes = [vp, C.c_int64, C.POINTER(SolveStatsC), f64p]
        L.vshe_she_results.argtypes = [vp, C.c_int64, f64p, f64p, f64p]
        L.vshe_she_export.argtypes = [vp, C.c_int64, C.c_int32, i64p, i32p, f64p, f64p]
        L.vshe_she_scaling.argtypes = [vp, C.c_int64, f64p, f64p]
        L.vshe_she_blocks.argtypes = [vp, C.c_int64, i64p]
        L.vshe_she_free.argtypes = [vp, C.c_int64]
        L.vshe_she_bench.argtypes = [vp, C.c_int64, C.c_int32, C.c_int32, f64p, C.POINTER(SolveStatsC)]
        L.vshe_she_run_batch.argtypes = [vp, C.c_int32, i64p, C.POINTER(SolveStatsC), f64p, f64p]
        L._she_ready = True
    return L


def coupling_tables(L):
    """Coupling tables a_{x,y,z}, b_{x,y,z} of order L from the library's quadrature (no GPU needed)."""
    from .abi import Coupling
    D = (L + 1) ** 2
    out = np.zeros((6, D, D))
    rc = _she_lib().vshe_coupling_tables_compute(L, ptr(out, C.c_double))
    if rc:
        raise VsheError(rc, "vshe_coupling_tables_compute")
    return Coupling(L, out)


def she_plan(dev, cfg, coupling=None, **opts):
    """vshe_she_plan: the host set-up of a SHE problem alone (no GPU) -> dict of the sizes and the
    footprint bound the library admits the problem by."""
    from .abi import DeviceDesc, she_config_c
    L = _she_lib()
    L.vshe_she_plan.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(SheInfoC)]
    desc = DeviceDesc(dev)
    cfgc = she_config_c(cfg)
    cpl = coupling if coupling is not None else coupling_tables(cfg.max_expansion_order)
    o, keep = make_opts(**opts) if opts else (None, None)
    inf = SheInfoC()
    rc = L.vshe_she_plan(C.byref(desc.c), C.byref(cfgc), C.byref(cpl.c), C.byref(o) if o is not None else None, C.byref(inf))
    if rc:
        raise VsheError(rc, "vshe_she_plan")
    keys = ("n_energies", "n_even", "n_odd", "n_cells", "n_facets", "n_contacts", "hbar_omega", "bytes_estimate")
    return {k: getattr(inf, k) for k in keys}


def she_space(dev, cfg, coupling=None):
    """vshe_she_space: the (x, H) space of the host set-up (no GPU) -> dict of "energies" (N_H),
    per cell and energy (shape (n_cells, N_H)) "even_index" (first even unknown in x_full, -1:
    none), "even_order", "kinetic_energy" and "density_of_states", per facet and energy
    "odd_index" and "odd_order"."""
    from .abi import DeviceDesc, she_config_c
    info = she_plan(dev, cfg, coupling)
    L = _she_lib()
    L.vshe_she_space.argtypes = [C.c_void_p] * 10
    desc = DeviceDesc(dev)
    cfgc = she_config_c(cfg)
    cpl = coupling if coupling is not None else coupling_tables(cfg.max_expansion_order)
    nh, nc, nf = info["n_energies"], info["n_cells"], info["n_facets"]
    out = {"energies": np.zeros(nh), "even_index": np.zeros((nc, nh), np.int64), "even_order": np.zeros((nc, nh), np.int32),
           "kinetic_energy": np.zeros((nc, nh)), "density_of_states": np.zeros((nc, nh)),
           "odd_index": np.zeros((nf, nh), np.int64), "odd_order": np.zeros((nf, nh), np.int32)}
    order = ("energies", "even_index", "even_order", "kinetic_energy", "density_of_states", "odd_index", "odd_order")
    rc = L.vshe_she_space(C.byref(desc.c), C.byref(cfgc), C.byref(cpl.c), *[out[k].ctypes.data for k in order])
    if rc:
        raise VsheError(rc, "vshe_she_space")
    return out


def she_node_order(dev, cfg, coupling=None, fill_level=0):
    """vshe_she_node_order: the multicolour order of the reduced rows the SHE pipeline uses (host
    only) -> (perm, colour), n_even entries each."""
    from .abi import DeviceDesc, she_config_c
    info = she_plan(dev, cfg, coupling)
    L = _she_lib()
    L.vshe_she_node_order.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p]
    desc = DeviceDesc(dev)
    cfgc = she_config_c(cfg)
    cpl = coupling if coupling is not None else coupling_tables(cfg.max_expansion_order)
    perm = np.zeros(info["n_even"], np.int32)
    colour = np.zeros(info["n_even"], np.int32)
    rc = L.vshe_she_node_order(C.byref(desc.c), C.byref(cfgc), C.byref(cpl.c), int(fill_level), perm.ctypes.data, colour.ctypes.data)
    if rc:
        raise VsheError(rc, "vshe_she_node_order")
    return perm, colour


class PoissonStatsC(C.Structure):
    _fields_ = [("status", C.c_int32), ("iterations", C.c_int32), ("rel_residual", C.c_double),
                ("rhs_norm", C.c_double), ("update_norm", C.c_double), ("n_unknowns", C.c_int64)]


class PoissonProblem:
    """The outer loop's Gummel update of the potential on the device (vshe_poisson_*)."""

    def __init__(self, ctx: Context, dev, facet_centroid=None, **opts):
        from .abi import DeviceDesc
        from .devices import facet_centres
        L = lib()
        i64p, i32p, f64p = C.POINTER(C.c_int64), C.POINTER(C.c_int32), C.POINTER(C.c_double)
        L.vshe_poisson_create.argtypes = [C.c_void_p, C.c_void_p, f64p, C.c_void_p, i64p]
        L.vshe_poisson_update.argtypes = [C.c_void_p, C.c_int64, f64p, f64p, f64p, C.c_double, f64p, C.c_void_p]
        L.vshe_poisson_export.argtypes = [C.c_void_p, C.c_int64, i64p, i32p, f64p, f64p, i64p]
        L.vshe_poisson_free.argtypes = [C.c_void_p, C.c_int64]
        self.ctx, self.dev = ctx, dev
        self._desc = DeviceDesc(dev)
        self._fc = np.ascontiguousarray(facet_centres(dev) if facet_centroid is None else facet_centroid, np.float64)
        o, self._keep = make_opts(precision="fp64", **opts) if opts else (None, None)
        h = C.c_int64()
        ctx._check(L.vshe_poisson_create(ctx.h, C.byref(self._desc.c), ptr(self._fc, C.c_double),
                                         C.byref(o) if o is not None else None, C.byref(h)))
        self.h = h.value

    def update(self, potential, n, p, damping=1.0):
        """-> (new potential, stats dict); raises on a failed solve."""
        nc = self.dev.n_cells
        psi = np.ascontiguousarray(potential, np.float64)
        nn = np.ascontiguousarray(n, np.float64)
        pp = np.ascontiguousarray(p, np.float64)
        out = np.zeros(nc)
        st = PoissonStatsC()
        rc = lib().vshe_poisson_update(self.ctx.h, self.h, ptr(psi, C.c_double), ptr(nn, C.c_double), ptr(pp, C.c_double),
                                       float(damping), ptr(out, C.c_double), C.byref(st))
        self.ctx._check(rc)
        return out, {k: getattr(st, k) for k, _ in PoissonStatsC._fields_}

    def export(self):
        """-> (row_ptr, col, val, rhs) of the last assembled system."""
        nnz = C.c_int64()
        L = lib()
        self.ctx._check(L.vshe_poisson_export(self.ctx.h, self.h, None, None, None, None, C.byref(nnz)))
        nu = int(np.sum(self.dev.contact_id < 0))
        rp = np.zeros(nu + 1, np.int64)
        ci = np.zeros(nnz.value, np.int32)
        v = np.zeros(nnz.value)
        b = np.zeros(nu)
        self.ctx._check(L.vshe_poisson_export(self.ctx.h, self.h, ptr(rp, C.c_int64), ptr(ci, C.c_int32), ptr(v, C.c_double),
                                              ptr(b, C.c_double), C.byref(nnz)))
        return rp, ci, v, b

    def free(self):
        if self.h:
            lib().vshe_poisson_free(self.ctx.h, self.h)
            self.h = 0


class GummelOptsC(C.Structure):
    _fields_ = [("max_iters", C.c_int32), ("tol", C.c_double), ("damping", C.c_double)]


class GummelStatsC(C.Structure):
    _fields_ = [("status", C.c_int32), ("iterations", C.c_int32), ("potential_increment", C.c_double),
                ("rhs_norm", C.c_double), ("initial_rhs_norm", C.c_double), ("she_iterations", C.c_int64)]


def gummel_solve(ctx: Context, dev, cfg, density0, p0, coupling=None, facet_centroid=None, max_iters=100, tol=1e-8,
                 damping=0.3, she_tol=1e-12, she_max_iters=20000, **she_opts):
    """Self-consistent electron SHE + Poisson (vshe_gummel_solve) -> (potential, density, currents,
    history (iterations x 3: ||b_Poisson||, ||dpsi||, SHE iterations), stats dict)."""
    from .abi import DeviceDesc, she_config_c
    from .devices import facet_centres
    L = _she_lib()
    f64p = C.POINTER(C.c_double)
    L.vshe_gummel_solve.argtypes = [C.c_void_p, C.c_void_p, f64p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                    f64p, f64p, f64p, f64p, f64p, f64p, C.c_void_p]
    desc = DeviceDesc(dev)
    cfgc = she_config_c(cfg)
    cpl = coupling if coupling is not None else coupling_tables(cfg.max_expansion_order)
    fc = np.ascontiguousarray(facet_centres(dev) if facet_centroid is None else facet_centroid, np.float64)
    o, keep = make_opts(tol=she_tol, max_iters=she_max_iters, **she_opts)
    g = GummelOptsC(int(max_iters), float(tol), float(damping))
    n0 = np.ascontiguousarray(density0, np.float64)
    pp = np.ascontiguousarray(p0, np.float64)
    psi = np.zeros(dev.n_cells)
    dens = np.zeros(dev.n_cells)
    cur = np.zeros(max(dev.n_contacts, 1))
    hist = np.zeros(3 * int(max_iters))
    st = GummelStatsC()
    rc = L.vshe_gummel_solve(ctx.h, C.byref(desc.c), ptr(fc, C.c_double), C.byref(cfgc), C.byref(cpl.c), C.byref(o), C.byref(g),
                             ptr(n0, C.c_double), ptr(pp, C.c_double), ptr(psi, C.c_double), ptr(dens, C.c_double),
                             ptr(cur, C.c_double), ptr(hist, C.c_double), C.byref(st))
    stats = {k: getattr(st, k) for k, _ in GummelStatsC._fields_}
    if rc and rc != -6:
        ctx._check(rc)
    stats["rc"] = rc
    return psi, dens, cur[:dev.n_contacts], hist.reshape(-1, 3)[:stats["iterations"]], stats


class SheProblem:
    """A SHE problem assembled, eliminated, normalised and solved on the device (vshe_she_*)."""

    def __init__(self, ctx: Context, dev, cfg, coupling=None, **opts):
        from .abi import DeviceDesc, she_config_c
        L = _she_lib()
        self.ctx = ctx
        self.dev = dev
        self._desc = DeviceDesc(dev)
        self._cfg = she_config_c(cfg)
        self._cpl = coupling if coupling is not None else coupling_tables(cfg.max_expansion_order)
        o, self._keep = make_opts(**opts)
        h = C.c_int64()
        rc = L.vshe_she_create(ctx.h, C.byref(self._desc.c), C.byref(self._cfg), C.byref(self._cpl.c), C.byref(o), C.byref(h))
        ctx._check(rc)
        self.h = h.value
        self.info = self.get_info()

    def get_info(self):
        inf = SheInfoC()
        self.ctx._check(_she_lib().vshe_she_info_get(self.ctx.h, self.h, C.byref(inf)))
        return {k: getattr(inf, k) for k, _ in SheInfoC._fields_}

    def free(self):
        if self.h:
            _she_lib().vshe_she_free(self.ctx.h, self.h)
            self.h = 0

    def assemble(self, upto=3):
        self.ctx._check(_she_lib().vshe_she_assemble(self.ctx.h, self.h, upto))

    def solve(self):
        st = SolveStatsC()
        rc = _she_lib().vshe_she_solve(self.ctx.h, self.h, C.byref(st))
        if rc and rc != -6:
            self.ctx._check(rc)
        return stats_dict(st)

    def finish(self):
        r = C.c_double()
        self.ctx._check(_she_lib().vshe_she_finish(self.ctx.h, self.h, C.byref(r)))
        return r.value

    def run(self):
        st = SolveStatsC()
        r = C.c_double()
        rc = _she_lib().vshe_she_run(self.ctx.h, self.h, C.byref(st), C.byref(r))
        if rc and rc != -6:
            self.ctx._check(rc)
        return stats_dict(st), r.value

    def bench(self, warmup, steps):
        """Per-run device times (ms) of assemble + solve + finish, and the last run's stats."""
        ms = np.zeros(steps)
        st = SolveStatsC()
        rc = _she_lib().vshe_she_bench(self.ctx.h, self.h, warmup, steps, ptr(ms, C.c_double), C.byref(st))
        if rc and rc != -6:
            self.ctx._check(rc)
        return ms, stats_dict(st)

    def results(self):
        nfull = self.info["n_even"] + self.info["n_odd"]
        x = np.zeros(nfull)
        dens = np.zeros(self.dev.n_cells)
        cur = np.zeros(max(self.info["n_contacts"], 1))
        self.ctx._check(_she_lib().vshe_she_results(self.ctx.h, self.h, ptr(x, C.c_double), ptr(dens, C.c_double), ptr(cur, C.c_double)))
        return x, dens, cur[:self.info["n_contacts"]]

    def export(self, which):
        """which: 'full' or 'reduced' -> (row_ptr, col, val, rhs) of the current device state."""
        w = 0 if which == "full" else 1
        n = self.info["n_even"] + self.info["n_odd"] if w == 0 else self.info["n_even"]
        nnz = self.info["nnz_full"] if w == 0 else self.info["nnz_reduced"]
        rp = np.zeros(n + 1, np.int64)
        ci = np.zeros(nnz, np.int32)
        v = np.zeros(nnz)
        b = np.zeros(n)
        self.ctx._check(_she_lib().vshe_she_export(self.ctx.h, self.h, w, ptr(rp, C.c_int64), ptr(ci, C.c_int32), ptr(v, C.c_double), ptr(b, C.c_double)))
        return rp, ci, v, b

    def blocks(self):
        """Energy-slab row offsets of the reduced system (n_energies + 1)."""
        b = np.zeros(self.info["n_energies"] + 1, np.int64)
        self.ctx._check(_she_lib().vshe_she_blocks(self.ctx.h, self.h, ptr(b, C.c_int64)))
        return b

    def scaling(self):
        n = self.info["n_even"]
        s = np.zeros(n)
        f = np.zeros(n)
        self.ctx._check(_she_lib().vshe_she_scaling(self.ctx.h, self.h, ptr(s, C.c_double), ptr(f, C.c_double)))
        return s, f


def she_run_batch(ctx: Context, problems):
    """Assemble, solve (one batch) and finish several SHE problems: per-problem stats, full
    residuals, and the device time of the whole call in ms."""
    hs = np.array([p.h for p in problems], np.int64)
    st = (SolveStatsC * len(problems))()
    fr = np.zeros(len(problems))
    ms = C.c_double()
    rc = _she_lib().vshe_she_run_batch(ctx.h, len(problems), ptr(hs, C.c_int64), st, ptr(fr, C.c_double), C.byref(ms))
    if rc and rc != -6:
        ctx._check(rc)
    return [stats_dict(s) for s in st], fr, ms.value


# ---------------------------------------------------------------- served stream
class ServerOptsC(C.Structure):
    _fields_ = [("hbm_budget", C.c_size_t), ("max_active", C.c_int32), ("solve", SolveOptsC), ("stagnation_iters", C.c_int32)]


class ServerResultC(C.Structure):
    _fields_ = [("status", C.c_int32), ("iterations", C.c_int32), ("refinements", C.c_int32),
                ("rel_residual", C.c_double), ("full_residual", C.c_double), ("queue_ms", C.c_double),
                ("latency_ms", C.c_double), ("n_unknowns", C.c_int64)]


class Server:
    """Continuous-batching request loop on one context (vshe_server_*)."""

    def __init__(self, ctx: Context, hbm_budget=0, max_active=0, stagnation_iters=0, **solve):
        L = lib()
        L.vshe_server_create.argtypes = [C.c_void_p, C.POINTER(ServerOptsC), C.POINTER(C.c_void_p)]
        L.vshe_server_submit.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(SolveOptsC), C.POINTER(C.c_int64)]
        L.vshe_server_wait.argtypes = [C.c_void_p, C.c_int64, C.c_double, C.POINTER(ServerResultC), C.POINTER(C.c_double), C.POINTER(C.c_double)]
        L.vshe_server_destroy.argtypes = [C.c_void_p]
        self.ctx = ctx
        o = ServerOptsC()
        o.hbm_budget = int(hbm_budget)
        o.max_active = int(max_active)
        o.stagnation_iters = int(stagnation_iters)
        so, self._keep = make_opts(**solve)
        o.solve = so
        h = C.c_void_p()
        ctx._check(L.vshe_server_create(ctx.h, C.byref(o), C.byref(h)))
        self.h = h
        self._meta = {}

    def submit(self, dev, cfg, coupling=None, **solve):
        from .abi import DeviceDesc, she_config_c
        desc = DeviceDesc(dev)
        cfgc = she_config_c(cfg)
        cpl = coupling if coupling is not None else coupling_tables(cfg.max_expansion_order)
        o = None
        if solve:
            o, _ = make_opts(**solve)
        t = C.c_int64()
        rc = lib().vshe_server_submit(self.h, C.byref(desc.c), C.byref(cfgc), C.byref(cpl.c), C.byref(o) if o is not None else None, C.byref(t))
        if rc:
            raise VsheError(rc, "vshe_server_submit")
        self._meta[t.value] = (dev.n_cells, dev.n_contacts)
        return t.value

    def wait(self, ticket, timeout_ms=-1.0, raise_on_error=True):
        """-> (result dict, densities, currents); raises on a failed request (other than not
        converged) unless raise_on_error is False, in which case the result carries the status."""
        nc, ncont = self._meta.pop(ticket)
        r = ServerResultC()
        dens = np.zeros(nc)
        cur = np.zeros(max(ncont, 1))
        rc = lib().vshe_server_wait(self.h, ticket, float(timeout_ms), C.byref(r), ptr(dens, C.c_double), ptr(cur, C.c_double))
        res = {k: getattr(r, k) for k, _ in ServerResultC._fields_}
        if rc and rc != -6 and raise_on_error:
            raise VsheError(rc, "served request %d failed (%s)" % (ticket, ERRORS.get(rc, "?")))
        if rc:
            res["status"] = rc
        return res, dens, cur[:ncont]

    def close(self):
        if getattr(self, "h", None):
            lib().vshe_server_destroy(self.h)
            self.h = None

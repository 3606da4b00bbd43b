"""ctypes binding of the CPU oracle (oracle/she_oracle.cpp).

TEST INFRASTRUCTURE: imported only by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py, always as the checker or the timed CPU
reference, never as part of the product path.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB = os.path.join(HERE, "_build", "libvshe_oracle.so")
LIB_MT = os.path.join(HERE, "_build", "libvshe_oracle_mt.so")
sys.path.insert(0, os.path.join(ROOT, "viennashe-dev_b200"))
from vshe.abi import DeviceDesc, she_config_c, Coupling, ptr  # noqa: E402

i32p = C.POINTER(C.c_int32)
i64p = C.POINTER(C.c_int64)
f64p = C.POINTER(C.c_double)

_lib = None
_lib_mt = None


def build():
    subprocess.check_call(["sh", os.path.join(HERE, "build.sh")])


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        L = C.CDLL(LIB)
        L.vsheo_create.restype = C.c_void_p
        L.vsheo_create.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_char_p, C.c_int]
        L.vsheo_destroy.argtypes = [C.c_void_p]
        L.vsheo_info.argtypes = [C.c_void_p, i64p]
        L.vsheo_energies.argtypes = [C.c_void_p, f64p, f64p, f64p, f64p]
        L.vsheo_mapping.argtypes = [C.c_void_p, i64p, i64p, i32p, i32p, f64p]
        L.vsheo_matrix.argtypes = [C.c_void_p, C.c_int, i64p, i32p, f64p, f64p]
        L.vsheo_scaling.argtypes = [C.c_void_p, f64p, f64p]
        L.vsheo_blocks.argtypes = [C.c_void_p, i64p]
        L.vsheo_finish.argtypes = [C.c_void_p, f64p, f64p, f64p, f64p, C.c_int, f64p]
        L.vsheo_csr_solve.argtypes = [C.c_int64, i64p, i32p, f64p, f64p, f64p, C.c_int, C.c_int, C.c_double,
                                      C.c_int64, i64p, C.c_double, C.c_int, i32p, f64p, f64p, f64p]
        L.vsheo_ilu0_values.argtypes = [C.c_int64, i64p, i32p, f64p, C.c_int64, i64p, f64p]
        L.vsheo_ilu0_apply.argtypes = [C.c_int64, i64p, i32p, f64p, C.c_int64, i64p, f64p, f64p]
        L.vsheo_dense_solve.argtypes = [C.c_int64, i64p, i32p, f64p, f64p, f64p]
        L.vsheo_spmv.argtypes = [C.c_int64, i64p, i32p, f64p, f64p, f64p]
        L.vsheo_harmonics.argtypes = [C.c_int, C.c_int, i64p, C.c_int]
        L.vsheo_harmonics.restype = C.c_int
        L.vsheo_bench_serial.argtypes = [C.c_int64, i64p, i32p, f64p, f64p, C.c_int, f64p, f64p, f64p]
        _lib = L
    return _lib


class CSR:
    def __init__(self, rp, ci, v, rhs=None):
        self.rp = np.ascontiguousarray(rp, np.int64)
        self.ci = np.ascontiguousarray(ci, np.int32)
        self.v = np.ascontiguousarray(v, np.float64)
        self.rhs = None if rhs is None else np.ascontiguousarray(rhs, np.float64)

    @property
    def n(self):
        return len(self.rp) - 1

    @property
    def nnz(self):
        return int(self.rp[-1])

    def dense(self):
        A = np.zeros((self.n, self.n))
        for i in range(self.n):
            A[i, self.ci[self.rp[i]:self.rp[i + 1]]] += self.v[self.rp[i]:self.rp[i + 1]]
        return A


class OracleProblem:
    """setup + assembly + elimination + scaling/normalisation on the CPU."""

    def __init__(self, dev, cfg, coupling: Coupling):
        self.dev = dev
        self._desc = DeviceDesc(dev)
        self._cfg = she_config_c(cfg)
        self._cpl = coupling
        err = C.create_string_buffer(512)
        h = lib().vsheo_create(C.byref(self._desc.c), C.byref(self._cfg), C.byref(coupling.c), err, 512)
        if not h:
            raise RuntimeError("oracle: " + err.value.decode())
        self.h = h
        info = np.zeros(9, np.int64)
        lib().vsheo_info(h, ptr(info, C.c_int64))
        self.NH, self.n_even, self.n_odd = int(info[0]), int(info[1]), int(info[2])
        self.nnz = {0: int(info[3]), 1: int(info[4]), 2: int(info[5]), 3: int(info[6])}

    def __del__(self):
        try:
            if getattr(self, "h", None):
                lib().vsheo_destroy(self.h)
        except Exception:
            pass

    def energies(self):
        H = np.zeros(self.NH)
        sc = np.zeros(self.dev.n_cells)
        sf = np.zeros(self.dev.n_facets)
        w = np.zeros(1)
        lib().vsheo_energies(self.h, ptr(H, C.c_double), ptr(sc, C.c_double), ptr(sf, C.c_double), ptr(w, C.c_double))
        return H, sc, sf, float(w[0])

    def mapping(self):
        nc, nf, NH = self.dev.n_cells, self.dev.n_facets, self.NH
        ic = np.zeros(nc * NH, np.int64)
        jf = np.zeros(nf * NH, np.int64)
        oc = np.zeros(nc * NH, np.int32)
        of = np.zeros(nf * NH, np.int32)
        bc = np.zeros(nc * NH)
        lib().vsheo_mapping(self.h, ptr(ic, C.c_int64), ptr(jf, C.c_int64), ptr(oc, C.c_int32), ptr(of, C.c_int32), ptr(bc, C.c_double))
        return ic, jf, oc, of, bc

    def matrix(self, which):
        n = self.n_even + self.n_odd if which in (0, 1) else self.n_even
        nnz = self.nnz[which]
        rp = np.zeros(n + 1, np.int64)
        ci = np.zeros(nnz, np.int32)
        v = np.zeros(nnz)
        b = np.zeros(n)
        lib().vsheo_matrix(self.h, which, ptr(rp, C.c_int64), ptr(ci, C.c_int32), ptr(v, C.c_double), ptr(b, C.c_double))
        return CSR(rp, ci, v, b)

    def scaling(self):
        s = np.zeros(self.n_even)
        f = np.zeros(self.n_even)
        lib().vsheo_scaling(self.h, ptr(s, C.c_double), ptr(f, C.c_double))
        return s, f

    def blocks(self):
        b = np.zeros(self.NH + 1, np.int64)
        lib().vsheo_blocks(self.h, ptr(b, C.c_int64))
        return b

    def finish(self, x_red):
        x_red = np.ascontiguousarray(x_red, np.float64)
        xf = np.zeros(self.n_even + self.n_odd)
        dens = np.zeros(self.dev.n_cells)
        nct = max(self.dev.n_contacts, 1)
        cur = np.zeros(nct)
        res = np.zeros(1)
        lib().vsheo_finish(self.h, ptr(x_red, C.c_double), ptr(xf, C.c_double), ptr(dens, C.c_double),
                           ptr(cur, C.c_double), nct, ptr(res, C.c_double))
        return xf, dens, cur, float(res[0])


def poisson_assemble(dev, facet_centroid, psi, n, p) -> CSR:
    """The Gummel-linearised Poisson system of the reference (poisson_oracle.cpp:
    viennashe/assemble.hpp:165-345) for the potential psi and densities n, p; rows are the
    non-contact cells in cell order."""
    L = lib()
    if not getattr(L, "_poisson_ready", False):
        L.vsheo_poisson_assemble.restype = C.c_int64
        L.vsheo_poisson_assemble.argtypes = [C.c_void_p, f64p, f64p, f64p, f64p, C.c_int64, i64p, i32p, f64p, f64p, i64p]
        L._poisson_ready = True
    desc = DeviceDesc(dev)
    fc = np.ascontiguousarray(facet_centroid, np.float64)
    psi = np.ascontiguousarray(psi, np.float64)
    n = np.ascontiguousarray(n, np.float64)
    p = np.ascontiguousarray(p, np.float64)
    nc = dev.n_cells
    cap = nc * (2 * dev.dim + 2) + 16
    rp = np.zeros(nc + 1, np.int64)
    ci = np.zeros(cap, np.int32)
    v = np.zeros(cap)
    b = np.zeros(nc)
    nnz = np.zeros(1, np.int64)
    nu = L.vsheo_poisson_assemble(C.byref(desc.c), ptr(fc, C.c_double), ptr(psi, C.c_double), ptr(n, C.c_double),
                                  ptr(p, C.c_double), cap, ptr(rp, C.c_int64), ptr(ci, C.c_int32), ptr(v, C.c_double),
                                  ptr(b, C.c_double), ptr(nnz, C.c_int64))
    if nu < 0:
        raise ValueError("poisson_assemble: capacity or material error")
    k = int(nnz[0])
    return CSR(rp[:nu + 1], ci[:k], v[:k], b[:nu])


def poisson_update(dev, facet_centroid, psi, n, p, damping=1.0, tol=1e-13):
    """One Gummel step of the potential (viennashe/simulator.hpp:1029-1052, 606-647): assemble,
    solve A dpsi = b (the oracle's ILU(0) + BiCGStab), psi_new = psi + dpsi on unknown cells and
    the description's potential on contact cells, then (1 - damping) psi + damping psi_new.
    -> (psi_out, dpsi, A)."""
    A = poisson_assemble(dev, facet_centroid, psi, n, p)
    if np.any(A.rhs != 0.0):
        dpsi, st = csr_solve(A, A.rhs, precond=1, tol=tol, maxit=20000)
        if st["rc"] != 0:
            raise RuntimeError("oracle Poisson solve: %s" % st)
    else:
        dpsi = np.zeros(A.n)
    psi = np.asarray(psi, np.float64)
    unk = dev.contact_id < 0
    new = np.array(dev.potential, np.float64)
    new[unk] = psi[unk] + dpsi
    return psi * (1.0 - damping) + new * damping, dpsi, A


def gummel_solve(dev, cfg, cpl, n0, p0, max_iters=100, tol=1e-8, damping=0.3, she_tol=1e-12):
    """The electron SHE + Poisson Gummel loop of viennashe/simulator.hpp:895-1130 on the oracle:
    the Poisson step (poisson_update), the oracle SHE for the new potential, the logarithmic
    density damping of simulator.hpp:560-577 and the reference's stopping rules.
    -> (potential, density, currents, history (||b||, ||dpsi||, SHE iterations) per iteration)."""
    import dataclasses
    from vshe import devices as D
    fc = D.facet_centres(dev)
    psi = np.array(dev.potential, np.float64)
    n = np.array(n0, np.float64)
    p = np.array(p0, np.float64)
    semi = (dev.contact_id < 0) & (dev.cell_material == D.SI)
    no_damping = break_after = False
    initial = 0.0
    hist, cur = [], None
    for it in range(1, max_iters + 1):
        if it == max_iters:
            no_damping = True
        alpha = 1.0 if no_damping else damping
        A = poisson_assemble(dev, fc, psi, n, p)
        res, psi, dpsi = float(np.linalg.norm(A.rhs)), *poisson_update(dev, fc, psi, n, p, damping=alpha)[:2]
        P = OracleProblem(dataclasses.replace(dev, potential=psi.copy()), cfg, cpl)
        M = P.matrix(3)
        x, st = csr_solve(M, M.rhs, precond=1, tol=she_tol, maxit=20000)
        if st["rc"] != 0:
            raise RuntimeError("oracle SHE solve: %s" % st)
        _, dens, cur, _ = P.finish(x)
        if no_damping:
            n[semi] = dens[semi]
        else:
            nv = np.maximum(dens[semi], n[semi] * 1e-10)
            n[semi] = np.power(n[semi], 1.0 - alpha) * np.power(nv, alpha)
        inc = float(np.linalg.norm(dpsi))
        hist.append((res, inc, st["iters"]))
        if break_after or res == 0.0:
            break
        if it == 1:
            initial = res
        elif res / initial < 1e-10 or inc < tol:
            no_damping = break_after = True
    return psi, n, cur, np.array(hist)


def csr_solve(A: CSR, b, precond=1, tol=1e-10, maxit=5000, ilut_p=20, ilut_tau=1e-3, blocks=None):
    b = np.ascontiguousarray(b, np.float64)
    x = np.zeros(A.n)
    it = np.zeros(1, np.int32)
    rr = np.zeros(1)
    ts = np.zeros(1)
    tv = np.zeros(1)
    bp = None if blocks is None else np.ascontiguousarray(blocks, np.int64)
    nb = 0 if bp is None else len(bp) - 1
    rc = lib().vsheo_csr_solve(A.n, ptr(A.rp, C.c_int64), ptr(A.ci, C.c_int32), ptr(A.v, C.c_double),
                               ptr(b, C.c_double), ptr(x, C.c_double), precond, ilut_p, ilut_tau, nb,
                               None if bp is None else ptr(bp, C.c_int64), tol, maxit,
                               ptr(it, C.c_int32), ptr(rr, C.c_double), ptr(ts, C.c_double), ptr(tv, C.c_double))
    return x, dict(rc=rc, iters=int(it[0]), relres=float(rr[0]), t_setup=float(ts[0]), t_solve=float(tv[0]))


def iluk_csr(A: CSR, fill_level, blocks=None):
    """ILU(k) factor (levels of fill <= k, Saad Alg. 10.5 + IKJ) as a CSR (rp, ci, values)."""
    bp = None if blocks is None else np.ascontiguousarray(blocks, np.int64)
    nb = 0 if bp is None else len(bp) - 1
    L = lib()
    L.vsheo_iluk_csr.argtypes = [C.c_int64, C.POINTER(C.c_int64), C.POINTER(C.c_int32), C.POINTER(C.c_double), C.c_int32,
                                 C.c_int64, C.POINTER(C.c_int64), C.POINTER(C.c_int64), C.POINTER(C.c_int64),
                                 C.POINTER(C.c_int32), C.POINTER(C.c_double)]
    nnz = np.zeros(1, np.int64)
    args = (A.n, ptr(A.rp, C.c_int64), ptr(A.ci, C.c_int32), ptr(A.v, C.c_double), int(fill_level), nb,
            None if bp is None else ptr(bp, C.c_int64), ptr(nnz, C.c_int64))
    if L.vsheo_iluk_csr(*args, None, None, None):
        raise RuntimeError("oracle iluk failed")
    rp = np.zeros(A.n + 1, np.int64)
    ci = np.zeros(int(nnz[0]), np.int32)
    lu = np.zeros(int(nnz[0]))
    if L.vsheo_iluk_csr(*args, ptr(rp, C.c_int64), ptr(ci, C.c_int32), ptr(lu, C.c_double)):
        raise RuntimeError("oracle iluk failed")
    return rp, ci, lu


def _blocks_arg(blocks):
    bp = None if blocks is None else np.ascontiguousarray(blocks, np.int64)
    return bp, (0 if bp is None else len(bp) - 1), (None if bp is None else ptr(bp, C.c_int64))


def ilut_csr(A: CSR, p, tau, blocks=None):
    """ILUT(p, tau) factor (Saad Alg. 10.6) as one CSR (rp, ci, values), columns ascending;
    restricted to the blocks when they are given."""
    L = lib()
    L.vsheo_ilut_csr.argtypes = [C.c_int64, C.POINTER(C.c_int64), C.POINTER(C.c_int32), C.POINTER(C.c_double), C.c_int32,
                                 C.c_double, C.c_int64, C.POINTER(C.c_int64), C.POINTER(C.c_int64), C.POINTER(C.c_int64),
                                 C.POINTER(C.c_int32), C.POINTER(C.c_double)]
    nnz = np.zeros(1, np.int64)
    bp, nb, bptr = _blocks_arg(blocks)
    args = (A.n, ptr(A.rp, C.c_int64), ptr(A.ci, C.c_int32), ptr(A.v, C.c_double), int(p), float(tau), nb, bptr,
            ptr(nnz, C.c_int64))
    if L.vsheo_ilut_csr(*args, None, None, None):
        raise RuntimeError("oracle ilut failed")
    rp = np.zeros(A.n + 1, np.int64)
    ci = np.zeros(int(nnz[0]), np.int32)
    lu = np.zeros(int(nnz[0]))
    if L.vsheo_ilut_csr(*args, ptr(rp, C.c_int64), ptr(ci, C.c_int32), ptr(lu, C.c_double)):
        raise RuntimeError("oracle ilut failed")
    return rp, ci, lu


def ilut_passed(A: CSR, p, tau, blocks=None):
    """Per row, the columns whose entries passed ILUT(p, tau)'s tau test before the p-largest
    rule (CSR pattern rp, ci); restricted to the blocks when they are given."""
    L = lib()
    L.vsheo_ilut_passed.argtypes = [C.c_int64, C.POINTER(C.c_int64), C.POINTER(C.c_int32), C.POINTER(C.c_double), C.c_int32,
                                    C.c_double, C.c_int64, C.POINTER(C.c_int64), C.POINTER(C.c_int64), C.POINTER(C.c_int64),
                                    C.POINTER(C.c_int32)]
    nnz = np.zeros(1, np.int64)
    bp, nb, bptr = _blocks_arg(blocks)
    args = (A.n, ptr(A.rp, C.c_int64), ptr(A.ci, C.c_int32), ptr(A.v, C.c_double), int(p), float(tau), nb, bptr,
            ptr(nnz, C.c_int64))
    if L.vsheo_ilut_passed(*args, None, None):
        raise RuntimeError("oracle ilut failed")
    rp = np.zeros(A.n + 1, np.int64)
    ci = np.zeros(int(nnz[0]), np.int32)
    if L.vsheo_ilut_passed(*args, ptr(rp, C.c_int64), ptr(ci, C.c_int32)):
        raise RuntimeError("oracle ilut failed")
    return rp, ci


def ilu0_values(A: CSR, blocks=None):
    lu = np.zeros(A.nnz)
    bp = None if blocks is None else np.ascontiguousarray(blocks, np.int64)
    nb = 0 if bp is None else len(bp) - 1
    rc = lib().vsheo_ilu0_values(A.n, ptr(A.rp, C.c_int64), ptr(A.ci, C.c_int32), ptr(A.v, C.c_double), nb,
                                 None if bp is None else ptr(bp, C.c_int64), ptr(lu, C.c_double))
    if rc:
        raise RuntimeError("oracle ilu0 failed")
    return lu


def ilu0_apply(A: CSR, lu, b, blocks=None):
    lu = np.ascontiguousarray(lu, np.float64)
    b = np.ascontiguousarray(b, np.float64)
    x = np.zeros(A.n)
    bp = None if blocks is None else np.ascontiguousarray(blocks, np.int64)
    nb = 0 if bp is None else len(bp) - 1
    lib().vsheo_ilu0_apply(A.n, ptr(A.rp, C.c_int64), ptr(A.ci, C.c_int32), ptr(lu, C.c_double), nb,
                           None if bp is None else ptr(bp, C.c_int64), ptr(b, C.c_double), ptr(x, C.c_double))
    return x


def dense_solve(A: CSR, b):
    b = np.ascontiguousarray(b, np.float64)
    x = np.zeros(A.n)
    rc = lib().vsheo_dense_solve(A.n, ptr(A.rp, C.c_int64), ptr(A.ci, C.c_int32), ptr(A.v, C.c_double), ptr(b, C.c_double), ptr(x, C.c_double))
    if rc:
        raise RuntimeError("singular")
    return x


def spmv(A: CSR, x):
    x = np.ascontiguousarray(x, np.float64)
    y = np.zeros(A.n)
    lib().vsheo_spmv(A.n, ptr(A.rp, C.c_int64), ptr(A.ci, C.c_int32), ptr(A.v, C.c_double), ptr(x, C.c_double), ptr(y, C.c_double))
    return y


def bench_serial(A: CSR, b, iters):
    b = np.ascontiguousarray(b, np.float64)
    tf = np.zeros(1)
    ti = np.zeros(1)
    rr = np.zeros(1)
    done = lib().vsheo_bench_serial(A.n, ptr(A.rp, C.c_int64), ptr(A.ci, C.c_int32), ptr(A.v, C.c_double),
                                    ptr(b, C.c_double), iters, ptr(tf, C.c_double), ptr(ti, C.c_double), ptr(rr, C.c_double))
    return dict(iters=int(done), t_factor=float(tf[0]), t_per_iter=float(ti[0]), relres=float(rr[0]))


def lib_mt():
    global _lib_mt
    if _lib_mt is None:
        if not os.path.exists(LIB_MT):
            build()
        L = C.CDLL(LIB_MT)
        L.vsheo_serial_solve_mt.argtypes = [C.c_int64, i64p, i32p, f64p, f64p, f64p, C.c_double, C.c_int32, C.c_int32, f64p, f64p]
        L.vsheo_serial_solve_mt.restype = C.c_int
        _lib_mt = L
    return _lib_mt


def serial_solve_mt(A: CSR, b, tol=1e-10, maxit=20000, threads=0, trace=False):
    """The reference's serial solver (natural-order ILU(0) + BiCGStab with r^ = r_0) on `threads`
    host threads (0: all), from x0 = 0 (serial_solver_mt.cpp).  Returns x and a dict with rc (0
    converged, 1 iteration limit, -1 breakdown, -2 a row without diagonal), iterations, the
    recursive relative residual, the factorisation and iteration seconds, the threads used and
    (trace=True) the elapsed seconds after every iteration."""
    b = np.ascontiguousarray(b, np.float64)
    x = np.zeros(A.n)
    out = np.zeros(5)
    it_s = np.zeros(maxit + 1) if trace else None
    rc = lib_mt().vsheo_serial_solve_mt(A.n, ptr(A.rp, C.c_int64), ptr(A.ci, C.c_int32), ptr(A.v, C.c_double),
                                        ptr(b, C.c_double), ptr(x, C.c_double), float(tol), int(maxit), int(threads),
                                        ptr(out, C.c_double), None if it_s is None else ptr(it_s, C.c_double))
    d = dict(rc=int(rc), iters=int(out[0]), relres=float(out[1]), t_factor=float(out[2]), t_iter=float(out[3]),
             threads=int(out[4]))
    if trace:
        d["iter_s"] = it_s[:d["iters"] + 1]
    return x, d


def golden_coupling(L):
    """The reference's tabulated coupling tables (tests/golden/coupling_L*.json)."""
    import json
    d = json.load(open(os.path.join(ROOT, "tests", "golden", "coupling_L%d.json" % L)))
    D = d["dim"]
    data = np.zeros((6, D, D))
    for t, name in enumerate(["a_x", "a_y", "a_z", "b_x", "b_y", "b_z"]):
        for r, c, v in d["entries"][name]:
            data[t, r, c] = v
    return Coupling(L, data)


def harmonics(L, kind):
    """Index sequence l*l + l + m of the reference's spherical_harmonics_iterator."""
    t = {"all": 0, "even": 1, "odd": 2}[kind]
    out = np.zeros(256, np.int64)
    k = lib().vsheo_harmonics(L, t, ptr(out, C.c_int64), 256)
    return out[:k].tolist()

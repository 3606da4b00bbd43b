"""vshe_csr_residual_noalloc: the entry point for callers that cannot allocate device memory
(their framework's allocator owns all of HBM, or cudaMalloc's device synchronisation is not
allowed in their loop).  It takes caller-owned device buffers and keeps its scratch in a fixed
array inside the library, so the test brings its own device buffers (torch tensors, standing in
for the caller's allocator) and checks, on two calls in a row, that r = b - A x and the norms
agree with what the library's allocating entry point vshe_system_spmv gives, and with the CPU
oracle's SpMV: b - y with y = A x within the SpMV parity bar (1e-13 of max|b|), and the norms to
1e-12 relative.  The calls run once on the default stream with a synchronisation after each, and
once queued back to back on a caller's own stream (the ordering the entry point documents for
calls on one stream), checked after both.

This file is collected last, so a run that stops at the first failure has run every other test
before it; it also passes on its own in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

from vshe import gpu
import cases

pytestmark = pytest.mark.gpu


def _lib():
    L = gpu.lib()
    L.vshe_csr_residual_noalloc.argtypes = [C.c_int64, C.c_int64] + [C.c_void_p] * 8
    L.vshe_csr_residual_noalloc.restype = C.c_int
    return L


def test_residual_noalloc_matches_allocating_entry_point(gpu_ctx):
    import torch
    dev, cfg = cases.bar_small(L=3, nx=12, ny=5, n_energies=30)
    A = cases.oracle_problem(dev, cfg).matrix(3)
    rng = np.random.default_rng(11)
    x = rng.standard_normal(A.n)
    b = A.rhs + rng.standard_normal(A.n)
    # the existing entry point: y = A x through a resident system (allocates inside the library)
    S = gpu_ctx.system(A.rp, A.ci, A.v, b, precision="fp64")
    try:
        y = S.spmv(x, "fp64")
    finally:
        S.free()
    r_ref = b - y
    n2_ref = np.array([r_ref @ r_ref, b @ b])
    import oracle_api as O
    assert np.max(np.abs((b - O.spmv(A, x)) - r_ref)) <= 1e-13 * np.max(np.abs(b))

    cuda = torch.device("cuda", 0)
    d_rp = torch.from_numpy(np.ascontiguousarray(A.rp, np.int64)).to(cuda)
    d_ci = torch.from_numpy(np.ascontiguousarray(A.ci, np.int32)).to(cuda)
    d_v = torch.from_numpy(np.ascontiguousarray(A.v, np.float64)).to(cuda)
    d_x = torch.from_numpy(x).to(cuda)
    d_b = torch.from_numpy(b).to(cuda)
    L = _lib()
    for call in range(2):
        d_r = torch.full((A.n,), float("nan"), dtype=torch.float64, device=cuda)
        d_n2 = torch.full((2,), float("nan"), dtype=torch.float64, device=cuda)
        torch.cuda.synchronize()
        rc = L.vshe_csr_residual_noalloc(A.n, A.nnz, d_rp.data_ptr(), d_ci.data_ptr(), d_v.data_ptr(), d_x.data_ptr(),
                                         d_b.data_ptr(), d_r.data_ptr(), d_n2.data_ptr(), None)
        assert rc == 0, gpu.lib().vshe_errstr(rc)
        torch.cuda.synchronize()
        r = d_r.cpu().numpy()
        n2 = d_n2.cpu().numpy()
        assert np.max(np.abs(r - r_ref)) <= 1e-13 * np.max(np.abs(b)), call
        assert np.all(np.abs(n2 - n2_ref) <= 1e-12 * n2_ref), (call, n2, n2_ref)
    # two calls queued on the caller's stream without a synchronisation between them
    stream = torch.cuda.Stream(device=cuda)
    outs = [(torch.full((A.n,), float("nan"), dtype=torch.float64, device=cuda),
             torch.full((2,), float("nan"), dtype=torch.float64, device=cuda)) for _ in range(2)]
    torch.cuda.synchronize()
    for d_r, d_n2 in outs:
        rc = L.vshe_csr_residual_noalloc(A.n, A.nnz, d_rp.data_ptr(), d_ci.data_ptr(), d_v.data_ptr(), d_x.data_ptr(),
                                         d_b.data_ptr(), d_r.data_ptr(), d_n2.data_ptr(), stream.cuda_stream)
        assert rc == 0, gpu.lib().vshe_errstr(rc)
    stream.synchronize()
    for d_r, d_n2 in outs:
        r = d_r.cpu().numpy()
        n2 = d_n2.cpu().numpy()
        assert np.max(np.abs(r - r_ref)) <= 1e-13 * np.max(np.abs(b))
        assert np.all(np.abs(n2 - n2_ref) <= 1e-12 * n2_ref), (n2, n2_ref)


def test_residual_noalloc_rejects_sizes_beyond_its_scratch():
    L = _lib()
    n = 64 * 1024 * 1024 + 1  # one row more than the fixed scratch covers; no pointer is read
    rc = L.vshe_csr_residual_noalloc(n, 1, 1, 1, 1, 1, 1, 1, 1, None)
    assert rc == -14
    assert "scratch capacity" in gpu.lib().vshe_errstr(rc).decode()

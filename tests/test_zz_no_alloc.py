"""sp_ell_pcg_noalloc: the Jacobi-PCG entry point that allocates nothing, for
callers that cannot allocate device memory (code running during CUDA stream
capture, where cudaMalloc is not allowed; serving loops that must stay out of
the allocator; frameworks that own all device memory through their own pool).
Such a caller hands over device buffers it already owns: here torch
allocations stand in for that pool.  The result must match the allocating
entry point sp_ell_dev_pcg on two calls in a row (the fixed work space is
reused, so the second call also checks that each call resets it).

Collected last on purpose (file name), so a run that stops at the first
failure has already run every other test."""
import ctypes as C

import numpy as np
import pytest

import madmax_b200 as mb
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def test_noalloc_pcg_matches_allocating_entry_point():
    import torch

    m = O.cube_mesh(8)
    et = O.fiber_types(m, [1, 1], 0.3)
    E, nu = (1e9, 2e10), (0.3, 0.2)
    A = O.assemble(m, et, E, nu, symmetric_bc=True)
    n, w = A.cols.shape
    B = mb.EllMatrix(n, n, w)
    B.cols[:] = A.cols
    B.vals[:] = A.vals
    h = mb._vp()
    mb.check(mb.lib().sp_ell_upload(C.byref(B.m), C.byref(h)), "sp_ell_upload")
    dev = torch.device("cuda", 0)
    cols_d = torch.tensor(A.cols, dtype=torch.int32, device=dev)
    vals_d = torch.tensor(A.vals, dtype=torch.float64, device=dev)
    rtol = 1e-10
    try:
        for call, strain in enumerate(([1e-3, 2e-4, 0, 0, 1e-4, 0], [0, -5e-4, 3e-4, 2e-3, 0, 1e-3])):
            r, _ = O.residual(m, et, E, nu, O.affine_bc(m, strain))
            b = -r
            x_ref = np.zeros(n)
            its_ref, rel_ref = C.c_int(), C.c_double()
            mb.check(mb.lib().sp_ell_dev_pcg(h, mb.ptr(b), mb.ptr(x_ref), rtol, 5000,
                                             C.byref(its_ref), C.byref(rel_ref)), "sp_ell_dev_pcg")
            b_d = torch.tensor(b, dtype=torch.float64, device=dev)
            x_d = torch.zeros(n, dtype=torch.float64, device=dev)
            torch.cuda.synchronize()
            its, rel = C.c_int(), C.c_double()
            rc = mb.lib().sp_ell_pcg_noalloc(n, w, cols_d.data_ptr(), vals_d.data_ptr(),
                                             b_d.data_ptr(), x_d.data_ptr(), rtol, 5000,
                                             C.byref(its), C.byref(rel), None)
            torch.cuda.synchronize()
            mb.check(rc, "sp_ell_pcg_noalloc")
            x = x_d.cpu().numpy()
            assert rel.value <= rtol, call
            assert abs(its.value - its_ref.value) <= 2, (call, its.value, its_ref.value)
            # same solve up to the summation order of the SpMV: equal to the
            # tolerance the other PCG tests use
            assert np.abs(x - x_ref).max() <= 1e-8 * np.abs(x_ref).max(), call
            assert np.linalg.norm(b - A.mvp(x)) <= 2 * rtol * np.linalg.norm(b), call
    finally:
        mb.lib().sp_ell_dev_free(h)


def test_noalloc_rejects_sizes_beyond_the_work_space():
    big = mb.SP_NOALLOC_MAX_ROWS + 1
    dummy = C.c_void_p(16)
    rc = mb.lib().sp_ell_pcg_noalloc(big, 81, dummy, dummy, dummy, dummy, 1e-8, 10, None, None,
                                     None)
    assert rc == mb.SP_ERR_ARG
    assert "exceed" in mb.last_error()

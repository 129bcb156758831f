"""sp_ell_pcg_noalloc: the Jacobi-PCG entry point that allocates nothing, for
callers that cannot allocate device memory (frameworks that own all device
memory through their own pool; serving loops that must stay out of the CUDA
allocator).  Such a caller hands over device buffers it already owns: here
torch allocations stand in for that pool.  The result must match the
allocating entry point sp_ell_dev_pcg on two calls in a row (the fixed work
space is reused, so the second call also checks that each call resets it).
The error paths (a column index outside the matrix, a zero diagonal) must
be reported, and a good solve right after them must succeed.

Collected last on purpose (file name), so a run that stops at the first
failure has already run every other test."""
import ctypes as C

import numpy as np
import pytest

import madmax_b200 as mb
from oracle import oracle as O

pytestmark = pytest.mark.gpu

E, NU = (1e9, 2e10), (0.3, 0.2)


def system(n_el=8):
    m = O.cube_mesh(n_el)
    et = O.fiber_types(m, [1, 1], 0.3)
    A = O.assemble(m, et, E, NU, symmetric_bc=True)
    return m, et, A


def rhs(m, et, strain):
    r, _ = O.residual(m, et, E, NU, O.affine_bc(m, strain))
    return -r


def noalloc(n, w, cols_d, vals_d, b_d, x_d, rtol, max_its, stream=None):
    its, rel = C.c_int(), C.c_double()
    rc = mb.lib().sp_ell_pcg_noalloc(n, w, cols_d.data_ptr(), vals_d.data_ptr(), b_d.data_ptr(),
                                     x_d.data_ptr(), rtol, max_its, C.byref(its), C.byref(rel),
                                     stream)
    return rc, its.value, rel.value


def test_noalloc_pcg_matches_allocating_entry_point():
    import torch

    m, et, A = system()
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
            b = rhs(m, et, strain)
            x_ref = np.zeros(n)
            its_ref, rel_ref = C.c_int(), C.c_double()
            mb.check(mb.lib().sp_ell_dev_pcg(h, mb.ptr(b), mb.ptr(x_ref), rtol, 5000,
                                             C.byref(its_ref), C.byref(rel_ref)), "sp_ell_dev_pcg")
            b_d = torch.tensor(b, dtype=torch.float64, device=dev)
            x_d = torch.zeros(n, dtype=torch.float64, device=dev)
            torch.cuda.synchronize()
            rc, its, rel = noalloc(n, w, cols_d, vals_d, b_d, x_d, rtol, 5000)
            torch.cuda.synchronize()
            mb.check(rc, "sp_ell_pcg_noalloc")
            x = x_d.cpu().numpy()
            assert rel <= rtol, call
            assert abs(its - its_ref.value) <= 2, (call, its, its_ref.value)
            # same solve up to the summation order of the SpMV: equal to the
            # tolerance the other PCG tests use
            assert np.abs(x - x_ref).max() <= 1e-8 * np.abs(x_ref).max(), call
            assert np.linalg.norm(b - A.mvp(x)) <= 2 * rtol * np.linalg.norm(b), call
    finally:
        mb.lib().sp_ell_dev_free(h)


def test_noalloc_errors_then_recovers_on_a_caller_stream():
    """A column index past the last row is skipped and reported
    (SP_ERR_RANGE), a zero diagonal is reported (SP_ERR_ARG), never a NaN
    success; a good solve right after, on a stream the caller owns, matches
    the oracle (the work space's flags and reduction ticket were reset)."""
    import torch

    m, et, A = system(4)
    n, w = A.cols.shape
    dev = torch.device("cuda", 0)
    b = rhs(m, et, [1e-3, 0, 0, 0, 0, 5e-4])
    b_d = torch.tensor(b, dtype=torch.float64, device=dev)
    vals_d = torch.tensor(A.vals, dtype=torch.float64, device=dev)
    # one padding slot of an interior row points past the matrix (a bad
    # index the kernel must skip, not read)
    bad_cols = A.cols.copy()
    row = n // 2
    slot = int(np.nonzero(bad_cols[row] < 0)[0][0]) if (bad_cols[row] < 0).any() else w - 1
    bad_cols[row, slot] = n + 5
    cols_bad_d = torch.tensor(bad_cols, dtype=torch.int32, device=dev)
    x_d = torch.zeros(n, dtype=torch.float64, device=dev)
    rc, _, _ = noalloc(n, w, cols_bad_d, vals_d, b_d, x_d, 1e-10, 100)
    torch.cuda.synchronize()
    assert rc == mb.SP_ERR_RANGE and "column" in mb.last_error()
    # a row whose diagonal is zero
    zvals = A.vals.copy()
    zvals[row][A.cols[row] == row] = 0.0
    vals_z_d = torch.tensor(zvals, dtype=torch.float64, device=dev)
    cols_d = torch.tensor(A.cols, dtype=torch.int32, device=dev)
    x_d.zero_()
    rc, _, _ = noalloc(n, w, cols_d, vals_z_d, b_d, x_d, 1e-10, 100)
    torch.cuda.synchronize()
    assert rc == mb.SP_ERR_ARG and "diagonal" in mb.last_error()
    # then a good solve on the caller's own stream
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        x_d = torch.zeros(n, dtype=torch.float64, device=dev)
    s.synchronize()
    rc, its, rel = noalloc(n, w, cols_d, vals_d, b_d, x_d, 1e-10, 5000,
                           stream=C.c_void_p(s.cuda_stream))
    s.synchronize()
    mb.check(rc, "sp_ell_pcg_noalloc after errors")
    assert its > 0 and rel <= 1e-10
    x = x_d.cpu().numpy()
    assert np.linalg.norm(b - A.mvp(x)) <= 2e-10 * np.linalg.norm(b)


def test_noalloc_rejects_sizes_beyond_the_work_space():
    big = mb.SP_NOALLOC_MAX_ROWS + 1
    dummy = C.c_void_p(16)
    rc = mb.lib().sp_ell_pcg_noalloc(big, 81, dummy, dummy, dummy, dummy, 1e-8, 10, None, None,
                                     None)
    assert rc == mb.SP_ERR_ARG
    assert "exceed" in mb.last_error()

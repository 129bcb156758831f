"""Parity of the drop-in ell.h compute calls on the GPU (ell_mvp,
ell_solve_jacobi) and of the resident device ELL (sp_ell_dev_*), through the
C ABI, against the reference's own results (golden fixtures made by running
its src/ell.c) and the oracle.  Integer/index work and the reference-order
FP64 calls are checked bit for bit."""
import ctypes as C
import json
import os

import numpy as np
import pytest

import madmax_b200 as mb
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def unhex(v):
    return np.array([float.fromhex(s) for s in v])


def as_lib_matrix(cols, vals, ncol=None):
    nrow, w = cols.shape
    A = mb.EllMatrix(nrow, ncol or nrow, w)
    A.cols[:] = cols
    A.vals[:] = vals
    return A


@pytest.mark.parametrize("n", [1, 2, 3])
def test_ell_mvp_bit_exact_vs_reference(golden_dir, n):
    g = np.load(os.path.join(golden_dir, "ell3d.npz"))
    A = as_lib_matrix(g[f"n{n}_cols"], g[f"n{n}_vals_bc"])
    y = A.mvp(g[f"n{n}_x"])
    assert np.array_equal(y, g[f"n{n}_y"])


def test_ell_mvp_ragged_rows_bit_exact():
    """Rows of different fill, empty rows, widths above one warp."""
    rng = np.random.default_rng(3)
    for nrow, w in ((1, 1), (7, 5), (300, 33), (1000, 81), (64, 100)):
        A = O.EllMatrix(nrow, nrow, w)
        for i in range(nrow):
            k = rng.integers(0, w + 1)
            A.cols[i, :k] = rng.choice(nrow, size=k, replace=k > nrow)
            A.vals[i, :k] = rng.standard_normal(k)
        x = rng.standard_normal(nrow)
        B = as_lib_matrix(A.cols.copy(), A.vals.copy())
        assert np.array_equal(B.mvp(x), A.mvp(x))


def test_ell_mvp_empty_matrix_and_null():
    A = mb.EllMatrix(4, 4, 3)
    assert np.array_equal(A.mvp(np.ones(4)), np.zeros(4))
    assert mb.lib().ell_mvp(C.byref(A.m), None, None) == 1


def test_ell_solve_jacobi_unity(golden_dir):
    """unity/unity_ell.c on the GPU: 388 iterations, x and err bit-exact."""
    d = json.load(open(os.path.join(golden_dir, "unity_ell.json")))["defined_inputs"]
    A = as_lib_matrix(np.array(d["cols"], dtype=np.int32), unhex(d["vals"]).reshape(10, 4))
    x, its, err = A.solve_jacobi(unhex(d["b"]), unhex(d["x0"]))
    assert its == d["its"] == 388
    assert np.array_equal(x, unhex(d["x"]))
    assert err == float.fromhex(d["err"])


def test_ell_solve_jacobi_bit_exact_vs_oracle():
    from tests.test_oracle_golden import dominant_ell, _orc_jacobi
    A = dominant_ell(n=2000, width=12, seed=11)
    b = np.random.default_rng(5).standard_normal(A.nrow)
    x0 = np.random.default_rng(6).standard_normal(A.nrow)
    xo = x0.copy()
    its_o, err_o = _orc_jacobi(A, b, xo)
    B = as_lib_matrix(A.cols.copy(), A.vals.copy())
    x, its, err = B.solve_jacobi(b, x0)
    assert its == its_o and err == err_o
    assert np.array_equal(x, xo)


def test_ell_dev_mvp_and_pcg():
    m = O.cube_mesh(8)
    et = O.fiber_types(m, [1, 1], 0.3)
    E, nu = (1e9, 2e10), (0.3, 0.2)
    A = O.assemble(m, et, E, nu, symmetric_bc=True)
    B = as_lib_matrix(A.cols.copy(), A.vals.copy())
    h = mb._vp()
    mb.check(mb.lib().sp_ell_upload(C.byref(B.m), C.byref(h)), "upload")
    try:
        x = np.random.default_rng(2).standard_normal(m.ndof)
        y = np.zeros(m.ndof)
        mb.check(mb.lib().sp_ell_dev_mvp_host(h, mb.ptr(x), mb.ptr(y)), "mvp")
        yo = A.mvp(x)
        assert np.abs(y - yo).max() <= 1e-13 * np.abs(yo).max()
        r, _ = O.residual(m, et, E, nu, O.affine_bc(m, [1e-3, 2e-4, 0, 0, 1e-4, 0]))
        b = -r
        xg = np.zeros(m.ndof)
        its, rel = C.c_int(), C.c_double()
        mb.check(mb.lib().sp_ell_dev_pcg(h, mb.ptr(b), mb.ptr(xg), 1e-10, 5000, C.byref(its),
                                         C.byref(rel)), "pcg")
        true_rel = np.linalg.norm(b - A.mvp(xg)) / np.linalg.norm(b)
        assert rel.value <= 1e-10 and true_rel <= 2e-10
        xo = np.zeros(m.ndof)
        ito, relo = C.c_int(), C.c_double()
        O.lib().orc_pcg(C.byref(A.s), O.ptr(b), O.ptr(xo), 1e-10, 5000, C.byref(ito),
                        C.byref(relo))
        assert abs(its.value - ito.value) <= 2
        assert np.abs(xg - xo).max() <= 1e-8 * np.abs(xo).max()
    finally:
        mb.lib().sp_ell_dev_free(h)


@pytest.mark.parametrize("lanes", [0, 4, 8, 16, 32])
def test_ell_dev_mvp_every_lane_width(lanes):
    """The resident SpMV at every lanes-per-row setting matches the
    reference-order product within rounding; true_nnz counts stored slots."""
    m = O.cube_mesh(6)
    et = O.fiber_types(m, [1, 1], 0.25)
    A = O.assemble(m, et, (1e9, 3e10), (0.3, 0.2), symmetric_bc=True)
    B = as_lib_matrix(A.cols.copy(), A.vals.copy())
    h = mb._vp()
    mb.check(mb.lib().sp_ell_upload(C.byref(B.m), C.byref(h)), "upload")
    try:
        mb.check(mb.lib().sp_ell_dev_set_lanes(h, lanes), "lanes")
        nrow, wp, nnz = C.c_int(), C.c_int(), C.c_longlong()
        mb.check(mb.lib().sp_ell_dev_info(h, C.byref(nrow), C.byref(wp), C.byref(nnz)), "info")
        assert nrow.value == m.ndof and wp.value == 84
        assert nnz.value == int((A.cols >= 0).sum())
        x = np.random.default_rng(lanes).standard_normal(m.ndof)
        y = np.zeros(m.ndof)
        mb.check(mb.lib().sp_ell_dev_mvp_host(h, mb.ptr(x), mb.ptr(y)), "mvp")
        yo = A.mvp(x)
        assert np.abs(y - yo).max() <= 1e-13 * np.abs(yo).max()
        assert mb.lib().sp_ell_dev_set_lanes(h, 3) == mb.SP_ERR_ARG
        used = C.c_int()
        mb.check(mb.lib().sp_ell_dev_lanes(h, C.byref(used), None, None), "lanes")
        assert used.value == lanes if lanes else used.value in (4, 8, 16, 32)
    finally:
        mb.lib().sp_ell_dev_free(h)


def test_ell_upload_autotunes_lanes_and_caches_the_choice():
    """sp_ell_upload times every lanes-per-row width on the uploaded matrix
    and keeps the fastest; a like matrix (same row width, same row-count
    octave) takes the cached choice without a trial."""
    m = O.cube_mesh(12)
    et = O.fiber_types(m, [1, 1], 0.3)
    A = O.assemble(m, et, (1e9, 2e10), (0.3, 0.2), symmetric_bc=True)
    handles = []
    try:
        reports = []
        for _ in range(2):
            B = as_lib_matrix(A.cols.copy(), A.vals.copy())
            h = mb._vp()
            mb.check(mb.lib().sp_ell_upload(C.byref(B.m), C.byref(h)), "upload")
            handles.append(h)
            lanes, cached = C.c_int(), C.c_int()
            us = (C.c_float * 4)()
            mb.check(mb.lib().sp_ell_dev_lanes(h, C.byref(lanes), us, C.byref(cached)), "lanes")
            reports.append((lanes.value, list(us), cached.value))
        (l0, us0, c0), (l1, us1, c1) = reports
        assert l0 in (4, 8, 16, 32) and all(t > 0 for t in us0)
        # the chosen width is the fastest of the trial
        assert us0[(4, 8, 16, 32).index(l0)] == min(us0)
        assert c1 == 1 and l1 == l0 and us1 == us0
        x = np.random.default_rng(3).standard_normal(m.ndof)
        y = np.zeros(m.ndof)
        mb.check(mb.lib().sp_ell_dev_mvp_host(handles[1], mb.ptr(x), mb.ptr(y)), "mvp")
        yo = A.mvp(x)
        assert np.abs(y - yo).max() <= 1e-13 * np.abs(yo).max()
    finally:
        for h in handles:
            mb.lib().sp_ell_dev_free(h)


def test_reference_unity_program_linked_to_library(golden_dir, tmp_path):
    """The reference's unity/unity_ell.c, compiled unchanged against
    include/ell.h and linked to libsputnik_b200.so (oracle/Makefile target
    dropin), prints what the reference build prints."""
    import subprocess
    exe = os.path.join(os.path.dirname(O.LIB_PATH), "_ref", "unity_ell_b200")
    if not os.path.exists(exe):
        pytest.skip("drop-in build of unity_ell.c not present")
    out = subprocess.run([exe], cwd=tmp_path, capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stderr
    d = json.load(open(os.path.join(golden_dir, "unity_ell.json")))
    lines = out.stdout.splitlines()
    i0 = lines.index("m=")
    mat = [[float(v) for v in ln.split()] for ln in lines[i0 + 1:i0 + 11]]
    assert mat == d["printed_matrix"]
    assert int([ln for ln in lines if ln.startswith("its")][0].split("=")[1]) == 388
    x = [float(v) for v in open(tmp_path / "sol.dat").read().split()]
    assert x == d["printed_x"]

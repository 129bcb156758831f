"""Pins the CPU oracle (oracle/oracle.c) to the reference: its own compiled
ell.c/fem.c (oracle/_ref, when present), its unity_ell test program's output
and the 2D tensor of exs/README.md.  CPU only."""
import json
import os

import numpy as np
import pytest

from oracle import oracle as O


def unhex(v):
    return np.array([float.fromhex(s) for s in v])


@pytest.fixture(scope="module")
def unity(golden_dir):
    return json.load(open(os.path.join(golden_dir, "unity_ell.json")))


def build_unity_oracle():
    """unity/unity_ell.c:14-31 with the oracle's ELL functions."""
    n = 10
    A = O.EllMatrix(n, n, 4)
    me = np.array([1, -1, -1, 1], dtype=np.float64)
    b = np.zeros(n)
    for i in range(n - 1):
        b[i] = 1.0
        ix = np.array([i, i + 1], dtype=np.int32)
        O.lib().orc_ell_add_vals(O.C.byref(A.s), O.ptr(ix, O._ip), 2, O.ptr(ix, O._ip), 2,
                                 O.ptr(me))
    L = O.lib()
    L.orc_ell_set_zero_row.argtypes = [O.C.POINTER(O.Ell), O.C.c_int, O.C.c_double]
    L.orc_ell_set_zero_col_ref.argtypes = [O.C.POINTER(O.Ell), O.C.c_int, O.C.c_double]
    L.orc_ell_set_zero_row(O.C.byref(A.s), 0, 1.0)
    L.orc_ell_set_zero_row(O.C.byref(A.s), n - 1, 1.0)
    L.orc_ell_set_zero_col_ref(O.C.byref(A.s), 0, 1.0)
    L.orc_ell_set_zero_col_ref(O.C.byref(A.s), n - 1, 1.0)
    return A, b


def test_unity_ell_matrix_and_jacobi(unity):
    A, b = build_unity_oracle()
    d = unity["defined_inputs"]
    assert A.cols.tolist() == d["cols"]
    assert np.array_equal(A.vals.ravel(), unhex(d["vals"]))
    # printed matrix of the reference program, including the -1 that the
    # early-returning ell_set_zero_col leaves in row 1, column 0
    dense = np.zeros((10, 10))
    for i in range(10):
        for j in range(4):
            if A.cols[i, j] >= 0:
                dense[i, A.cols[i, j]] = A.vals[i, j]
    assert dense.tolist() == unity["printed_matrix"]
    assert dense[1, 0] == -1.0
    x = np.zeros(10)
    its = O.C.c_int()
    err = O.C.c_double()
    O.lib().orc_jacobi(O.C.byref(A.s), O.ptr(b), O.ptr(x), 100000, 1e-10, O.C.byref(its),
                       O.C.byref(err))
    assert its.value == d["its"] == unity["printed_its"] == 388
    assert np.array_equal(x, unhex(d["x"]))
    assert err.value == float.fromhex(d["err"])
    assert np.allclose(x, unity["printed_x"], atol=5e-7)


def test_hexa8_tables_match_reference(golden_dir):
    g = np.load(os.path.join(golden_dir, "fem_tables.npz"))
    xp, sh, ds = np.zeros(24), np.zeros(64), np.zeros(192)
    O.lib().orc_hexa8_tables(O.ptr(xp), O.ptr(sh), O.ptr(ds))
    assert np.array_equal(xp.reshape(8, 3), g["xp_hexa_8"])
    assert np.array_equal(sh.reshape(8, 8), g["sh_hexa_8"])
    assert np.array_equal(ds.reshape(8, 3, 8), g["ds_hexa_8"])


def test_struct_2d_tables_match_reference(golden_dir):
    g = np.load(os.path.join(golden_dir, "fem_tables.npz"))
    for tag in ("a", "b"):
        h = g[f"struct2d_{tag}_h"]
        m = O.mesh(2, [3, 3], [2 * h[0], 2 * h[1]])
        dsh, wp = np.zeros(32), np.zeros(4)
        O.lib().orc_struct_dsh(O.C.byref(m), O.ptr(dsh), O.ptr(wp))
        assert np.array_equal(dsh.reshape(4, 2, 4), g[f"struct2d_{tag}_dsh"])
        assert np.array_equal(wp, g[f"struct2d_{tag}_wp"])


@pytest.mark.parametrize("n", [1, 2, 3])
def test_ell3d_assembly_bit_exact(golden_dir, n):
    g = np.load(os.path.join(golden_dir, "ell3d.npz"))
    m = O.cube_mesh(n)
    et = g[f"n{n}_etype"]
    assert np.array_equal(O.fiber_types(m, [1.0, 1.0], 0.3 if n > 1 else 0.1), et)
    A = O.assemble(m, et, (1e9, 1e10), (0.3, 0.2), symmetric_bc=False)
    assert np.array_equal(A.cols, g[f"n{n}_cols"])
    assert np.array_equal(A.vals, g[f"n{n}_vals_bc"])
    assert np.array_equal(A.mvp(g[f"n{n}_x"]), g[f"n{n}_y"])


@pytest.mark.parametrize("n", [2, 3])
def test_symmetric_bc_same_solution(n):
    """Deviation D1: clearing the boundary columns in every row (needed by
    CG) leaves the Newton correction unchanged."""
    m = O.cube_mesh(n)
    et = O.fiber_types(m, [1.0, 1.0], 0.3)
    E, nu = (1e9, 1e10), (0.3, 0.2)
    u0 = O.affine_bc(m, [1e-3, 0, 0, 5e-4, 0, 0])
    r, _ = O.residual(m, et, E, nu, u0)
    b = -r
    xs = []
    for sym in (False, True):
        A = O.assemble(m, et, E, nu, symmetric_bc=sym)
        dense = np.zeros((m.ndof, m.ndof))
        for i in range(m.ndof):
            for j in range(81):
                c = A.cols[i, j]
                if c >= 0:
                    dense[i, c] += A.vals[i, j]
        xs.append(np.linalg.solve(dense, b))
        if sym:
            assert np.allclose(dense, dense.T, rtol=0, atol=1e-6 * np.abs(dense).max())
    assert np.allclose(xs[0], xs[1], rtol=1e-10, atol=1e-14)


def test_readme_2d_tensor(golden_dir):
    """exs/README.md:154-157 -- reproduced at fiber radius 0.9."""
    d = json.load(open(os.path.join(golden_dir, "readme_2d.json")))
    m = O.mesh(2, d["struct_n_nodes"], d["size"])
    et = O.fiber_types(m, d["size"], d["reproducing_radius"])
    C6, _ = O.fd_tangent(m, et, (1e6, 1e7), (0.3, 0.3), [0, 0, 0], rtol=1e-10, lin_rtol=1e-11)
    ref = np.array(d["C"])
    nz = ref != 0
    rel = np.abs(C6[nz] - ref[nz]) / np.abs(ref[nz])
    assert rel.max() < 5e-4, rel
    # C11 and C21 agree to the printed precision
    assert rel[0] < 1e-6 and rel[2] < 1e-6


def test_oracle_pcg_true_residual():
    m = O.cube_mesh(6)
    et = O.fiber_types(m, [1, 1], 0.3)
    sa, st, u, stats = O.homogenize(m, et, (1e9, 5e10), (0.3, 0.25),
                                    [[1e-3, 0, 0, 0, 0, 0], [0, 0, 0, 2e-3, 0, 0]], want_u=True)
    assert (stats[:, 2] <= 1e-8).all()
    # strain average equals the applied macro strain (affine boundary data)
    assert np.allclose(sa[0], [1e-3, 0, 0, 0, 0, 0], atol=1e-12)
    assert np.allclose(sa[1], [0, 0, 0, 2e-3, 0, 0], atol=1e-12)


def _ref_jacobi(A, b, x):
    import ctypes as C
    R = O.ref()

    class Solver(C.Structure):
        _fields_ = [("max_its", C.c_int), ("its", C.c_int), ("min_err", C.c_double),
                    ("err", C.c_double)]

    R.ell_solve_jacobi.argtypes = [C.POINTER(Solver), C.POINTER(O.Ell), O._dp, O._dp]
    s = Solver()
    R.ell_solve_jacobi(C.byref(s), C.byref(A.s), O.ptr(b), O.ptr(x))
    return s.its, s.err


def _orc_jacobi(A, b, x):
    import ctypes as C
    its, err = C.c_int(), C.c_double()
    O.lib().orc_jacobi(C.byref(A.s), O.ptr(b), O.ptr(x), 100000, 1e-10, C.byref(its),
                       C.byref(err))
    return its.value, err.value


def dominant_ell(n=300, width=9, seed=7):
    """Random diagonally dominant ELL matrix (stationary Jacobi converges)."""
    rng = np.random.default_rng(seed)
    A = O.EllMatrix(n, n, width)
    import ctypes as C
    for i in range(n):
        cols = rng.choice(n, size=width - 1, replace=False)
        cols = cols[cols != i][: width - 2]
        vals = rng.uniform(-1, 1, size=len(cols))
        O.lib().orc_ell_add_val.argtypes = [C.POINTER(O.Ell), C.c_int, C.c_int, C.c_double]
        O.lib().orc_ell_add_val(C.byref(A.s), i, i, float(np.abs(vals).sum() * 1.5 + 0.1))
        for c, v in zip(cols, vals):
            O.lib().orc_ell_add_val(C.byref(A.s), i, int(c), float(v))
    return A


def test_oracle_jacobi_matches_reference_library():
    """Stationary Jacobi (src/ell.c:143-184): oracle == reference bit for bit."""
    if not O.ref_available():
        pytest.skip("reference library not built here")
    A = dominant_ell()
    b = np.random.default_rng(1).standard_normal(A.nrow)
    x1, x2 = np.zeros(A.nrow), np.zeros(A.nrow)
    r1 = _ref_jacobi(A, b, x1)
    r2 = _orc_jacobi(A, b, x2)
    assert r1 == r2 and r1[0] < 100000
    assert np.array_equal(x1, x2)


def test_reference_jacobi_diverges_on_hex8_elasticity():
    """The reference's ELL solver is a stationary Jacobi iteration; on the 3D
    hex8 elasticity operator its iteration matrix has spectral radius > 1 and
    the iterate overflows to NaN (same in the oracle).  This is why the hot
    path uses Jacobi-preconditioned CG (the reference's PETSc route)."""
    m = O.cube_mesh(3)
    et = O.fiber_types(m, [1, 1], 0.3)
    A = O.assemble(m, et, (1.0, 3.0), (0.3, 0.2), symmetric_bc=False)
    r, _ = O.residual(m, et, (1.0, 3.0), (0.3, 0.2), O.affine_bc(m, [1e-1, 0, 0, 0, 0, 0]))
    x = np.zeros(m.ndof)
    its, err = _orc_jacobi(A, -r, x)
    assert its == 100000 and not np.isfinite(err)
    if O.ref_available():
        x1 = np.zeros(m.ndof)
        its1, err1 = _ref_jacobi(A, -r, x1)
        assert its1 == its and np.array_equal(np.isnan(x1), np.isnan(x))

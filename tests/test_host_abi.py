"""Host side of the C ABI, on the CPU: the library loads and exports every
symbol include/*.h declares; the drop-in ELL container and fem tables behave
bit for bit like the reference's (its own ell.c/fem.c compiled from source,
or the committed fixtures); integer set-up (ELL pattern, classification,
admission budget) matches the oracle.  No compute call reaches a GPU here."""
import ctypes as C
import os
import re

import numpy as np
import pytest

import madmax_b200 as mb
from oracle import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for h in ("ell.h", "fem.h", "solvers.h", "sputnik_b200.h"):
        txt = open(os.path.join(ROOT, "include", h)).read()
        txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
        txt = re.sub(r"#ifdef PETSC.*?#endif", "", txt, flags=re.S)
        # function-pointer typedefs declare no symbol
        txt = re.sub(r"^\s*typedef\s+\w+\s*\(\s*\*\s*\w+\s*\)\s*\([^;]*;", "", txt, flags=re.M)
        names |= set(re.findall(r"^\s*(?:const\s+)?[\w]+\s*\**\s*(\w+)\s*\(", txt, flags=re.M))
        names |= set(re.findall(r"^extern\s+[\w\s\*]+?\b(\w+)\s*;", txt, flags=re.M))
    return names


def test_library_exports_every_declared_symbol():
    L = mb.load()
    assert mb.MISSING == []
    names = declared_symbols()
    assert {"ell_mvp", "fem_init", "sp_batch_launch", "sp_server_replay", "xp_hexa_8",
            "solver", "sp_fe2_run", "sp_micro_serve", "sp_vtu_write", "sp_rve_fields"} <= names
    assert "int" not in names
    missing = [n for n in sorted(names) if not hasattr(L, n)]
    assert missing == []


def ref_or_skip():
    if not O.ref_available():
        pytest.skip("reference library not built here")
    return O.ref()


def test_ell_container_ops_match_reference_library():
    """Random sequences of ell_set/add/get/zero calls on the drop-in and on
    the reference's src/ell.c: same arrays, same return codes."""
    R = ref_or_skip()
    R.ell_set_val.argtypes = [C.POINTER(O.Ell), C.c_int, C.c_int, C.c_double]
    R.ell_add_val.argtypes = [C.POINTER(O.Ell), C.c_int, C.c_int, C.c_double]
    R.ell_get_val.argtypes = [C.POINTER(O.Ell), C.c_int, C.c_int, O._dp]
    L = mb.lib()
    rng = np.random.default_rng(0)
    n, w = 12, 5
    a = O.Ell()
    R.ell_init(C.byref(a), n, n, w)
    b = mb.EllMatrix(n, n, w)
    for _ in range(3000):
        op = rng.integers(0, 7)
        i, j = int(rng.integers(-1, n + 1)), int(rng.integers(-1, n + 1))
        v = float(rng.standard_normal())
        if op == 0:
            r1 = R.ell_set_val(C.byref(a), i, j, v)
            r2 = L.ell_set_val(C.byref(b.m), i, j, v)
        elif op in (1, 2):
            r1 = R.ell_add_val(C.byref(a), i, j, v)
            r2 = L.ell_add_val(C.byref(b.m), i, j, v)
        elif op == 3:
            x1, x2 = C.c_double(7.0), C.c_double(7.0)
            r1 = R.ell_get_val(C.byref(a), i, j, C.byref(x1))
            r2 = L.ell_get_val(C.byref(b.m), i, j, C.byref(x2))
            assert x1.value == x2.value
        elif op == 4 and 0 <= i < n:
            r1 = R.ell_set_zero_row(C.byref(a), i, v)
            r2 = L.ell_set_zero_row(C.byref(b.m), i, v)
        elif op == 5 and 0 <= i < n:
            r1 = R.ell_set_zero_col(C.byref(a), i, v)
            r2 = L.ell_set_zero_col(C.byref(b.m), i, v)
        elif op == 6 and rng.random() < 0.01:
            r1 = R.ell_set_zero_mat(C.byref(a))
            r2 = L.ell_set_zero_mat(C.byref(b.m))
        else:
            continue
        assert r1 == r2
    assert np.array_equal(np.ctypeslib.as_array(a.cols, shape=(n, w)), b.cols)
    assert np.array_equal(np.ctypeslib.as_array(a.vals, shape=(n, w)), b.vals)


def test_ell_add_vals_assembly_matches_golden(golden_dir):
    """3D element loop through the drop-in ell_add_vals: reference cols/vals."""
    g = np.load(os.path.join(golden_dir, "ell3d.npz"))
    for n in (1, 2, 3):
        m = O.cube_mesh(n)
        et = g[f"n{n}_etype"]
        _, Ke, _, _ = O.operators(m, (1e9, 1e10), (0.3, 0.2))
        A = mb.EllMatrix(m.ndof, m.ndof, 81)
        mb.lib().ell_set_zero_mat(C.byref(A.m))
        for e, idx in enumerate(O.elem_dofs(m)):
            assert A.add_vals(idx, idx, Ke[et[e]].ravel()) == 0
        assert np.array_equal(A.cols, g[f"n{n}_cols"])
        assert np.array_equal(A.vals, g[f"n{n}_vals_raw"])
        for node in O.boundary_nodes(m):
            for d in range(3):
                mb.lib().ell_set_zero_row(C.byref(A.m), int(node) * 3 + d, 1.0)
                mb.lib().ell_set_zero_col(C.byref(A.m), int(node) * 3 + d, 1.0)
        assert np.array_equal(A.vals, g[f"n{n}_vals_bc"])


def fem_table(name, npe, dim, ngp):
    L = mb.lib()
    xp = C.POINTER(C.POINTER(C.c_double)).in_dll(L, f"xp_{name}")
    wp = C.POINTER(C.c_double).in_dll(L, f"wp_{name}")
    sh = C.POINTER(C.POINTER(C.c_double)).in_dll(L, f"sh_{name}")
    ds = C.POINTER(C.POINTER(C.POINTER(C.c_double))).in_dll(L, f"ds_{name}")
    return (np.array([[xp[g][d] for d in range(dim)] for g in range(ngp)]),
            np.array([wp[g] for g in range(ngp)]),
            np.array([[sh[a][g] for g in range(ngp)] for a in range(npe)]),
            np.array([[[ds[a][d][g] for g in range(ngp)] for d in range(dim)] for a in range(npe)]))


def test_fem_tables_bit_exact(golden_dir):
    gold = np.load(os.path.join(golden_dir, "fem_tables.npz"))
    assert mb.lib().fem_init() == 0
    for name, dims in {"segm_2": (2, 1, 2), "tria_3": (3, 2, 3), "quad_4": (4, 2, 4),
                       "tetra_4": (4, 3, 4), "prism_6": (6, 3, 6), "hexa_8": (8, 3, 8)}.items():
        xp, wp, sh, ds = fem_table(name, *dims)
        assert np.array_equal(xp, gold[f"xp_{name}"]), name
        assert np.array_equal(wp, gold[f"wp_{name}"]), name
        assert np.array_equal(sh, gold[f"sh_{name}"]), name
        assert np.array_equal(ds, gold[f"ds_{name}"]), name


def struct_tables(h, dim):
    shp = C.POINTER(C.POINTER(C.c_double))()
    dshp = C.POINTER(C.POINTER(C.POINTER(C.c_double)))()
    wpp = C.POINTER(C.c_double)()
    hh = np.array(list(h) + [1.0] * (3 - len(h)))
    assert mb.lib().fem_init_struct(C.byref(shp), C.byref(dshp), C.byref(wpp), mb.ptr(hh), dim) == 0
    npe = 4 if dim == 2 else 8
    dsh = np.array([[[dshp[a][d][g] for g in range(npe)] for d in range(dim)] for a in range(npe)])
    wp = np.array([wpp[g] for g in range(npe)])
    return dsh, wp


def test_fem_init_struct_2d_bit_exact_and_3d_filled(golden_dir):
    gold = np.load(os.path.join(golden_dir, "fem_tables.npz"))
    for tag in ("a", "b"):
        dsh, wp = struct_tables(gold[f"struct2d_{tag}_h"], 2)
        assert np.array_equal(dsh, gold[f"struct2d_{tag}_dsh"])
        assert np.array_equal(wp, gold[f"struct2d_{tag}_wp"])
    # 3D (empty in the reference): equals the oracle's hexa8 restatement
    m = O.mesh(3, [4, 5, 6], [0.75, 1.0, 1.25])
    dsh, wp = struct_tables((m.hx, m.hy, m.hz), 3)
    od, ow = np.zeros(192), np.zeros(8)
    O.lib().orc_struct_dsh(C.byref(m), O.ptr(od), O.ptr(ow))
    assert np.array_equal(dsh, od.reshape(8, 3, 8)) and np.array_equal(wp, ow)


def test_fem_jacobian_helpers_match_reference():
    R = ref_or_skip()
    L = mb.lib()
    rng = np.random.default_rng(4)
    for dim in (2, 3):
        def mat():
            rows = [(C.c_double * dim)(*rng.standard_normal(dim)) for _ in range(dim)]
            return (C.POINTER(C.c_double) * dim)(*[C.cast(r, C.POINTER(C.c_double)) for r in rows]), rows
        jac, keep1 = mat()
        i1, k2 = mat()
        i2, k3 = mat()
        d1, d2 = C.c_double(), C.c_double()
        R.fem_invjac.argtypes = [C.c_int, C.c_void_p, C.c_void_p, O._dp]
        R.fem_invjac(dim, C.cast(jac, C.c_void_p), C.cast(i1, C.c_void_p), C.byref(d1))
        L.fem_invjac(dim, C.cast(jac, C.c_void_p), C.cast(i2, C.c_void_p), C.byref(d2))
        assert d1.value == d2.value
        assert all(i1[r][c] == i2[r][c] for r in range(dim) for c in range(dim))


def test_ell_pattern_matches_reference_and_oracle(golden_dir):
    g = np.load(os.path.join(golden_dir, "ell3d.npz"))
    for n in (1, 2, 3):
        assert np.array_equal(mb.ell_pattern(n), g[f"n{n}_cols"])
    for n in ((4, 4, 4), (2, 5, 3)):
        m = O.mesh(3, [k + 1 for k in n], [1, 1, 1])
        A = O.assemble(m, np.zeros(m.nelm, dtype=np.uint8), (1, 2), (0.3, 0.3))
        assert np.array_equal(mb.ell_pattern(n), A.cols)


@pytest.mark.parametrize("n,r,nfib,desv", [(10, 0.25, (1, 1), (0, 0)), (20, 0.35, (1, 1), (0, 0)),
                                          (16, 0.1, (2, 2), (0.05, 0.0)), (9, 0.5, (1, 1), (0.1, -0.1))])
def test_classification_bit_exact(n, r, nfib, desv):
    d = mb.rve_desc(n, r, nfib=nfib, desv=desv)
    m = O.cube_mesh(n)
    assert np.array_equal(mb.classify(d), O.fiber_types(m, [1, 1], r, nfib=nfib, desv=desv))


def test_server_budget_accounting():
    descs = (mb.sp_rve_desc * 4)(*[mb.rve_desc(n) for n in (8, 12, 16, 20)])
    o = mb.server_opts()
    b = C.c_size_t()
    mb.check(mb.lib().sp_server_plan_bytes(4, descs, C.byref(o), C.byref(b)), "plan_bytes")
    assert b.value > 4 * 3 * 21 ** 3 * 84 * 4  # at least the FP32 matrices
    o.hbm_budget = 10 * 1000 * 1000  # 10 MB: cannot hold the geometries
    rc = mb.lib().sp_server_plan_bytes(4, descs, C.byref(o), C.byref(b))
    assert rc == mb.SP_ERR_BUDGET and "budget" in mb.last_error()


def test_no_device_no_fallback():
    if mb.device_count() > 0:
        pytest.skip("a GPU is present")
    A = mb.EllMatrix(4, 4, 2)
    x = np.ones(4)
    y = np.zeros(4)
    assert mb.lib().ell_mvp(C.byref(A.m), mb.ptr(x), mb.ptr(y)) == mb.ELL_ERR_CUDA
    h = mb._vp()
    assert mb.lib().sp_rve_create(C.byref(mb.rve_desc(2)), C.byref(h)) == mb.SP_ERR_CUDA
    assert "CUDA" in mb.last_error() or "device" in mb.last_error()


@pytest.mark.parametrize("compiler,std", [("gcc", "-std=c11"), ("g++", "-std=c++17")])
def test_public_headers_compile_standalone(tmp_path, compiler, std):
    """Each public header is self-contained C (and C++): a translation unit
    that includes only it compiles without warnings."""
    import shutil
    import subprocess
    if not shutil.which(compiler):
        pytest.skip(f"{compiler} not found")
    for h in ("ell.h", "fem.h", "solvers.h", "sputnik_b200.h"):
        src = tmp_path / ("inc.c" if compiler == "gcc" else "inc.cpp")
        src.write_text(f'#include "{h}"\nint sp_header_probe(void) {{ return 0; }}\n')
        r = subprocess.run([compiler, std, "-Wall", "-Wextra", "-Werror", "-fsyntax-only",
                            "-I", os.path.join(ROOT, "include"), str(src)],
                           capture_output=True, text=True)
        assert r.returncode == 0, (h, r.stderr[-2000:])


def test_solvers_header_includes_slepc_under_dslepc(tmp_path):
    """The macro program is built with -DSLEPC and declares its EPS solver
    through solvers.h (inc/solvers.h:20-22, macro/inc/macro.h:12): with
    -DSLEPC the header pulls in slepceps.h, found first on the caller's
    include path (here a stub that defines EPS)."""
    import shutil
    import subprocess
    if not shutil.which("gcc"):
        pytest.skip("gcc not found")
    stub = tmp_path / "stub"
    stub.mkdir()
    (stub / "slepceps.h").write_text("typedef struct sp_stub_eps *EPS;\n")
    src = tmp_path / "macro_like.c"
    src.write_text('#include "solvers.h"\nEPS eps;\nsolver_t solver;\n'
                   "int sp_probe(void) { return eps == 0 && solver.type == SOLVER_NULL; }\n")
    inc = ["-I", os.path.join(ROOT, "include"), "-I", str(stub)]
    ok = subprocess.run(["gcc", "-std=gnu11", "-Wall", "-Werror", "-DSLEPC", "-fsyntax-only"] +
                        inc + [str(src)], capture_output=True, text=True)
    assert ok.returncode == 0, ok.stderr[-2000:]
    # without -DSLEPC the stub is not included, so EPS is unknown
    no = subprocess.run(["gcc", "-std=gnu11", "-fsyntax-only"] + inc + [str(src)],
                        capture_output=True, text=True)
    assert no.returncode != 0 and "EPS" in no.stderr
